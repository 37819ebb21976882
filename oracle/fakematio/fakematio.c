/* fakematio: a MAT level-5 reader behind the libmatio calls of the
 * reference's loader (src/graph.c:38-128).  TEST INFRASTRUCTURE ONLY.
 *
 * Files are mapped read-only.  A MAT file is a 128-byte header followed by
 * data elements; each top-level element is a miMATRIX, possibly wrapped in
 * miCOMPRESSED (zlib).  Inside a miMATRIX come the array flags (class in
 * the low byte), the dimensions, the name, then per class: for sparse the
 * row indices (ir), the column starts (jc) and the values (skipped: the
 * loader reads the pattern only); for struct the field-name length, the
 * names and one miMATRIX per field per element.  Any integer storage type
 * of ir/jc/dims is accepted.  Big-endian files are refused.
 *
 * A file that starts with "CSRB" is the CSR binary format (magic, version
 * u32 = 1, n u32, pad u32, m u64, row_ptr u64[n+1], col u32[m]); it is
 * served as one n x n sparse variable "A" whose column starts are the row
 * pointers and whose row indices are the columns, which for a symmetric
 * graph is the same matrix.  It needs m < 2^32, the limit of the 32-bit
 * column starts. */
#define _GNU_SOURCE
#include "matio.h"

#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

enum { miINT8 = 1, miUINT8, miINT16, miUINT16, miINT32, miUINT32, miSINGLE, miRES8, miDOUBLE,
       miRES10, miRES11, miINT64, miUINT64, miMATRIX, miCOMPRESSED };

struct mat_t {
    unsigned char *map;
    size_t size;
    size_t pos;
    int csrbin;
    int served;
};

typedef struct {
    int nfields;
    matvar_t **fields; /* nel * nfields */
    size_t nel;
} struct_data;

typedef struct {
    int owns_ir, owns_jc;
} sparse_own;

mat_t *Mat_Open(const char *matname, int mode)
{
    (void)mode;
    int fd = open(matname, O_RDONLY);
    if (fd < 0)
        return NULL;
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size < 8) {
        close(fd);
        return NULL;
    }
    void *p = mmap(NULL, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (p == MAP_FAILED)
        return NULL;
    mat_t *m = (mat_t *)calloc(1, sizeof(mat_t));
    if (!m) {
        munmap(p, (size_t)st.st_size);
        return NULL;
    }
    m->map = (unsigned char *)p;
    m->size = (size_t)st.st_size;
    if (memcmp(m->map, "CSRB", 4) == 0) {
        m->csrbin = 1;
        return m;
    }
    if (m->size < 128 || m->map[126] != 'I' || m->map[127] != 'M') {
        fprintf(stderr, "fakematio: %s is not a little-endian MAT level-5 file\n", matname);
        munmap(p, m->size);
        free(m);
        return NULL;
    }
    m->pos = 128;
    return m;
}

int Mat_Close(mat_t *mat)
{
    if (!mat)
        return 0;
    munmap(mat->map, mat->size);
    free(mat);
    return 0;
}

/* One element inside buf[0, len): its type, payload and the next offset. */
static int next_el(const unsigned char *buf, size_t len, size_t *off, uint32_t *type,
                   const unsigned char **data, uint32_t *nbytes)
{
    if (*off + 8 > len)
        return -1;
    uint32_t w0, w1;
    memcpy(&w0, buf + *off, 4);
    memcpy(&w1, buf + *off + 4, 4);
    if (w0 >> 16) { /* small data element: 4 bytes of payload in the tag */
        *type = w0 & 0xffff;
        *nbytes = w0 >> 16;
        if (*nbytes > 4)
            return -1;
        *data = buf + *off + 4;
        *off += 8;
        return 0;
    }
    *type = w0;
    *nbytes = w1;
    if (*off + 8 + (size_t)w1 > len)
        return -1;
    *data = buf + *off + 8;
    *off += 8 + (((size_t)w1 + 7) & ~(size_t)7);
    if (*off > len)
        *off = len;
    return 0;
}

static size_t el_size(uint32_t type)
{
    switch (type) {
    case miINT8: case miUINT8: return 1;
    case miINT16: case miUINT16: return 2;
    case miINT32: case miUINT32: case miSINGLE: return 4;
    case miDOUBLE: case miINT64: case miUINT64: return 8;
    default: return 0;
    }
}

static uint64_t el_get(const unsigned char *d, uint32_t type, size_t i)
{
    switch (type) {
    case miINT8: return (uint64_t)(int64_t)((const int8_t *)d)[i];
    case miUINT8: return d[i];
    case miINT16: { int16_t v; memcpy(&v, d + 2 * i, 2); return (uint64_t)(int64_t)v; }
    case miUINT16: { uint16_t v; memcpy(&v, d + 2 * i, 2); return v; }
    case miINT32: { int32_t v; memcpy(&v, d + 4 * i, 4); return (uint64_t)(int64_t)v; }
    case miUINT32: { uint32_t v; memcpy(&v, d + 4 * i, 4); return v; }
    case miINT64: { int64_t v; memcpy(&v, d + 8 * i, 8); return (uint64_t)v; }
    case miUINT64: { uint64_t v; memcpy(&v, d + 8 * i, 8); return v; }
    case miDOUBLE: { double v; memcpy(&v, d + 8 * i, 8); return (uint64_t)v; }
    case miSINGLE: { float v; memcpy(&v, d + 4 * i, 4); return (uint64_t)v; }
    default: return 0;
    }
}

static mat_uint32_t *to_u32(const unsigned char *d, uint32_t type, uint32_t nbytes, size_t *count)
{
    size_t es = el_size(type);
    if (!es)
        return NULL;
    size_t k = nbytes / es;
    mat_uint32_t *out = (mat_uint32_t *)malloc((k ? k : 1) * sizeof(mat_uint32_t));
    if (!out)
        return NULL;
    for (size_t i = 0; i < k; ++i)
        out[i] = (mat_uint32_t)el_get(d, type, i);
    *count = k;
    return out;
}

static matvar_t *parse_matrix(const unsigned char *buf, size_t len, const char *name_override);

static void free_var(matvar_t *v)
{
    if (!v)
        return;
    if (v->class_type == MAT_C_SPARSE && v->data) {
        mat_sparse_t *s = (mat_sparse_t *)v->data;
        sparse_own *own = (sparse_own *)v->internal;
        if (!own || own->owns_ir)
            free(s->ir);
        if (!own || own->owns_jc)
            free(s->jc);
        free(s);
    } else if (v->class_type == MAT_C_STRUCT && v->data) {
        struct_data *sd = (struct_data *)v->data;
        for (size_t i = 0; i < sd->nel * (size_t)sd->nfields; ++i)
            free_var(sd->fields[i]);
        free(sd->fields);
        free(sd);
    }
    free(v->internal);
    free(v->dims);
    free(v->name);
    free(v);
}

static matvar_t *parse_matrix(const unsigned char *buf, size_t len, const char *name_override)
{
    matvar_t *v = (matvar_t *)calloc(1, sizeof(matvar_t));
    if (!v)
        return NULL;
    v->nbytes = len;
    if (len == 0) { /* empty element */
        v->class_type = MAT_C_EMPTY;
        v->name = strdup(name_override ? name_override : "");
        return v;
    }
    size_t off = 0;
    uint32_t type, nb;
    const unsigned char *d;
    /* array flags */
    if (next_el(buf, len, &off, &type, &d, &nb) || type != miUINT32 || nb < 8)
        goto bad;
    uint32_t flags;
    memcpy(&flags, d, 4);
    v->class_type = (enum matio_classes)(flags & 0xff);
    v->isLogical = (flags & 0x200) != 0;
    v->isGlobal = (flags & 0x400) != 0;
    v->isComplex = (flags & 0x800) != 0;
    /* dimensions */
    if (next_el(buf, len, &off, &type, &d, &nb))
        goto bad;
    size_t es = el_size(type);
    if (!es)
        goto bad;
    v->rank = (int)(nb / es);
    v->dims = (size_t *)calloc((size_t)v->rank + 1, sizeof(size_t));
    if (!v->dims)
        goto bad;
    for (int i = 0; i < v->rank; ++i)
        v->dims[i] = (size_t)el_get(d, type, (size_t)i);
    /* name */
    if (next_el(buf, len, &off, &type, &d, &nb))
        goto bad;
    if (name_override) {
        v->name = strdup(name_override);
    } else {
        v->name = (char *)malloc((size_t)nb + 1);
        if (v->name) {
            memcpy(v->name, d, nb);
            v->name[nb] = 0;
        }
    }
    if (!v->name)
        goto bad;

    if (v->class_type == MAT_C_SPARSE) {
        mat_sparse_t *s = (mat_sparse_t *)calloc(1, sizeof(mat_sparse_t));
        if (!s)
            goto bad;
        v->data = s;
        v->data_type = MAT_T_DOUBLE;
        if (next_el(buf, len, &off, &type, &d, &nb) || !(s->ir = to_u32(d, type, nb, &s->nir)))
            goto bad;
        if (next_el(buf, len, &off, &type, &d, &nb) || !(s->jc = to_u32(d, type, nb, &s->njc)))
            goto bad;
        s->nzmax = s->nir;
        if (v->rank < 2 || s->njc != v->dims[1] + 1) {
            fprintf(stderr, "fakematio: sparse '%s' has %zu column starts for %zu columns\n",
                    v->name, s->njc, v->rank >= 2 ? v->dims[1] : 0);
            goto bad;
        }
        /* values (and the imaginary part) are not needed by the loader */
    } else if (v->class_type == MAT_C_STRUCT) {
        v->data_type = MAT_T_STRUCT;
        if (next_el(buf, len, &off, &type, &d, &nb) || nb < 4)
            goto bad;
        int32_t fnl;
        memcpy(&fnl, d, 4);
        if (fnl <= 0)
            goto bad;
        if (next_el(buf, len, &off, &type, &d, &nb))
            goto bad;
        int nfields = (int)(nb / (uint32_t)fnl);
        size_t nel = 1;
        for (int i = 0; i < v->rank; ++i)
            nel *= v->dims[i];
        struct_data *sd = (struct_data *)calloc(1, sizeof(struct_data));
        if (!sd)
            goto bad;
        v->data = sd;
        sd->nfields = nfields;
        sd->nel = nel;
        sd->fields = (matvar_t **)calloc(nel * (size_t)nfields + 1, sizeof(matvar_t *));
        if (!sd->fields)
            goto bad;
        char fname[256];
        for (size_t e = 0; e < nel; ++e) {
            for (int f = 0; f < nfields; ++f) {
                size_t k = (size_t)fnl < sizeof(fname) - 1 ? (size_t)fnl : sizeof(fname) - 1;
                memcpy(fname, d + (size_t)f * (size_t)fnl, k);
                fname[k] = 0;
                uint32_t t2, n2;
                const unsigned char *d2;
                if (next_el(buf, len, &off, &t2, &d2, &n2) || t2 != miMATRIX)
                    goto bad;
                sd->fields[e * (size_t)nfields + (size_t)f] = parse_matrix(d2, n2, fname);
                if (!sd->fields[e * (size_t)nfields + (size_t)f])
                    goto bad;
            }
        }
    } else {
        v->data_type = MAT_T_UNKNOWN; /* numeric, char, cell, ...: contents not needed */
    }
    return v;
bad:
    free_var(v);
    return NULL;
}

static matvar_t *serve_csrbin(mat_t *m)
{
    if (m->size < 24)
        return NULL;
    uint32_t ver, n;
    uint64_t nnz;
    memcpy(&ver, m->map + 4, 4);
    memcpy(&n, m->map + 8, 4);
    memcpy(&nnz, m->map + 16, 8);
    size_t need = 24 + 8 * ((size_t)n + 1) + 4 * (size_t)nnz;
    if (ver != 1 || m->size < need) {
        fprintf(stderr, "fakematio: truncated or unknown CSR binary file\n");
        return NULL;
    }
    if (nnz > 0xffffffffull) {
        fprintf(stderr, "fakematio: %llu entries exceed 32-bit column starts\n",
                (unsigned long long)nnz);
        return NULL;
    }
    const unsigned char *rp = m->map + 24;
    matvar_t *v = (matvar_t *)calloc(1, sizeof(matvar_t));
    mat_sparse_t *s = (mat_sparse_t *)calloc(1, sizeof(mat_sparse_t));
    sparse_own *own = (sparse_own *)calloc(1, sizeof(sparse_own));
    size_t *dims = (size_t *)calloc(2, sizeof(size_t));
    mat_uint32_t *jc = (mat_uint32_t *)malloc(((size_t)n + 1) * sizeof(mat_uint32_t));
    if (!v || !s || !own || !dims || !jc) {
        free(v); free(s); free(own); free(dims); free(jc);
        return NULL;
    }
    for (size_t i = 0; i <= n; ++i) {
        uint64_t x;
        memcpy(&x, rp + 8 * i, 8);
        jc[i] = (mat_uint32_t)x;
    }
    own->owns_jc = 1;
    own->owns_ir = 0; /* points into the mapping */
    s->ir = (mat_uint32_t *)(m->map + 24 + 8 * ((size_t)n + 1));
    s->nir = s->nzmax = (size_t)nnz;
    s->jc = jc;
    s->njc = (size_t)n + 1;
    dims[0] = dims[1] = n;
    v->rank = 2;
    v->dims = dims;
    v->name = strdup("A");
    v->class_type = MAT_C_SPARSE;
    v->data_type = MAT_T_DOUBLE;
    v->isLogical = 1;
    v->data = s;
    v->internal = own;
    return v;
}

matvar_t *Mat_VarReadNext(mat_t *mat)
{
    if (!mat)
        return NULL;
    if (mat->csrbin) {
        if (mat->served)
            return NULL;
        mat->served = 1;
        return serve_csrbin(mat);
    }
    while (mat->pos + 8 <= mat->size) {
        uint32_t type, nb;
        const unsigned char *d;
        size_t off = mat->pos;
        if (next_el(mat->map, mat->size, &off, &type, &d, &nb))
            return NULL;
        if (type == miCOMPRESSED) {
            /* compressed elements are not padded: the next one starts right after */
            mat->pos = (size_t)(d - mat->map) + nb;
            uLongf cap = (uLongf)nb * 4 + 1024;
            for (;;) {
                unsigned char *out = (unsigned char *)malloc(cap);
                if (!out)
                    return NULL;
                z_stream zs;
                memset(&zs, 0, sizeof(zs));
                zs.next_in = (Bytef *)d;
                zs.avail_in = nb;
                zs.next_out = out;
                zs.avail_out = (uInt)(cap > 0xffffffffu ? 0xffffffffu : cap);
                inflateInit(&zs);
                int zr = inflate(&zs, Z_FINISH);
                size_t got = zs.total_out;
                inflateEnd(&zs);
                if (zr == Z_STREAM_END) {
                    size_t o2 = 0;
                    uint32_t t2, n2;
                    const unsigned char *d2;
                    matvar_t *v = NULL;
                    if (!next_el(out, got, &o2, &t2, &d2, &n2) && t2 == miMATRIX)
                        v = parse_matrix(d2, n2, NULL);
                    free(out);
                    if (v)
                        return v;
                    break; /* not a matrix: skip it */
                }
                free(out);
                if (!(zr == Z_BUF_ERROR || zr == Z_OK) || got < cap)
                    return NULL; /* corrupt stream (not merely a short buffer) */
                cap *= 4;
            }
            continue;
        }
        mat->pos = off;
        if (type == miMATRIX)
            return parse_matrix(d, nb, NULL);
    }
    return NULL;
}

matvar_t *Mat_VarGetStructFieldByName(matvar_t *matvar, const char *field_name, size_t index)
{
    if (!matvar || matvar->class_type != MAT_C_STRUCT || !matvar->data)
        return NULL;
    struct_data *sd = (struct_data *)matvar->data;
    if (index >= sd->nel)
        return NULL;
    for (int f = 0; f < sd->nfields; ++f) {
        matvar_t *v = sd->fields[index * (size_t)sd->nfields + (size_t)f];
        if (v && v->name && strcmp(v->name, field_name) == 0)
            return v;
    }
    return NULL;
}

void Mat_VarFree(matvar_t *matvar)
{
    /* A field handed out by Mat_VarGetStructFieldByName is owned by its
     * struct; the reference frees the field it kept and drops the struct, so
     * a field is freed here on its own and the struct is left alone. */
    free_var(matvar);
}
