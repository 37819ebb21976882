/*
 * Graph file I/O: MATLAB level-5 .mat (the reference's format, read there
 * through libmatio, src/graph.c:38-128), Matrix Market, and a raw binary
 * CSR (.csrbin) for graphs larger than a MAT v5 file can hold.
 *
 * The .mat reader follows the MAT-File Level 5 format as published by The
 * MathWorks: a 128-byte header, then tagged data elements, miCOMPRESSED
 * elements being zlib streams of one miMATRIX element.  Only what the
 * reference reads is handled: struct variables (to find Problem.A) and
 * sparse variables (their ir/jc arrays).
 */
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <zlib.h>

#include "graph.h"
#include "host_common.h"

enum {
    miINT8 = 1, miUINT8 = 2, miINT16 = 3, miUINT16 = 4, miINT32 = 5, miUINT32 = 6,
    miSINGLE = 7, miDOUBLE = 9, miINT64 = 12, miUINT64 = 13, miMATRIX = 14,
    miCOMPRESSED = 15
};
enum { mxSTRUCT_CLASS = 2, mxSPARSE_CLASS = 5 };

void free_csr(CSRGraph *g)
{
    if (!g)
        return;
    free(g->row_ptr);
    free(g->col_idx);
    g->row_ptr = NULL;
    g->col_idx = NULL;
    g->n = 0;
    g->m = 0;
}

/* ------------------------------------------------------------ buffers */

typedef struct {
    const unsigned char *p;
    size_t len;
} span;

static int read_file(const char *path, unsigned char **buf, size_t *len)
{
    FILE *f = fopen(path, "rb");
    if (!f)
        return 1;
    if (fseek(f, 0, SEEK_END) != 0) {
        fclose(f);
        return 1;
    }
    long sz = ftell(f);
    if (sz < 0) {
        fclose(f);
        return 1;
    }
    rewind(f);
    *buf = (unsigned char *)malloc(sz ? (size_t)sz : 1);
    if (!*buf) {
        fclose(f);
        return 3;
    }
    if (sz && fread(*buf, 1, (size_t)sz, f) != (size_t)sz) {
        free(*buf);
        fclose(f);
        return 1;
    }
    fclose(f);
    *len = (size_t)sz;
    return 0;
}

static uint32_t rd32(const unsigned char *p)
{
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
}

/* One data element: type, payload, and total bytes consumed (tag +
 * payload + padding to 8). */
typedef struct {
    uint32_t type;
    span data;
    size_t consumed;
} melem;

static int next_elem(span s, melem *e)
{
    if (s.len < 8)
        return -1;
    uint32_t t = rd32(s.p), nb = rd32(s.p + 4);
    if (t >> 16) { /* small data element: payload packed in the tag */
        e->type = t & 0xffff;
        e->data.p = s.p + 4;
        e->data.len = t >> 16;
        if (e->data.len > 4)
            return -1;
        e->consumed = 8;
        return 0;
    }
    e->type = t;
    if ((uint64_t)nb > s.len - 8)
        return -1;
    e->data.p = s.p + 8;
    e->data.len = nb;
    size_t pad = (t == miCOMPRESSED) ? 0 : ((8 - (nb & 7)) & 7);
    e->consumed = 8 + (size_t)nb + pad;
    if (e->consumed > s.len)
        e->consumed = s.len;
    return 0;
}

static int inflate_all(span in, unsigned char **out, size_t *out_len)
{
    z_stream z;
    memset(&z, 0, sizeof(z));
    if (inflateInit(&z) != Z_OK)
        return 3;
    size_t cap = in.len * 4 + 1024, len = 0;
    unsigned char *buf = (unsigned char *)malloc(cap);
    if (!buf) {
        inflateEnd(&z);
        return 3;
    }
    z.next_in = (unsigned char *)in.p;
    z.avail_in = 0;
    size_t fed = 0;
    int rc = Z_OK;
    while (rc != Z_STREAM_END) {
        if (z.avail_in == 0 && fed < in.len) {
            size_t chunk = in.len - fed > (1u << 30) ? (1u << 30) : in.len - fed;
            z.next_in = (unsigned char *)in.p + fed;
            z.avail_in = (uInt)chunk;
            fed += chunk;
        }
        if (len == cap) {
            size_t ncap = cap * 2;
            unsigned char *nb = (unsigned char *)realloc(buf, ncap);
            if (!nb) {
                free(buf);
                inflateEnd(&z);
                return 3;
            }
            buf = nb;
            cap = ncap;
        }
        size_t room = cap - len > (1u << 30) ? (1u << 30) : cap - len;
        z.next_out = buf + len;
        z.avail_out = (uInt)room;
        rc = inflate(&z, Z_NO_FLUSH);
        len += room - z.avail_out;
        if (rc == Z_BUF_ERROR && z.avail_in == 0 && fed >= in.len)
            break; /* truncated stream: keep what inflated */
        if (rc != Z_OK && rc != Z_STREAM_END && rc != Z_BUF_ERROR) {
            free(buf);
            inflateEnd(&z);
            return 4;
        }
    }
    inflateEnd(&z);
    *out = buf;
    *out_len = len;
    return 0;
}

/* Integer array element -> uint64 values (ir/jc may be any integer type). */
static int int_array(const melem *e, uint64_t **out, uint64_t *count)
{
    size_t w;
    switch (e->type) {
    case miINT8: case miUINT8: w = 1; break;
    case miINT16: case miUINT16: w = 2; break;
    case miINT32: case miUINT32: w = 4; break;
    case miINT64: case miUINT64: w = 8; break;
    case miDOUBLE: w = 8; break;
    default: return 4;
    }
    uint64_t n = e->data.len / w;
    uint64_t *v = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
    if (!v)
        return 3;
    const unsigned char *p = e->data.p;
    for (uint64_t i = 0; i < n; ++i) {
        switch (e->type) {
        case miINT8: v[i] = (uint64_t)(int64_t)((const int8_t *)p)[i]; break;
        case miUINT8: v[i] = p[i]; break;
        case miINT16: { int16_t x; memcpy(&x, p + 2 * i, 2); v[i] = (uint64_t)(int64_t)x; } break;
        case miUINT16: { uint16_t x; memcpy(&x, p + 2 * i, 2); v[i] = x; } break;
        case miINT32: { int32_t x; memcpy(&x, p + 4 * i, 4); v[i] = (uint64_t)(int64_t)x; } break;
        case miUINT32: { uint32_t x; memcpy(&x, p + 4 * i, 4); v[i] = x; } break;
        case miDOUBLE: { double x; memcpy(&x, p + 8 * i, 8); v[i] = (uint64_t)(int64_t)x; } break;
        default: memcpy(&v[i], p + 8 * i, 8); break;
        }
    }
    *out = v;
    *count = n;
    return 0;
}

/* CSC (ir, jc) of an nrows x ncols sparse matrix -> CSR with the column
 * index as the neighbour, rows counted/scanned/scattered as in the
 * reference (src/graph.c:56-117).  Row ids outside [0,nrows) are skipped. */
static int csc_to_csr(uint64_t nrows, uint64_t ncols, const uint64_t *ir, uint64_t nir,
                      const uint64_t *jc, uint64_t njc, CSRGraph *out)
{
    if (nrows > 0xfffffffeull || njc < ncols + 1)
        return 4;
    uint64_t nz = jc[ncols];
    if (nz > nir)
        nz = nir;
    uint32_t n = (uint32_t)nrows;
    uint64_t *row_ptr = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t *col = (uint32_t *)malloc((nz ? nz : 1) * sizeof(uint32_t));
    uint64_t *head = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    if (!row_ptr || !col || !head) {
        free(row_ptr);
        free(col);
        free(head);
        return 3;
    }
    for (uint64_t c = 0; c < ncols; ++c)
        for (uint64_t j = jc[c]; j < jc[c + 1] && j < nz; ++j)
            if ((int64_t)ir[j] >= 0 && ir[j] < n)
                row_ptr[ir[j] + 1]++;
    for (uint32_t i = 0; i < n; ++i)
        row_ptr[i + 1] += row_ptr[i];
    memcpy(head, row_ptr, (size_t)n * sizeof(uint64_t));
    for (uint64_t c = 0; c < ncols; ++c)
        for (uint64_t j = jc[c]; j < jc[c + 1] && j < nz; ++j)
            if ((int64_t)ir[j] >= 0 && ir[j] < n)
                col[head[ir[j]]++] = (uint32_t)c;
    free(head);
    out->n = n;
    out->m = row_ptr[n];
    out->row_ptr = row_ptr;
    out->col_idx = col;
    return 0;
}

typedef struct {
    uint32_t cls;
    uint64_t dims[2];
    char name[64];
    span body; /* the elements after the name */
} mmatrix;

static int parse_matrix_header(span s, mmatrix *M)
{
    melem e;
    memset(M, 0, sizeof(*M));
    if (next_elem(s, &e) || e.type != miUINT32 || e.data.len < 8)
        return 4;
    M->cls = rd32(e.data.p) & 0xff;
    s.p += e.consumed;
    s.len -= e.consumed;
    if (next_elem(s, &e) || (e.type != miINT32 && e.type != miUINT32))
        return 4;
    uint32_t nd = (uint32_t)(e.data.len / 4);
    M->dims[0] = nd > 0 ? rd32(e.data.p) : 0;
    M->dims[1] = nd > 1 ? rd32(e.data.p + 4) : 1;
    s.p += e.consumed;
    s.len -= e.consumed;
    if (next_elem(s, &e))
        return 4;
    size_t nl = e.data.len < sizeof(M->name) - 1 ? e.data.len : sizeof(M->name) - 1;
    memcpy(M->name, e.data.p, nl);
    M->name[nl] = 0;
    s.p += e.consumed;
    s.len -= e.consumed;
    M->body = s;
    return 0;
}

/* The CSC arrays of a sparse matrix element. */
static int sparse_arrays(const mmatrix *M, uint64_t **ir, uint64_t *nir, uint64_t **jc,
                         uint64_t *njc)
{
    span s = M->body;
    melem eir, ejc;
    if (next_elem(s, &eir))
        return 4;
    s.p += eir.consumed;
    s.len -= eir.consumed;
    if (next_elem(s, &ejc))
        return 4;
    *ir = *jc = NULL;
    int rc = int_array(&eir, ir, nir);
    if (rc == 0)
        rc = int_array(&ejc, jc, njc);
    if (rc != 0) {
        free(*ir);
        free(*jc);
        *ir = *jc = NULL;
    }
    return rc;
}

static int sparse_to_csr(const mmatrix *M, void *arg)
{
    uint64_t *ir = NULL, *jc = NULL, nir = 0, njc = 0;
    int rc = sparse_arrays(M, &ir, &nir, &jc, &njc);
    if (rc == 0)
        rc = csc_to_csr(M->dims[0], M->dims[1], ir, nir, jc, njc, (CSRGraph *)arg);
    free(ir);
    free(jc);
    return rc;
}

/* The CSC arrays as they are (row indices that are negative or do not fit
 * 32 bits become UINT32_MAX, which every reader drops as out of range). */
static int sparse_to_csc(const mmatrix *M, void *arg)
{
    mat_csc *out = (mat_csc *)arg;
    uint64_t *ir = NULL, *jc = NULL, nir = 0, njc = 0;
    int rc = sparse_arrays(M, &ir, &nir, &jc, &njc);
    if (rc != 0)
        return rc;
    if (M->dims[0] > 0xfffffffeull || M->dims[1] > 0xfffffffeull || njc < M->dims[1] + 1) {
        free(ir);
        free(jc);
        return 4;
    }
    uint64_t nz = jc[M->dims[1]];
    if (nz > nir)
        nz = nir;
    uint32_t *ir32 = (uint32_t *)malloc((nz ? nz : 1) * sizeof(uint32_t));
    if (!ir32) {
        free(ir);
        free(jc);
        return 3;
    }
    for (uint64_t j = 0; j < nz; ++j)
        ir32[j] = ir[j] > 0xffffffffull ? 0xffffffffu : (uint32_t)ir[j];
    free(ir);
    out->nrows = (uint32_t)M->dims[0];
    out->ncols = (uint32_t)M->dims[1];
    out->nnz = nz;
    out->jc = jc;
    out->ir = ir32;
    return 0;
}

/* Finds field `want` of a 1x1 struct; returns its miMATRIX payload. */
static int struct_field(const mmatrix *M, const char *want, span *field)
{
    span s = M->body;
    melem e;
    if (next_elem(s, &e) || e.data.len < 4)
        return 2;
    uint32_t flen = rd32(e.data.p);
    s.p += e.consumed;
    s.len -= e.consumed;
    if (next_elem(s, &e) || flen == 0)
        return 2;
    uint32_t nf = (uint32_t)(e.data.len / flen);
    const unsigned char *names = e.data.p;
    s.p += e.consumed;
    s.len -= e.consumed;
    for (uint32_t f = 0; f < nf; ++f) {
        melem fe;
        if (next_elem(s, &fe) || fe.type != miMATRIX)
            return 2;
        if (strncmp((const char *)names + (size_t)f * flen, want, flen) == 0) {
            *field = fe.data;
            return 0;
        }
        s.p += fe.consumed;
        s.len -= fe.consumed;
    }
    return 2;
}

/* Walks the MAT file for struct Problem's field A, or else the first
 * sparse variable (src/graph.c:49-63), and hands it to fn. */
static int mat_find_sparse(const char *path, int (*fn)(const mmatrix *, void *), void *arg)
{
    unsigned char *buf = NULL;
    size_t len = 0;
    int rc = read_file(path, &buf, &len);
    if (rc) {
        fprintf(stderr, "Error opening .mat file: %s\n", path);
        return rc == 3 ? 3 : 1;
    }
    if (len < 128 || buf[126] != 'I' || buf[127] != 'M') {
        free(buf);
        fprintf(stderr, "Not a little-endian MAT level-5 file: %s\n", path);
        return 1;
    }
    span s = {buf + 128, len - 128};
    rc = 2;
    while (s.len >= 8) {
        melem e;
        if (next_elem(s, &e)) {
            rc = 4;
            break;
        }
        unsigned char *inflated = NULL;
        size_t ilen = 0;
        span mat = {NULL, 0};
        if (e.type == miCOMPRESSED) {
            int zr = inflate_all(e.data, &inflated, &ilen);
            if (zr) {
                rc = zr;
                break;
            }
            melem inner;
            if (next_elem((span){inflated, ilen}, &inner) == 0 && inner.type == miMATRIX)
                mat = inner.data;
        } else if (e.type == miMATRIX) {
            mat = e.data;
        }
        int done = 0;
        if (mat.p && mat.len) {
            mmatrix M;
            if (parse_matrix_header(mat, &M) == 0) {
                if (strcmp(M.name, "Problem") == 0 && M.cls == mxSTRUCT_CLASS) {
                    span field;
                    rc = 2;
                    if (struct_field(&M, "A", &field) == 0) {
                        mmatrix A;
                        if (parse_matrix_header(field, &A) == 0 && A.cls == mxSPARSE_CLASS)
                            rc = fn(&A, arg);
                    }
                    done = 1;
                } else if (M.cls == mxSPARSE_CLASS) {
                    rc = fn(&M, arg);
                    done = 1;
                }
            }
        }
        free(inflated);
        if (done)
            break;
        s.p += e.consumed;
        s.len -= e.consumed;
    }
    free(buf);
    if (rc == 2)
        fprintf(stderr, "No sparse matrix found in .mat file %s\n", path);
    return rc;
}

int load_csr_from_mat(const char *path, CSRGraph *out)
{
    memset(out, 0, sizeof(*out));
    return mat_find_sparse(path, sparse_to_csr, out);
}

int load_csc_from_mat(const char *path, mat_csc *out)
{
    memset(out, 0, sizeof(*out));
    return mat_find_sparse(path, sparse_to_csc, out);
}

void free_mat_csc(mat_csc *c)
{
    if (!c)
        return;
    free(c->jc);
    free(c->ir);
    memset(c, 0, sizeof(*c));
}

/* ----------------------------------------------------------- MAT writer */

static int put_tag(FILE *f, uint32_t type, uint32_t nbytes)
{
    uint32_t t[2] = {type, nbytes};
    return fwrite(t, 4, 2, f) == 2 ? 0 : 1;
}

static int put_pad(FILE *f, uint64_t nbytes)
{
    static const unsigned char z[8] = {0};
    size_t pad = (8 - (nbytes & 7)) & 7;
    return (pad && fwrite(z, 1, pad, f) != pad) ? 1 : 0;
}

int save_csr_to_mat(const char *path, const CSRGraph *g)
{
    uint64_t nnz = g->m, n = g->n;
    /* ir is int32 and element sizes are uint32 in MAT v5 */
    if (nnz * 4 + 64 > 0xffffffffull || nnz > 0x7fffffffull || (n + 1) * 4 > 0xffffffffull)
        return 4;
    FILE *f = fopen(path, "wb");
    if (!f)
        return 1;
    char hdr[128];
    memset(hdr, ' ', sizeof(hdr));
    const char *txt = "MATLAB 5.0 MAT-file, written by libccb200 save_csr_to_mat";
    memcpy(hdr, txt, strlen(txt));
    memset(hdr + 116, 0, 8);
    hdr[124] = 0x00;
    hdr[125] = 0x01;
    hdr[126] = 'I';
    hdr[127] = 'M';
    int bad = fwrite(hdr, 1, 128, f) != 128;
    uint64_t a_ir = nnz * 4, a_jc = (n + 1) * 4, a_pr = nnz;
    uint64_t a_body = 16 + 16 + 8 + (8 + a_ir + ((8 - (a_ir & 7)) & 7)) +
                      (8 + a_jc + ((8 - (a_jc & 7)) & 7)) + (8 + a_pr + ((8 - (a_pr & 7)) & 7));
    uint64_t s_body = 16 + 16 + 16 + 8 + (8 + 32) + (8 + a_body);
    if (8 + s_body > 0xffffffffull) {
        fclose(f);
        return 4;
    }
    uint32_t u[2];
    int32_t d[2];
    bad |= put_tag(f, miMATRIX, (uint32_t)s_body);
    u[0] = mxSTRUCT_CLASS;
    u[1] = 0;
    bad |= put_tag(f, miUINT32, 8) || fwrite(u, 4, 2, f) != 2;
    d[0] = 1;
    d[1] = 1;
    bad |= put_tag(f, miINT32, 8) || fwrite(d, 4, 2, f) != 2;
    bad |= put_tag(f, miINT8, 7) || fwrite("Problem\0", 1, 8, f) != 8;
    uint32_t small[2] = {(4u << 16) | miINT32, 32};
    bad |= fwrite(small, 4, 2, f) != 2;
    char fname[32] = {'A'};
    bad |= put_tag(f, miINT8, 32) || fwrite(fname, 1, 32, f) != 32;
    bad |= put_tag(f, miMATRIX, (uint32_t)a_body);
    u[0] = mxSPARSE_CLASS | 0x200; /* logical */
    u[1] = (uint32_t)(nnz ? nnz : 1);
    bad |= put_tag(f, miUINT32, 8) || fwrite(u, 4, 2, f) != 2;
    d[0] = (int32_t)n;
    d[1] = (int32_t)n;
    bad |= put_tag(f, miINT32, 8) || fwrite(d, 4, 2, f) != 2;
    bad |= put_tag(f, miINT8, 0);
    /* CSC of the transpose == CSR of g; equal to g's CSC for symmetric g */
    bad |= put_tag(f, miINT32, (uint32_t)a_ir);
    for (uint64_t i = 0; i < nnz && !bad; ++i) {
        int32_t x = (int32_t)g->col_idx[i];
        bad |= fwrite(&x, 4, 1, f) != 1;
    }
    bad |= put_pad(f, a_ir);
    bad |= put_tag(f, miINT32, (uint32_t)a_jc);
    for (uint64_t i = 0; i <= n && !bad; ++i) {
        int32_t x = (int32_t)g->row_ptr[i];
        bad |= fwrite(&x, 4, 1, f) != 1;
    }
    bad |= put_pad(f, a_jc);
    bad |= put_tag(f, miUINT8, (uint32_t)a_pr);
    for (uint64_t i = 0; i < nnz && !bad; ++i)
        bad |= fputc(1, f) == EOF;
    bad |= put_pad(f, a_pr);
    bad |= fclose(f) != 0;
    return bad ? 1 : 0;
}

/* -------------------------------------------------------------- csrbin */

static const char kMagic[4] = {'C', 'S', 'R', 'B'};

int save_csr_to_csrbin(const char *path, const CSRGraph *g)
{
    FILE *f = fopen(path, "wb");
    if (!f)
        return 1;
    uint32_t ver = 1, n = g->n;
    uint64_t m = g->m;
    int bad = fwrite(kMagic, 1, 4, f) != 4 || fwrite(&ver, 4, 1, f) != 1 ||
              fwrite(&n, 4, 1, f) != 1 || fwrite(&ver, 4, 1, f) != 1 || fwrite(&m, 8, 1, f) != 1;
    bad |= fwrite(g->row_ptr, 8, (size_t)n + 1, f) != (size_t)n + 1;
    if (m)
        bad |= fwrite(g->col_idx, 4, (size_t)m, f) != (size_t)m;
    bad |= fclose(f) != 0;
    return bad ? 1 : 0;
}

int load_csr_from_csrbin(const char *path, CSRGraph *out)
{
    memset(out, 0, sizeof(*out));
    FILE *f = fopen(path, "rb");
    if (!f)
        return 1;
    char mg[4];
    uint32_t ver = 0, n = 0, pad = 0;
    uint64_t m = 0;
    if (fread(mg, 1, 4, f) != 4 || memcmp(mg, kMagic, 4) != 0 || fread(&ver, 4, 1, f) != 1 ||
        ver != 1 || fread(&n, 4, 1, f) != 1 || fread(&pad, 4, 1, f) != 1 ||
        fread(&m, 8, 1, f) != 1) {
        fclose(f);
        return 5;
    }
    uint64_t *row = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    uint32_t *col = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    if (!row || !col) {
        free(row);
        free(col);
        fclose(f);
        return 3;
    }
    int bad = fread(row, 8, (size_t)n + 1, f) != (size_t)n + 1;
    if (m)
        bad |= fread(col, 4, (size_t)m, f) != (size_t)m;
    fclose(f);
    if (bad || row[n] != m || row[0] != 0) {
        free(row);
        free(col);
        return 5;
    }
    out->n = n;
    out->m = m;
    out->row_ptr = row;
    out->col_idx = col;
    return 0;
}

/* ------------------------------------------------------- Matrix Market */

static int cmp_u64(const void *a, const void *b)
{
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

int load_csr_from_mtx(const char *path, int symmetrize, int drop_self_loops, CSRGraph *out)
{
    memset(out, 0, sizeof(*out));
    FILE *f = fopen(path, "r");
    if (!f)
        return 1;
    char line[1024];
    int symmetric_file = 0, header = 0;
    uint64_t rows = 0, cols = 0, nnz = 0;
    while (fgets(line, sizeof(line), f)) {
        if (line[0] == '%') {
            if (!header && strncmp(line, "%%MatrixMarket", 14) == 0) {
                for (char *p = line; *p; ++p)
                    *p = (char)tolower((unsigned char)*p);
                if (!strstr(line, "coordinate")) {
                    fclose(f);
                    return 4;
                }
                symmetric_file = strstr(line, "symmetric") != NULL;
                header = 1;
            }
            continue;
        }
        if (sscanf(line, "%lu %lu %lu", &rows, &cols, &nnz) == 3)
            break;
    }
    if (rows == 0 || rows > 0xfffffffeull || cols > 0xfffffffeull) {
        fclose(f);
        return 2;
    }
    int twice = symmetrize || symmetric_file;
    uint64_t *keys = (uint64_t *)malloc((nnz * (twice ? 2 : 1) + 1) * sizeof(uint64_t));
    if (!keys) {
        fclose(f);
        return 3;
    }
    uint64_t k = 0;
    uint32_t n = (uint32_t)(rows > cols ? rows : cols);
    for (uint64_t i = 0; i < nnz && fgets(line, sizeof(line), f);) {
        unsigned long r, c;
        if (line[0] == '%' || sscanf(line, "%lu %lu", &r, &c) != 2)
            continue;
        ++i;
        if (r < 1 || c < 1 || r > n || c > n)
            continue;
        r--;
        c--;
        if (drop_self_loops && r == c)
            continue;
        keys[k++] = ((uint64_t)r << 32) | c;
        if (twice && r != c)
            keys[k++] = ((uint64_t)c << 32) | r;
    }
    fclose(f);
    qsort(keys, k, sizeof(uint64_t), cmp_u64);
    uint64_t u = 0;
    for (uint64_t i = 0; i < k; ++i)
        if (u == 0 || keys[i] != keys[u - 1])
            keys[u++] = keys[i];
    uint64_t *row = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t *col = (uint32_t *)malloc((u ? u : 1) * sizeof(uint32_t));
    if (!row || !col) {
        free(keys);
        free(row);
        free(col);
        return 3;
    }
    for (uint64_t i = 0; i < u; ++i) {
        row[(keys[i] >> 32) + 1]++;
        col[i] = (uint32_t)keys[i];
    }
    for (uint32_t v = 0; v < n; ++v)
        row[v + 1] += row[v];
    free(keys);
    out->n = n;
    out->m = u;
    out->row_ptr = row;
    out->col_idx = col;
    return 0;
}

int load_csr_from_file(const char *path, int symmetrize, int drop_self_loops, CSRGraph *out)
{
    (void)symmetrize;
    (void)drop_self_loops;
    const char *ext = path ? strrchr(path, '.') : NULL;
    if (!ext)
        ext = "";
    if (strcasecmp(ext, ".mtx") == 0 || strcasecmp(ext, ".txt") == 0)
        return -1; /* as the reference, src/graph.c:22-25 */
    if (strcasecmp(ext, ".mat") == 0)
        return load_csr_from_mat(path, out);
    if (strcasecmp(ext, ".csrbin") == 0)
        return load_csr_from_csrbin(path, out);
    fprintf(stderr, "Unsupported file extension: %s\n", ext);
    return 99;
}
