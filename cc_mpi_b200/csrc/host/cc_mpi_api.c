/*
 * Reference-facing partitioned calls (include/cc_mpi.h, include/graph_dist.h)
 * on top of the C ABI.
 *
 * A DistCSRGraph of this build describes the whole graph; its device copy is
 * kept in a registry keyed by the host row_ptr pointer, created when the
 * graph is loaded (as the reference's scatter happens at load time,
 * src/graph_dist.c:142-342) and released by free_dist_csr.
 */
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "cc_mpi.h"
#include "ccgpu.h"
#include "host_common.h"

/* ------------------------------------------------------------ registry */

typedef struct mirror {
    const uint64_t *host_row_ptr;
    ccgpu_graph *dev; /* its label array holds solves with host output */
    struct mirror *next;
} mirror;

static pthread_mutex_t g_reg_mu = PTHREAD_MUTEX_INITIALIZER;
static mirror *g_reg = NULL;

static mirror *reg_find(const uint64_t *row_ptr)
{
    for (mirror *m = g_reg; m; m = m->next)
        if (m->host_row_ptr == row_ptr)
            return m;
    return NULL;
}

static int reg_get(const DistCSRGraph *Gd, mirror **out)
{
    pthread_mutex_lock(&g_reg_mu);
    mirror *m = reg_find(Gd->row_ptr);
    if (!m) {
        m = (mirror *)calloc(1, sizeof(mirror));
        int rc = m ? ccgpu_graph_upload(Gd->row_ptr, Gd->col_idx, Gd->n_global, Gd->m_global,
                                        &m->dev)
                   : CCGPU_ERR_OOM;
        if (rc != CCGPU_OK) {
            free(m);
            pthread_mutex_unlock(&g_reg_mu);
            return rc;
        }
        m->host_row_ptr = Gd->row_ptr;
        m->next = g_reg;
        g_reg = m;
    }
    pthread_mutex_unlock(&g_reg_mu);
    *out = m;
    return CCGPU_OK;
}

static void reg_drop(const uint64_t *row_ptr)
{
    pthread_mutex_lock(&g_reg_mu);
    for (mirror **pp = &g_reg; *pp; pp = &(*pp)->next) {
        if ((*pp)->host_row_ptr == row_ptr) {
            mirror *m = *pp;
            *pp = m->next;
            ccgpu_graph_free(m->dev);
            free(m);
            break;
        }
    }
    pthread_mutex_unlock(&g_reg_mu);
}

/* ------------------------------------------------------------- threads */

static int g_cc_threads = 0;

void cc_mpi_set_num_threads(int nthreads)
{
    g_cc_threads = nthreads > 0 ? nthreads : 0; /* src/cc_mpi.c:32-35 */
}

int cc_mpi_get_num_threads(void)
{
    return g_cc_threads;
}

/* -------------------------------------------------------------- loading */

static int fill_dist(const CSRGraph *g, int use_edge, DistCSRGraph *out, cc_group *grp)
{
    const int parts = cc_group_size(grp);
    out->n_global = g->n;
    out->m_global = g->m;
    out->n_local = g->n;
    out->m_local = g->m;
    out->v_start = 0;
    out->v_end = g->n;
    out->row_ptr = g->row_ptr;
    out->col_idx = g->col_idx;
    out->part_bounds = NULL;
    out->part_size = 0;
    out->part_kind = 0;
    if (g->n == 0)
        return 0;
    mirror *m = NULL;
    if (reg_get(out, &m) != CCGPU_OK) {
        fprintf(stderr, "load_dist_csr: %s\n", ccgpu_last_error());
        return 100;
    }
    if (use_edge && parts > 1) { /* src/graph_dist.c:183-206 */
        if ((uint32_t)parts > g->n) {
            fprintf(stderr, "load_dist_csr: %d partitions for %u vertices\n", parts, g->n);
            reg_drop(out->row_ptr);
            return 100;
        }
        uint32_t *b = (uint32_t *)malloc(((size_t)parts + 1) * sizeof(uint32_t));
        if (!b || ccgpu_partition_bounds(ccgpu_graph_row_ptr(m->dev), g->n, parts, 1, b,
                                         NULL) != CCGPU_OK) {
            fprintf(stderr, "load_dist_csr: %s\n", b ? ccgpu_last_error() : "host OOM");
            free(b);
            reg_drop(out->row_ptr);
            return 100;
        }
        out->part_bounds = b;
        out->part_size = parts;
        out->part_kind = 1;
    }
    return 0;
}

/* A .mat graph for the partitioned path: the CSC arrays go to the device and
 * are transposed there (ccgpu_graph_from_csc), the device CSR becomes the
 * graph's mirror, and the host CSR the DistCSRGraph exposes is copied back
 * from it.  Returns the loader's codes (src/graph.c:46,69,88), 100 on a
 * device failure. */
static int load_mat_on_device(const char *path, CSRGraph *full)
{
    mat_csc c;
    int rc = load_csc_from_mat(path, &c);
    if (rc != 0)
        return rc;
    ccgpu_graph *dev = NULL;
    rc = ccgpu_graph_from_csc(c.jc, c.ir, c.nrows, c.ncols, c.nnz, &dev);
    free_mat_csc(&c);
    if (rc != CCGPU_OK) {
        fprintf(stderr, "load_dist_csr: %s\n", ccgpu_last_error());
        return 100;
    }
    const uint32_t n = ccgpu_graph_n(dev);
    const uint64_t m = ccgpu_graph_m(dev);
    full->n = n;
    full->m = m;
    full->row_ptr = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    full->col_idx = (uint32_t *)malloc((size_t)(m ? m : 1) * sizeof(uint32_t));
    if (!full->row_ptr || !full->col_idx) {
        ccgpu_graph_free(dev);
        return 3;
    }
    if (ccgpu_memcpy_d2h(full->row_ptr, ccgpu_graph_row_ptr(dev),
                         ((size_t)n + 1) * sizeof(uint64_t)) != CCGPU_OK ||
        ccgpu_memcpy_d2h(full->col_idx, ccgpu_graph_col_idx(dev),
                         (size_t)m * sizeof(uint32_t)) != CCGPU_OK) {
        fprintf(stderr, "load_dist_csr: %s\n", ccgpu_last_error());
        ccgpu_graph_free(dev);
        return 100;
    }
    mirror *mr = (mirror *)calloc(1, sizeof(mirror));
    if (!mr) {
        ccgpu_graph_free(dev);
        return 3;
    }
    mr->host_row_ptr = full->row_ptr;
    mr->dev = dev;
    pthread_mutex_lock(&g_reg_mu);
    mr->next = g_reg;
    g_reg = mr;
    pthread_mutex_unlock(&g_reg_mu);
    return 0;
}

int load_dist_csr_from_file(const char *path, int symmetrize, int drop_self_loops, int use_edge,
                            DistCSRGraph *out, MPI_Comm comm)
{
    if (!out)
        return 99;
    memset(out, 0, sizeof(*out));
    CSRGraph full;
    memset(&full, 0, sizeof(full));
    const char *ext = strrchr(path ? path : "", '.');
    int rc;
    if (ext && strcasecmp(ext, ".mat") == 0)
        rc = load_mat_on_device(path, &full);
    else
        rc = load_csr_from_file(path, symmetrize, drop_self_loops, &full);
    if (rc != 0) {
        if (full.row_ptr)
            reg_drop(full.row_ptr);
        free_csr(&full);
        return rc;
    }
    rc = fill_dist(&full, use_edge, out, comm ? comm : cc_group_world());
    if (rc != 0) {
        free_csr(&full);
        memset(out, 0, sizeof(*out));
    }
    return rc;
}

int dist_csr_from_csr(const CSRGraph *g, int use_edge, DistCSRGraph *out, MPI_Comm comm)
{
    if (!g || !out)
        return 99;
    memset(out, 0, sizeof(*out));
    int rc = fill_dist(g, use_edge, out, comm ? comm : cc_group_world());
    if (rc != 0)
        memset(out, 0, sizeof(*out));
    return rc;
}

void free_dist_csr_view(DistCSRGraph *g)
{
    if (!g)
        return;
    if (g->row_ptr)
        reg_drop(g->row_ptr);
    free(g->part_bounds);
    memset(g, 0, sizeof(*g));
}

void free_dist_csr(DistCSRGraph *g)
{
    if (!g)
        return;
    if (g->row_ptr)
        reg_drop(g->row_ptr);
    free(g->row_ptr);
    free(g->col_idx);
    free(g->part_bounds);
    memset(g, 0, sizeof(*g)); /* src/graph_dist.c:360-378 */
}

/* --------------------------------------------------------------- solve */

int cc_mpi_solve(const DistCSRGraph *Gd, uint32_t *labels_global, int chunk_size,
                 int exchange_interval, MPI_Comm comm, ccgpu_dist_stats *stats)
{
    if (!Gd)
        return ccb200_set_error(CCGPU_ERR_INVALID, "NULL DistCSRGraph");
    if (Gd->n_global == 0 || Gd->n_local == 0)
        return CCGPU_OK; /* src/cc_mpi.c:247-248 */
    if (Gd->n_local != Gd->n_global || Gd->v_start != 0)
        return ccb200_set_error(CCGPU_ERR_LIMIT,
                                      "DistCSRGraph holds vertices [%u, %u) of %u: this build "
                                      "keeps every partition in one process and needs the whole "
                                      "graph",
                                      Gd->v_start, Gd->v_end, Gd->n_global);
    cc_group *grp = comm ? comm : cc_group_world();
    const int parts = cc_group_size(grp);
    if (Gd->part_kind != 0 && Gd->part_size != parts)
        return ccb200_set_error(CCGPU_ERR_INVALID,
                                      "graph was partitioned for %d parts, group has %d",
                                      Gd->part_size, parts);
    mirror *m = NULL;
    int rc = reg_get(Gd, &m);
    if (rc != CCGPU_OK)
        return rc;
    uint32_t *d_labels = NULL;
    if (labels_global) {
        rc = ccgpu_graph_label_array(m->dev, &d_labels);
        if (rc != CCGPU_OK)
            return rc;
    }
    ccgpu_dist_opts o;
    ccgpu_dist_opts_default(&o);
    o.parts = parts;
    o.use_edge = (Gd->part_kind != 0) ? 1 : 0;
    o.chunk_size = chunk_size;
    o.exchange_interval = exchange_interval < 1 ? 1 : exchange_interval;
    o.verbose = cc_group_verbose(grp);
    ccgpu_dist_stats s;
    rc = ccgpu_dist_cc(NULL, ccgpu_graph_row_ptr(m->dev), ccgpu_graph_col_idx(m->dev),
                       Gd->n_global, Gd->m_global, &o, d_labels, NULL,
                       &s, NULL);
    if (rc != CCGPU_OK)
        return rc;
    if (labels_global) {
        rc = ccgpu_memcpy_d2h(labels_global, d_labels, (size_t)Gd->n_global * sizeof(uint32_t));
        if (rc != CCGPU_OK)
            return rc;
    }
    cc_group_store_stats(grp, &s);
    if (stats)
        *stats = s;
    return CCGPU_OK;
}

void compute_connected_components_mpi_advanced(const DistCSRGraph *restrict Gd,
                                               uint32_t *restrict labels_global, int chunk_size,
                                               int exchange_interval, MPI_Comm comm)
{
    int rc = cc_mpi_solve(Gd, labels_global, chunk_size, exchange_interval, comm, NULL);
    if (rc != CCGPU_OK)
        ccb200_fail("compute_connected_components_mpi_advanced", rc);
}

uint32_t count_connected_components(const uint32_t *restrict labels_global, uint32_t n_global)
{
    if (n_global == 0 || labels_global == NULL)
        return 0;
    unsigned char *seen = (unsigned char *)calloc(n_global, 1);
    if (!seen) {
        fprintf(stderr, "count_connected_components: Failed to allocate bitmap\n");
        return 0;
    }
    uint32_t c = 0;
    for (uint32_t v = 0; v < n_global; ++v) {
        uint32_t r = labels_global[v];
        if (r < n_global && !seen[r]) {
            seen[r] = 1;
            c++;
        }
    }
    free(seen);
    return c;
}
