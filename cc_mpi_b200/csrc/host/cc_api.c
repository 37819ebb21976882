/*
 * Reference-facing local CC calls (include/cc.h) on top of the C ABI.
 *
 * compute_connected_components_pthreads keeps the reference's signature and
 * chunk semantics (include/cc.h:27-28, src/cc_pthreads.c:152-229); the work
 * runs on the current CUDA device.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cc.h"
#include "ccgpu.h"
#include "host_common.h"

static int g_exit_on_error = 1;

int ccb200_set_exit_on_error(int on)
{
    int prev = g_exit_on_error;
    g_exit_on_error = on ? 1 : 0;
    return prev;
}

int ccb200_exit_on_error(void)
{
    return g_exit_on_error;
}

void ccb200_fail(const char *where, int status)
{
    fprintf(stderr, "%s: %s (status %d)\n", where, ccgpu_last_error(), status);
    fflush(stderr);
    if (g_exit_on_error)
        exit(EXIT_FAILURE);
}

static void solve_host(const CSRGraph *G, uint32_t *labels, int chunk_size, const char *who)
{
    if (!G || !labels) {
        fprintf(stderr, "%s: NULL graph or labels\n", who);
        if (g_exit_on_error)
            exit(EXIT_FAILURE);
        return;
    }
    if (G->n == 0)
        return;
    ccgpu_cc_opts o;
    ccgpu_cc_opts_default(&o);
    o.chunk_size = chunk_size > 0 ? chunk_size : DEFAULT_CHUNK_SIZE;
    int rc = ccgpu_local_cc_host(NULL, G->row_ptr, G->col_idx, G->n, G->m, labels, &o, NULL);
    if (rc != CCGPU_OK)
        ccb200_fail(who, rc);
}

void compute_connected_components_pthreads(const CSRGraph *restrict G, uint32_t *restrict labels,
                                           int num_threads, int chunk_size)
{
    (void)num_threads; /* a host-thread count; the GPU schedule ignores it */
    solve_host(G, labels, chunk_size, "compute_connected_components_pthreads");
}

void compute_connected_components(const CSRGraph *restrict G, uint32_t *restrict labels)
{
    solve_host(G, labels, DEFAULT_CHUNK_SIZE, "compute_connected_components");
}

void compute_connected_components_bfs(const CSRGraph *restrict G, uint32_t *restrict labels)
{
    solve_host(G, labels, DEFAULT_CHUNK_SIZE, "compute_connected_components_bfs");
}

void compute_connected_components_omp(const CSRGraph *restrict G, uint32_t *restrict labels,
                                      int chunk_size)
{
    solve_host(G, labels, chunk_size, "compute_connected_components_omp");
}

void compute_connected_components_cilk(const CSRGraph *restrict G, uint32_t *restrict labels,
                                       int chunk_size)
{
    solve_host(G, labels, chunk_size, "compute_connected_components_cilk");
}

uint32_t count_unique_labels(const uint32_t *restrict labels, uint32_t n)
{
    if (!labels || n == 0)
        return 0;
    unsigned char *seen = (unsigned char *)calloc(n, 1);
    if (!seen) {
        fprintf(stderr, "count_unique_labels: out of host memory\n");
        return 0;
    }
    uint32_t c = 0;
    for (uint32_t v = 0; v < n; ++v) {
        uint32_t r = labels[v];
        if (r < n && !seen[r]) {
            seen[r] = 1;
            c++;
        }
    }
    free(seen);
    return c;
}
