/*
 * Reference-facing boundary edge calls (include/boundary_sort.h) and the
 * host vector helpers (include/vec_helpers.h), plus runtime_utils.h.
 *
 * boundary_edges_sort / boundary_edges_dedup keep the reference's
 * in-place, host-array contract (src/boundary_sort.c:93-119); the arrays
 * travel to HBM and are sorted there by the LSD radix sort.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "boundary_sort.h"
#include "ccgpu.h"
#include "host_common.h"
#include "runtime_utils.h"

static int pairs_to_device(const BoundaryEdge *edges, uint64_t count, void **d)
{
    int rc = ccgpu_alloc(d, (size_t)count * sizeof(BoundaryEdge));
    if (rc == CCGPU_OK)
        rc = ccgpu_memcpy_h2d(*d, edges, (size_t)count * sizeof(BoundaryEdge));
    return rc;
}

void boundary_edges_sort(BoundaryEdge *edges, uint64_t count)
{
    if (!edges || count <= 1)
        return;
    uint32_t max_rep = 0, max_remote = 0;
    for (uint64_t i = 0; i < count; ++i) {
        if (edges[i].rep > max_rep)
            max_rep = edges[i].rep;
        if (edges[i].remote > max_remote)
            max_remote = edges[i].remote;
    }
    void *d = NULL;
    int rc = pairs_to_device(edges, count, &d);
    if (rc == CCGPU_OK)
        rc = ccgpu_boundary_sort(NULL, (uint32_t *)d, count, max_rep, max_remote, NULL);
    if (rc == CCGPU_OK)
        rc = ccgpu_memcpy_d2h(edges, d, (size_t)count * sizeof(BoundaryEdge));
    ccgpu_free(d);
    if (rc != CCGPU_OK)
        ccb200_fail("boundary_edges_sort", rc);
}

uint64_t boundary_edges_dedup(BoundaryEdge *edges, uint64_t count)
{
    if (!edges || count <= 1)
        return count;
    void *d = NULL;
    uint64_t kept = count;
    int rc = pairs_to_device(edges, count, &d);
    if (rc == CCGPU_OK)
        rc = ccgpu_boundary_dedup(NULL, (uint32_t *)d, count, &kept, NULL);
    if (rc == CCGPU_OK)
        rc = ccgpu_memcpy_d2h(edges, d, (size_t)kept * sizeof(BoundaryEdge));
    ccgpu_free(d);
    if (rc != CCGPU_OK) {
        ccb200_fail("boundary_edges_dedup", rc);
        return count;
    }
    return kept;
}

/* --------------------------------------------------------- runtime utils */

void mpi_die_abort(MPI_Comm comm, const char *msg)
{
    (void)comm;
    fprintf(stderr, "%s\n", msg ? msg : "mpi_die_abort");
    fflush(stderr);
    exit(EXIT_FAILURE);
}

int runtime_default_threads(void)
{
    long t = sysconf(_SC_NPROCESSORS_ONLN);
    return t > 0 ? (int)t : 1;
}

/* --------------------------------------------------------------- vectors */

#define VEC_IMPL(NAME, VT, ET, SZ)                                                   \
    void NAME##_init(VT *v)                                                          \
    {                                                                                \
        v->data = NULL;                                                              \
        v->size = 0;                                                                 \
        v->cap = 0;                                                                  \
    }                                                                                \
    void NAME##_free(VT *v)                                                          \
    {                                                                                \
        free(v->data);                                                               \
        NAME##_init(v);                                                              \
    }                                                                                \
    void NAME##_reserve(VT *v, SZ new_cap, MPI_Comm comm)                            \
    {                                                                                \
        if (new_cap <= v->cap)                                                       \
            return;                                                                  \
        ET *p = (ET *)realloc(v->data, (size_t)new_cap * sizeof(ET));                \
        if (!p)                                                                      \
            mpi_die_abort(comm, "OOM: " #NAME "_reserve");                           \
        v->data = p;                                                                 \
        v->cap = new_cap;                                                            \
    }                                                                                \
    void NAME##_push(VT *v, ET x, MPI_Comm comm)                                     \
    {                                                                                \
        if (v->size == v->cap)                                                       \
            NAME##_reserve(v, v->cap ? 2 * v->cap : 4096, comm);                     \
        v->data[v->size++] = x;                                                      \
    }

VEC_IMPL(u32vec, U32Vec, uint32_t, uint64_t)
VEC_IMPL(u32veci, U32VecI, uint32_t, int)
VEC_IMPL(bevec, BEVec, BoundaryEdge, uint64_t)
VEC_IMPL(bpvec, BPVec, BoundaryPair, uint64_t)
