/*
 * graph_dist.h - the partitioned CSR graph.
 *
 * Drop-in for the reference's include/graph_dist.h:15-49: same struct layout
 * and prototypes.  One process owns every partition of the group, so a
 * loaded DistCSRGraph describes the whole graph: n_local == n_global,
 * [v_start, v_end) == [0, n_global), row_ptr/col_idx are the full CSR with
 * global neighbour ids (as the reference's col_idx, include/graph_dist.h:
 * 12-13).  part_bounds/part_size/part_kind carry the group's partition
 * bounds exactly as the reference fills them (src/graph_dist.c:179-210):
 * edge-balanced bounds when use_edge and the group has more than one
 * partition, otherwise NULL/0/0 and block ranges.
 */
#ifndef GRAPH_DIST_H
#define GRAPH_DIST_H

#include <stdint.h>

#include "cc_comm.h"
#include "graph.h"

typedef struct
{
    uint32_t n_global;
    uint64_t m_global;
    uint32_t n_local;
    uint64_t m_local;
    uint32_t v_start;
    uint32_t v_end;
    uint64_t *row_ptr;
    uint32_t *col_idx;
    uint32_t *part_bounds;
    int part_size;
    int part_kind;
} DistCSRGraph;

/* Reference include/graph_dist.h:40-45.  Reads the file with
 * load_csr_from_file (".mat", or ".csrbin" for graphs MAT v5 cannot hold),
 * computes the group's partition bounds on the device and keeps the graph
 * resident in HBM for compute_connected_components_mpi_advanced (the upload
 * is part of loading, outside the solver's timed region as in the
 * reference, src/mpi_cc_benchmark.c:177-179 vs :207-211).  symmetrize and
 * drop_self_loops are ignored, as in the reference.  Returns the loader's
 * code (0 ok, 1/2/3 .mat errors, 99 bad extension, -1 .mtx), or 100 when
 * the device could not take the graph. */
int load_dist_csr_from_file(const char *path,
                            int symmetrize,
                            int drop_self_loops,
                            int use_edge,
                            DistCSRGraph *out,
                            MPI_Comm comm);

/* Builds a DistCSRGraph from an in-memory CSR the caller owns (no copy of
 * the host arrays; free_dist_csr must then not be called - use
 * free_dist_csr_view).  Same partitioning and device residency as the
 * loader.  Returns 0 or 100. */
int dist_csr_from_csr(const CSRGraph *g, int use_edge, DistCSRGraph *out, MPI_Comm comm);

/* Reference include/graph_dist.h:49: frees the arrays, the device copy and
 * zeroes the struct. */
void free_dist_csr(DistCSRGraph *graph);
/* Releases only the device copy and part_bounds of a dist_csr_from_csr graph. */
void free_dist_csr_view(DistCSRGraph *graph);

#endif /* GRAPH_DIST_H */
