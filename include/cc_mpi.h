/*
 * cc_mpi.h - partitioned connected components.
 *
 * Drop-in for the reference's include/cc_mpi.h:29-47.  The partitions of
 * the group live in the HBM of one B200 and the whole solve - local CC per
 * partition, boundary radix sort, ghosts, exchange plan, merge rounds with
 * the delta halo exchange - runs there (see ccgpu_dist_cc in ccgpu.h).
 */
#ifndef CC_MPI_H
#define CC_MPI_H

#include <stdint.h>

#include "cc.h"
#include "cc_comm.h"
#include "graph_dist.h"

/* Reference include/cc_mpi.h:29-33.  Gd must be a graph of this group
 * (load_dist_csr_from_file / dist_csr_from_csr; any other whole-graph
 * DistCSRGraph is uploaded on first use).  chunk_size goes to the local CC
 * as in the reference (1 static, > 1 dynamic grab size, <= 0 default).
 * exchange_interval is the number of merge rounds between delta exchanges
 * (< 1 means 1).  On return, when labels_global is not NULL,
 * labels_global[v] is the smallest vertex id of v's component for all
 * n_global vertices - the contract the reference documents
 * (include/cc_mpi.h:26-27) but never fills (src/cc_mpi.c:227).  Like the
 * reference it prints "Number of connected components: C" (unless the
 * group is silenced, cc_comm.h).  Errors print a message and exit, as the
 * reference aborts (src/runtime_utils.c:9-14), unless
 * ccb200_set_exit_on_error(0) was called. */
void compute_connected_components_mpi_advanced(const DistCSRGraph *restrict Gd,
                                               uint32_t *restrict labels_global,
                                               int chunk_size,
                                               int exchange_interval,
                                               MPI_Comm comm);

/* Status-returning twin of the call above. */
int cc_mpi_solve(const DistCSRGraph *Gd, uint32_t *labels_global, int chunk_size,
                 int exchange_interval, MPI_Comm comm, ccgpu_dist_stats *stats);

/* Reference include/cc_mpi.h:41 (src/cc_mpi.c:765-792): number of distinct
 * labels below n_global. */
uint32_t count_connected_components(const uint32_t *restrict labels_global, uint32_t n_global);

/* Reference include/cc_mpi.h:47.  The host-thread count of the reference's
 * pthread pools; kept and reported, the device schedule does not use it. */
void cc_mpi_set_num_threads(int nthreads);
int cc_mpi_get_num_threads(void);

#endif /* CC_MPI_H */
