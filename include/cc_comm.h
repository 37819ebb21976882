/*
 * cc_comm.h - the partition group that stands in for the reference's MPI
 * communicator.
 *
 * The reference runs one MPI rank per partition (src/mpi_cc_benchmark.c:33,
 * src/graph_dist.c:142-342).  Here one process owns every partition of a
 * graph and keeps them resident in the HBM of one B200; a cc_group carries
 * the partition count (the reference's -np) and the settings of the
 * partitioned solver.  MPI_Comm is typedef'd to it so that the
 * reference's prototypes (cc_mpi.h, graph_dist.h, exchange_plan.h, ...)
 * keep their exact shape.  Code that also links a real MPI defines
 * CCB200_EXTERNAL_MPI before including these headers and passes cc_group
 * pointers explicitly.
 */
#ifndef CC_COMM_H
#define CC_COMM_H

#include <stdint.h>

#include "ccgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cc_group cc_group;
typedef struct cc_request cc_request;

#ifndef CCB200_EXTERNAL_MPI
typedef cc_group *MPI_Comm;
typedef cc_request *MPI_Request;
#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_COMM_WORLD (cc_group_world())
#endif

/* A group of `parts` partitions (1 <= parts <= CCGPU_MAX_PARTS). */
cc_group *cc_group_create(int parts);
void cc_group_free(cc_group *g);
/* Number of partitions (the reference's MPI_Comm_size). */
int cc_group_size(const cc_group *g);
/* Rank a per-rank view stands for; 0 for a group itself. */
int cc_group_rank(const cc_group *g);

/* The process-wide group: its size is the CCB200_PARTITIONS environment
 * variable when set, else 1, until cc_group_set_world_size changes it. */
cc_group *cc_group_world(void);
int cc_group_set_world_size(int parts);

/* Per-rank views, for code written rank by rank against the reference's
 * per-rank calls (exchange_plan.h): view r acts as rank r of a size-`parts`
 * communicator.  The collective calls made through views (exchangeplan_build,
 * exchangeplan_exchange_delta, ...) must be made by `parts` host threads,
 * one per view, the way MPI ranks make them; they meet in the group. */
cc_group *cc_group_view(cc_group *g, int rank);
/* Blocks until every rank of the view's group has called it. */
int cc_group_barrier(cc_group *view);

/* 1 (default): the partitioned solver prints the reference's summary lines
 * ("CC merge converged in N rounds", "Number of connected components: C");
 * 2: also the per-phase lines; 0: silent. */
void cc_group_set_verbose(cc_group *g, int verbose);
int cc_group_verbose(const cc_group *g);
/* Statistics of the group's last compute_connected_components_mpi_advanced
 * call; returns 0 when there was one. */
int cc_group_last_stats(const cc_group *g, ccgpu_dist_stats *out);

#ifdef __cplusplus
}
#endif

#endif /* CC_COMM_H */
