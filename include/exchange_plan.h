/*
 * exchange_plan.h - the reference's per-rank halo-exchange plan
 * (include/exchange_plan.h of CC_mpi), with the same struct layout and
 * prototypes.
 *
 * The partitioned solver does its exchanges inside HBM; these calls serve
 * code written rank by rank against the reference's API.  Each rank is a
 * host thread holding a per-rank view of a partition group
 * (cc_group_view, include/cc_comm.h) as its MPI_Comm; the collective calls
 * meet in the group the way MPI ranks meet in a communicator.  The
 * neighbourhood exchanges synchronise only between neighbours, so a rank
 * whose plan has no neighbours (comm_graph == MPI_COMM_NULL) may skip them,
 * as in the reference.
 */
#ifndef EXCHANGE_PLAN_H
#define EXCHANGE_PLAN_H

#include <stdint.h>

#include "cc_comm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int (*OwnerFn)(uint32_t v, uint32_t n_global, int comm_size);

/* Per-rank communication state of the halo exchanges
 * (include/exchange_plan.h:10-40 of the reference). */
typedef struct {
    int comm_size;
    int comm_rank;

    int indegree;
    int outdegree;
    int *sources;
    int *dests;
    MPI_Comm comm_graph;

    int *need_from_counts;
    int *send_to_counts;
    int *need_from_displs;
    int *send_to_displs;

    uint32_t *need_from_flat;
    uint32_t *send_to_flat;
    uint32_t *need_from_gidx_flat;

    int total_need_from;
    int total_send_to;

    int *sendcounts;
    int *sdispls;
    int *recvcounts;
    int *rdispls;

    uint32_t *send_labels_flat;
    uint32_t *recv_labels_flat;
} ExchangePlan;

/* Builds the plan of this rank from its sorted unique ghost vertices
 * (reference include/exchange_plan.h:51-56, src/exchange_plan.c:48-225):
 * the ghosts each owner must send, exchanged with every other rank.
 * Collective over the group.  Returns 0. */
int exchangeplan_build(ExchangePlan *P, const uint32_t *ghost_vertices, uint32_t ghost_count,
                       uint32_t n_global, MPI_Comm comm, OwnerFn owner_fn);

/* Frees what the plan owns; safe on partially built plans
 * (include/exchange_plan.h:59, src/exchange_plan.c:17-46). */
void exchangeplan_free(ExchangePlan *P);

/* Delta exchange (include/exchange_plan.h:61-83, src/exchange_plan.c:242-425):
 * a label goes to a neighbour only when it fell below what was sent last
 * time (prev_sent, length total_send_to, updated); received labels land
 * in ghost_labels.  The label of a vertex v this rank owns is
 * comp_label[comp_of[v - v_start]].  sendbuf/recvbuf are grown with
 * realloc as needed.  Collective over the rank's neighbours. */
void exchangeplan_exchange_delta(const ExchangePlan *P, const uint32_t *comp_label,
                                 const uint32_t *comp_of, uint32_t v_start, uint32_t v_end,
                                 uint32_t *prev_sent, uint32_t *ghost_labels, MPI_Comm comm,
                                 uint64_t **sendbuf_io, int *sendcap_io, uint64_t **recvbuf_io,
                                 int *recvcap_io);

/* Legacy full exchange (include/exchange_plan.h:84-106,
 * src/exchange_plan.c:234-240,427-455): the caller fills
 * send_labels_flat; start sends it, finish receives into recv_labels_flat
 * and scatters it into ghost_labels. */
void exchangeplan_exchange_start(ExchangePlan *P, MPI_Request *req);
void exchangeplan_exchange_finish(ExchangePlan *P, uint32_t *ghost_labels, MPI_Request *req);
void exchangeplan_exchange(ExchangePlan *P, uint32_t *ghost_labels, MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif /* EXCHANGE_PLAN_H */
