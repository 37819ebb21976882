/*
 * The reference's per-rank halo-exchange plan (include/exchange_plan.h) on
 * the partition group: each rank is a host thread with a per-rank view of
 * the group as its MPI_Comm.
 *
 *   build  need-from lists per owner in ghost order, then the reference's
 *          Alltoall of counts and Alltoallv of vertex ids as reads of the
 *          other ranks' published plans between two group barriers
 *          (src/exchange_plan.c:48-225)
 *   delta  pack (position, label) pairs of labels that fell below what was
 *          last sent, post them, take every source's pairs, unpack into
 *          ghost_labels by ghost index (src/exchange_plan.c:242-425); the
 *          neighbourhood all-to-all becomes pairwise mailboxes in the group,
 *          so only neighbours wait on each other
 *   start / finish / exchange  the legacy full exchange of send_labels_flat
 *          (src/exchange_plan.c:234-240,427-455) over the same mailboxes
 *
 * Failures set ccgpu_last_error() and, like the reference's MPI_Abort,
 * exit unless ccb200_set_exit_on_error(0) was called.
 */
#include <stdlib.h>
#include <string.h>

#include "exchange_plan.h"
#include "host_common.h"

static void *xalloc(size_t n)
{
    return malloc(n ? n : 1);
}

void exchangeplan_free(ExchangePlan *P)
{
    if (!P)
        return;
    free(P->sources);
    free(P->dests);
    free(P->need_from_counts);
    free(P->send_to_counts);
    free(P->need_from_displs);
    free(P->send_to_displs);
    free(P->need_from_flat);
    free(P->need_from_gidx_flat);
    free(P->send_to_flat);
    free(P->sendcounts);
    free(P->sdispls);
    free(P->recvcounts);
    free(P->rdispls);
    free(P->send_labels_flat);
    free(P->recv_labels_flat);
    memset(P, 0, sizeof(*P));
    P->comm_graph = MPI_COMM_NULL;
}

static int plan_fail(ExchangePlan *P, const char *what)
{
    int st = ccb200_set_error(CCGPU_ERR_OOM, "exchangeplan_build: %s", what);
    exchangeplan_free(P);
    ccb200_fail("exchangeplan_build", st);
    return 1;
}

int exchangeplan_build(ExchangePlan *P, const uint32_t *ghost_vertices, uint32_t ghost_count,
                       uint32_t n_global, MPI_Comm comm, OwnerFn owner_fn)
{
    if (!P)
        return 1;
    exchangeplan_free(P);
    if (!comm || !owner_fn || (ghost_count && !ghost_vertices)) {
        ccb200_fail("exchangeplan_build",
                    ccb200_set_error(CCGPU_ERR_INVALID, "exchangeplan_build: NULL argument"));
        return 1;
    }
    const int size = cc_group_size(comm), rank = cc_group_rank(comm);
    P->comm_size = size;
    P->comm_rank = rank;
    P->need_from_counts = (int *)calloc((size_t)size, sizeof(int));
    P->send_to_counts = (int *)calloc((size_t)size, sizeof(int));
    P->need_from_displs = (int *)calloc((size_t)size, sizeof(int));
    P->send_to_displs = (int *)calloc((size_t)size, sizeof(int));
    if (!P->need_from_counts || !P->send_to_counts || !P->need_from_displs ||
        !P->send_to_displs)
        return plan_fail(P, "out of memory (counts)");

    /* need-from lists: ghosts grouped by owner, ghost order kept */
    int *owner = (int *)xalloc((size_t)ghost_count * sizeof(int));
    if (!owner)
        return plan_fail(P, "out of memory (owners)");
    for (uint32_t gi = 0; gi < ghost_count; ++gi) {
        owner[gi] = owner_fn(ghost_vertices[gi], n_global, size);
        if (owner[gi] != rank && owner[gi] >= 0 && owner[gi] < size)
            P->need_from_counts[owner[gi]]++;
    }
    int total_need = 0;
    for (int p = 0; p < size; ++p) {
        P->need_from_displs[p] = total_need;
        total_need += P->need_from_counts[p];
    }
    P->total_need_from = total_need;
    P->need_from_flat = (uint32_t *)xalloc((size_t)total_need * sizeof(uint32_t));
    P->need_from_gidx_flat = (uint32_t *)xalloc((size_t)total_need * sizeof(uint32_t));
    int *fill = (int *)calloc((size_t)size, sizeof(int));
    if (!P->need_from_flat || !P->need_from_gidx_flat || !fill) {
        free(owner);
        free(fill);
        return plan_fail(P, "out of memory (need-from lists)");
    }
    for (uint32_t gi = 0; gi < ghost_count; ++gi) {
        const int o = owner[gi];
        if (o == rank || o < 0 || o >= size)
            continue;
        const int at = P->need_from_displs[o] + fill[o]++;
        P->need_from_flat[at] = ghost_vertices[gi];
        P->need_from_gidx_flat[at] = gi;
    }
    free(owner);
    free(fill);

    /* the Alltoall of counts and the Alltoallv of ids: every rank publishes
     * its plan and reads what the others need from it */
    void **slots = cc_group_slots(comm);
    slots[rank] = P;
    if (cc_group_barrier(comm) != 0) {
        exchangeplan_free(P);
        ccb200_fail("exchangeplan_build", CCGPU_ERR_TIMEOUT);
        return 1;
    }
    int total_send = 0;
    for (int p = 0; p < size; ++p) {
        const ExchangePlan *Q = (const ExchangePlan *)slots[p];
        P->send_to_counts[p] = p == rank ? 0 : Q->need_from_counts[rank];
        P->send_to_displs[p] = total_send;
        total_send += P->send_to_counts[p];
    }
    P->total_send_to = total_send;
    P->send_to_flat = (uint32_t *)xalloc((size_t)total_send * sizeof(uint32_t));
    if (P->send_to_flat)
        for (int p = 0; p < size; ++p) {
            if (!P->send_to_counts[p])
                continue;
            const ExchangePlan *Q = (const ExchangePlan *)slots[p];
            memcpy(P->send_to_flat + P->send_to_displs[p],
                   Q->need_from_flat + Q->need_from_displs[rank],
                   (size_t)P->send_to_counts[p] * sizeof(uint32_t));
        }
    /* nobody may change its published plan before everyone has read it */
    if (cc_group_barrier(comm) != 0 || !P->send_to_flat) {
        const int st = P->send_to_flat ? CCGPU_ERR_TIMEOUT : CCGPU_ERR_OOM;
        exchangeplan_free(P);
        ccb200_fail("exchangeplan_build", st);
        return 1;
    }

    /* neighbourhood: sources we receive from, destinations we send to */
    for (int p = 0; p < size; ++p) {
        P->indegree += P->need_from_counts[p] > 0;
        P->outdegree += P->send_to_counts[p] > 0;
    }
    P->sources = P->indegree ? (int *)malloc((size_t)P->indegree * sizeof(int)) : NULL;
    P->dests = P->outdegree ? (int *)malloc((size_t)P->outdegree * sizeof(int)) : NULL;
    P->sendcounts = P->outdegree ? (int *)malloc((size_t)P->outdegree * sizeof(int)) : NULL;
    P->sdispls = P->outdegree ? (int *)malloc((size_t)P->outdegree * sizeof(int)) : NULL;
    P->recvcounts = P->indegree ? (int *)malloc((size_t)P->indegree * sizeof(int)) : NULL;
    P->rdispls = P->indegree ? (int *)malloc((size_t)P->indegree * sizeof(int)) : NULL;
    if ((P->indegree && (!P->sources || !P->recvcounts || !P->rdispls)) ||
        (P->outdegree && (!P->dests || !P->sendcounts || !P->sdispls)))
        return plan_fail(P, "out of memory (neighbourhood)");
    int ii = 0, oo = 0;
    for (int p = 0; p < size; ++p) {
        if (P->need_from_counts[p] > 0) {
            P->sources[ii] = p;
            P->recvcounts[ii] = P->need_from_counts[p];
            P->rdispls[ii] = P->need_from_displs[p];
            ++ii;
        }
        if (P->send_to_counts[p] > 0) {
            P->dests[oo] = p;
            P->sendcounts[oo] = P->send_to_counts[p];
            P->sdispls[oo] = P->send_to_displs[p];
            ++oo;
        }
    }
    P->comm_graph = (P->indegree || P->outdegree) ? comm : MPI_COMM_NULL;
    if (P->total_send_to)
        P->send_labels_flat = (uint32_t *)malloc((size_t)P->total_send_to * sizeof(uint32_t));
    if (P->total_need_from)
        P->recv_labels_flat = (uint32_t *)malloc((size_t)P->total_need_from * sizeof(uint32_t));
    if ((P->total_send_to && !P->send_labels_flat) ||
        (P->total_need_from && !P->recv_labels_flat))
        return plan_fail(P, "out of memory (label buffers)");
    return 0;
}

/* ----------------------------------------------------------- exchanges */

/* Appends a source's posted pairs to the receive buffer. */
struct take_u64 {
    uint64_t *buf;
    int used, cap, got;
};

static void copy_u64(void *arg, const void *buf, int off, int cnt)
{
    struct take_u64 *t = (struct take_u64 *)arg;
    int n = cnt;
    if (n > t->cap - t->used)
        n = t->cap - t->used;
    if (n > 0)
        memcpy(t->buf + t->used, (const uint64_t *)buf + off, (size_t)n * sizeof(uint64_t));
    t->got = n > 0 ? n : 0;
    t->used += t->got;
}

struct take_u32 {
    uint32_t *dst;
    int want;
};

static void copy_u32(void *arg, const void *buf, int off, int cnt)
{
    struct take_u32 *t = (struct take_u32 *)arg;
    const int n = cnt < t->want ? cnt : t->want;
    if (n > 0)
        memcpy(t->dst, (const uint32_t *)buf + off, (size_t)n * sizeof(uint32_t));
}

static int grow_u64(uint64_t **buf, int *cap, int want)
{
    if (*buf && *cap >= want)
        return 0;
    const int n = want > 0 ? want : 1;
    uint64_t *nb = (uint64_t *)realloc(*buf, (size_t)n * sizeof(uint64_t));
    if (!nb)
        return -1;
    *buf = nb;
    *cap = n;
    return 0;
}

void exchangeplan_exchange_delta(const ExchangePlan *P, const uint32_t *comp_label,
                                 const uint32_t *comp_of, uint32_t v_start, uint32_t v_end,
                                 uint32_t *prev_sent, uint32_t *ghost_labels, MPI_Comm comm,
                                 uint64_t **sendbuf_io, int *sendcap_io, uint64_t **recvbuf_io,
                                 int *recvcap_io)
{
    (void)comm;
    if (!P || P->comm_graph == MPI_COMM_NULL)
        return;
    if (!sendbuf_io || !sendcap_io || !recvbuf_io || !recvcap_io ||
        grow_u64(sendbuf_io, sendcap_io, P->total_send_to) ||
        grow_u64(recvbuf_io, recvcap_io, P->total_need_from)) {
        ccb200_fail("exchangeplan_exchange_delta",
                    ccb200_set_error(CCGPU_ERR_OOM, "exchangeplan_exchange_delta: buffers"));
        return;
    }
    const int size = P->comm_size;
    int off[CCGPU_MAX_PARTS], cnt[CCGPU_MAX_PARTS];
    memset(cnt, 0, sizeof(int) * (size_t)size);
    memset(off, 0, sizeof(int) * (size_t)size);
    /* pack: per destination, (position in its need-from list, label) of
     * every label below what was sent last time */
    uint64_t *sb = *sendbuf_io;
    int total = 0;
    for (int k = 0; k < P->outdegree; ++k) {
        const int dest = P->dests[k], base = P->send_to_displs[dest];
        off[dest] = total;
        for (int i = 0; i < P->send_to_counts[dest]; ++i) {
            const uint32_t v = P->send_to_flat[base + i];
            uint32_t lbl = v;
            if (v >= v_start && v < v_end)
                lbl = comp_label[comp_of[v - v_start]];
            if (lbl < prev_sent[base + i]) {
                prev_sent[base + i] = lbl;
                sb[total++] = ((uint64_t)(uint32_t)i << 32) | lbl;
            }
        }
        cnt[dest] = total - off[dest];
    }
    cc_group *me = P->comm_graph;
    int rc = cc_group_post(me, sb, off, cnt, P->outdegree);
    /* take every source's pairs (at most its need-from count for us) and
     * unpack them by ghost index */
    struct take_u64 t = {*recvbuf_io, 0, *recvcap_io, 0};
    for (int k = 0; rc == 0 && k < P->indegree; ++k) {
        const int src = P->sources[k], base = P->need_from_displs[src];
        const int from = t.used;
        rc = cc_group_take(me, src, copy_u64, &t);
        for (int i = from; rc == 0 && i < from + t.got; ++i) {
            const uint64_t pr = t.buf[i];
            const uint32_t pos = (uint32_t)(pr >> 32);
            if ((int)pos < P->need_from_counts[src])
                ghost_labels[P->need_from_gidx_flat[base + (int)pos]] = (uint32_t)pr;
        }
    }
    /* the send buffer may be reused once every destination has read it */
    if (rc == 0)
        rc = cc_group_drain(me);
    if (rc != 0)
        ccb200_fail("exchangeplan_exchange_delta", rc);
}

void exchangeplan_exchange_start(ExchangePlan *P, MPI_Request *req)
{
    if (!P || !req)
        return;
    *req = MPI_REQUEST_NULL;
    if (P->comm_graph == MPI_COMM_NULL || (!P->total_send_to && !P->total_need_from))
        return;
    const int rc = cc_group_post(P->comm_graph, P->send_labels_flat, P->send_to_displs,
                                 P->send_to_counts, P->outdegree);
    if (rc != 0) {
        ccb200_fail("exchangeplan_exchange_start", rc);
        return;
    }
    *req = (MPI_Request)(void *)P; /* pending: finish takes and drains */
}

void exchangeplan_exchange_finish(ExchangePlan *P, uint32_t *ghost_labels, MPI_Request *req)
{
    if (!P || !ghost_labels || !req)
        return;
    if (*req != MPI_REQUEST_NULL) {
        int rc = 0;
        for (int k = 0; rc == 0 && k < P->indegree; ++k) {
            const int src = P->sources[k];
            struct take_u32 t = {P->recv_labels_flat + P->need_from_displs[src],
                                 P->need_from_counts[src]};
            rc = cc_group_take(P->comm_graph, src, copy_u32, &t);
        }
        if (rc == 0)
            rc = cc_group_drain(P->comm_graph);
        *req = MPI_REQUEST_NULL;
        if (rc != 0) {
            ccb200_fail("exchangeplan_exchange_finish", rc);
            return;
        }
    }
    for (int i = 0; i < P->total_need_from; ++i)
        ghost_labels[P->need_from_gidx_flat[i]] = P->recv_labels_flat[i];
}

void exchangeplan_exchange(ExchangePlan *P, uint32_t *ghost_labels, MPI_Comm comm)
{
    (void)comm;
    MPI_Request req;
    exchangeplan_exchange_start(P, &req);
    exchangeplan_exchange_finish(P, ghost_labels, &req);
}
