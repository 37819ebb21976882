/*
 * Internal entry of the local-CC kernels, shared by the single-graph API
 * (local_cc.cu), the partitioned solver (dist_cc.cu) and the batched solver
 * (batch.cu).
 *
 * A solve may cover several independent "segments": vertex ranges
 * [seg[s], seg[s+1]) with no edge between ranges (the partitions of the
 * partitioned path, the graphs of a batch).  Each segment gets its own giant
 * root for the skip in the finish pass; labels are global vertex ids.
 */
#ifndef CCB200_LOCAL_CC_H
#define CCB200_LOCAL_CC_H

#include "ccgpu_internal.h"

struct LocalCCArgs {
    const uint64_t *row_ptr;  /* [n+1] (device)                         */
    const uint32_t *col;      /* [m]   (device)                         */
    uint32_t n;
    uint64_t m;
    uint32_t *labels;         /* [n] out: min id of the component       */
    const uint64_t *seg;      /* [nseg+1] segment vertex offsets or NULL */
    uint32_t nseg;            /* 1 when seg is NULL                      */
    ccgpu_cc_opts o;          /* resolved options                        */
    int seg_filter;           /* 1: ignore edges whose endpoints lie in
                               * different segments (the local subgraph
                               * of each partition, reference
                               * src/cc_mpi.c:252-297)                  */
    int stash;                /* 1: scratch holds each vertex's second
                               * neighbour, written by sampling round 0
                               * (same sector as the first) and read by
                               * round 1 instead of its row            */
    const uint64_t *row_end;  /* [n] or NULL: row v is [row_ptr[v],
                               * row_end[v]) instead of [row_ptr[v],
                               * row_ptr[v+1]) - rows given as sub-ranges
                               * of a larger column array (the local
                               * entries of sorted partition rows)     */
};

/* Device counters a solve leaves behind (for stats). */
struct LocalCCCounters {
    unsigned long long grab;
    uint32_t heavy_count;
    uint32_t pad;
    unsigned long long finish_rows;
    unsigned long long finish_edges;
};

struct LocalCCScratch {
    LocalCCCounters *counters;
    uint32_t *heavy_list;
    uint32_t heavy_cap;
    uint32_t *giants; /* [nseg] */
    uint32_t *stash;  /* [n] second neighbours, NULL unless args.stash */
};

/* Resolves defaults (NULL in -> defaults); CCGPU_ERR_INVALID on bad values. */
int cc_local_resolve_opts(const ccgpu_cc_opts *in, ccgpu_cc_opts *out);
/* Lays out the scratch of one solve (c->base NULL: sizing pass). */
void cc_local_carve(cc_carve *c, LocalCCScratch *s, const LocalCCArgs &a);
/* Launches the whole solve on `st`.  init_done: labels already hold the
 * initial forest and the counters are zeroed; sampled: step 1 already ran. */
int cc_local_run(ccgpu_ctx *ctx, const LocalCCArgs &a, const LocalCCScratch &s, cudaStream_t st,
                 int init_done, int sampled);
/* Launches only the init (+ first hook) pass. */
int cc_local_init(ccgpu_ctx *ctx, const LocalCCArgs &a, const LocalCCScratch &s,
                  cudaStream_t st);
/* Launches step 1 for vertices [v_lo, v_hi) only. */
int cc_local_sample_range(ccgpu_ctx *ctx, const LocalCCArgs &a, uint32_t v_lo, uint32_t v_hi,
                          cudaStream_t st);

#endif
