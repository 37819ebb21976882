/*
 * Internal core of the batched solver, shared by the packed-batch plans
 * (batch_cc.cu) and the request server (serve.cu).
 *
 * A batch is a list of graph descriptors: graph g's row pointers start at
 * row_ptr[gr[g].rp], its neighbour ids at col[gr[g].col] and its labels at
 * labels[gr[g].lab] (element offsets from three base pointers), so the
 * graphs may sit anywhere in device memory - packed back to back (plans) or
 * wherever a memory pool placed each request (server).
 */
#ifndef CCB200_BATCH_CORE_H
#define CCB200_BATCH_CORE_H

#include <vector>

#include "ccgpu_internal.h"

struct BGraph {
    uint64_t rp;  /* first row pointer (n + 1 entries, local 0 .. m) */
    uint64_t col; /* first neighbour id (m entries, local ids)       */
    uint64_t lab; /* first label (n entries)                         */
    uint64_t m;
    uint32_t n;
    uint32_t pad;
};

struct BatchClass {
    ccgpu_batch_class_opts o;
    std::vector<uint32_t> graphs; /* graphs of the class (indices into gr) */
    uint64_t vertices = 0, entries = 0;
    uint32_t tiles = 0;
    uint32_t *d_graphs = nullptr;
    size_t graphs_cap = 0;
    uint32_t *d_tile_g = nullptr, *d_tile_v0 = nullptr;
    size_t tile_cap = 0;
    unsigned long long *d_cnt = nullptr; /* [0] tile grab, [1] heavy count */
    uint64_t *d_heavy = nullptr;
    size_t heavy_cap = 0;
    uint32_t heavy_used = 0; /* capacity handed to the kernels */
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
};

struct BatchCore {
    ccgpu_ctx *ctx = nullptr;
    int sms = 148;
    ccgpu_batch_tuning tune;
    const uint64_t *row_ptr = nullptr;
    const uint32_t *col = nullptr;
    uint32_t *labels = nullptr;
    std::vector<BGraph> gr;
    BGraph *d_gr = nullptr;
    uint32_t *d_giants = nullptr, *d_comps = nullptr, *d_tiles_done = nullptr, *d_done = nullptr;
    uint32_t *d_pcnt = nullptr; /* persistent launches: [g_cap * 12] phase counters */
    int *d_err = nullptr;       /* persistent launches: 1 once a wait ran out      */
    unsigned long long *d_grab = nullptr; /* persistent launches: item counter */
    int persist_blocks = 0;     /* resident blocks of the persistent kernel per SM */
    size_t g_cap = 0;
    BatchClass cls[CCGPU_BATCH_CLASSES];
    cudaEvent_t fork = nullptr;
    void *h_stage = nullptr; /* pinned staging of the uploads */
    size_t stage_cap = 0;
    uint32_t *stash = nullptr; /* second-neighbour stash, indexed like labels */
    size_t stash_cap = 0;      /* entries (0: no stash)                      */
};

/* Validates and stores the tuning, creates the class streams and events. */
int batch_core_init(BatchCore *c, ccgpu_ctx *ctx, const ccgpu_batch_tuning *tuning);
void batch_core_free(BatchCore *c);
/* Reserves room for batches of up to `graphs` graphs, `tiles` tiles and
 * `heavy` queued rows per class, so that later batch_core_set calls
 * allocate nothing (device or pinned) while they fit. */
int batch_core_reserve(BatchCore *c, size_t graphs, size_t tiles, size_t heavy);
/* Sets the batch: classifies the graphs, builds every class's tile list
 * and uploads descriptors and tiles on `st` from pinned staging (the staging
 * stays in use until `st` passes the upload; sync = wait for it). */
int batch_core_set(BatchCore *c, const uint64_t *row_ptr, const uint32_t *col, uint32_t *labels,
                   const BGraph *gr, uint32_t G, cudaStream_t st, int sync);
/* Rebuilds and uploads class k's tile list after its options changed
 * (synchronous). */
int batch_core_retile(BatchCore *c, int k);
/* Gives the batch a second-neighbour stash of `entries` u32 (the extent of
 * the label array): sampling round 0 keeps each vertex's second neighbour
 * there and round 1 reads it instead of the row, in classes whose rows
 * average at least 8 entries. */
int batch_core_stash(BatchCore *c, size_t entries);
/* Enqueues the whole solve on st: per-graph outputs cleared, every class
 * on its own stream forked from st and joined back. */
int batch_core_enqueue(BatchCore *c, cudaStream_t st, int *kernels);
/* Enqueues class k's solve alone on st. */
int batch_core_enqueue_class(BatchCore *c, int k, cudaStream_t st, int *kernels);
/* Mean-row-length class of a graph. */
int batch_class_of(const ccgpu_batch_tuning &t, uint64_t n, uint64_t m);
int batch_check_tuning(ccgpu_batch_tuning *t);

#endif
