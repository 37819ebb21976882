/*
 * ccgpu.h - the thin C ABI between host code and the sm_100a kernels of the
 * B200 connected-components engine.
 *
 * Everything here takes plain pointers and sizes.  "d_" pointers are device
 * (HBM) pointers, "h_" pointers are host pointers; `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream).
 *
 * Every entry point returns a ccgpu_status; on failure a message is kept per
 * host thread and returned by ccgpu_last_error().  Kernels never trap: device
 * side waits are bounded and report CCGPU_ERR_TIMEOUT through the status.
 *
 * Labels produced by every solver are the minimum vertex id of each vertex's
 * component - the output contract of the reference's
 * compute_connected_components_mpi_advanced (include/cc_mpi.h:26-27) and the
 * value its pthreads label propagation converges to
 * (src/cc_pthreads.c:32-73,169-170).  Inputs are symmetric CSR graphs, as the
 * reference requires (its loader neither symmetrises nor drops self loops,
 * src/graph.c:17-18); neighbour ids >= n are ignored, as the reference's
 * merge ignores them (src/cc_mpi.c:269,389).
 */
#ifndef CCGPU_H
#define CCGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    CCGPU_OK = 0,
    CCGPU_ERR_INVALID = 1,  /* bad argument (NULL pointer, size, option)   */
    CCGPU_ERR_CUDA = 2,     /* a CUDA runtime call failed                   */
    CCGPU_ERR_OOM = 3,      /* a device or pinned-host allocation failed    */
    CCGPU_ERR_TIMEOUT = 4,  /* a bounded device-side wait ran out           */
    CCGPU_ERR_LIMIT = 5,    /* a size is above a stated maximum             */
    CCGPU_ERR_NODEVICE = 6, /* no CUDA device, or not an sm_100 device      */
    CCGPU_ERR_IO = 7,       /* file could not be read or written            */
    CCGPU_ERR_FORMAT = 8    /* file is not in a supported format            */
} ccgpu_status;

/* Message of the last failing call on this host thread ("" if none). */
const char *ccgpu_last_error(void);
/* Empties this thread's error message (lets callers of the void reference
 * calls tell success from failure). */
void ccgpu_clear_error(void);
/* Library version, major*10000 + minor*100 + patch. */
int ccgpu_version(void);
/* Checks that a usable sm_100 device is current.  CCGPU_ERR_NODEVICE if not. */
int ccgpu_device_check(void);

/* ------------------------------------------------------------------------
 * Contexts.  A context owns the device scratch (grow-only arena) that the
 * solvers need beyond their inputs and outputs.  Calls that share a context
 * must not overlap in time; use one context per concurrent host caller.
 * NULL as a context argument means the calling thread's device default
 * context, created on first use.
 * ---------------------------------------------------------------------- */
typedef struct ccgpu_ctx ccgpu_ctx;
int ccgpu_ctx_create(ccgpu_ctx **out);
void ccgpu_ctx_destroy(ccgpu_ctx *ctx);
/* Bytes of device scratch the context holds right now. */
size_t ccgpu_ctx_scratch_bytes(const ccgpu_ctx *ctx);
/* Kernels launched through the context so far (NULL = this thread's
 * default context). */
uint64_t ccgpu_ctx_launches(const ccgpu_ctx *ctx);

/* Launch profiler: when on, every kernel the context launches is bracketed
 * by CUDA events on its stream.  ccgpu_prof_collect synchronises on the
 * recorded events, writes the summed milliseconds and launch counts per
 * kernel id (arrays of ccgpu_prof_kernels() entries, either may be NULL)
 * since the previous collect, and starts a new window. */
int ccgpu_prof_enable(ccgpu_ctx *ctx, int on);
int ccgpu_prof_collect(ccgpu_ctx *ctx, double *ms, uint64_t *launches);
int ccgpu_prof_kernels(void);
const char *ccgpu_prof_name(int kernel_id);

/* ------------------------------------------------------------------------
 * Device memory and device-resident graphs (used by the host C layer).
 * ---------------------------------------------------------------------- */
int ccgpu_alloc(void **d_ptr, size_t bytes);
void ccgpu_free(void *d_ptr);
int ccgpu_memcpy_h2d(void *d_dst, const void *h_src, size_t bytes);
int ccgpu_memcpy_d2h(void *h_dst, const void *d_src, size_t bytes);

/* A CSR copied to HBM once and reused by many solves.  ccgpu_graph_free
 * waits for the device and keeps the arrays of one freed graph per device
 * for the next upload or CSC transposition that fits in them (they are
 * freed when a later graph needs more memory than is left). */
typedef struct ccgpu_graph ccgpu_graph;
int ccgpu_graph_upload(const uint64_t *h_row_ptr, const uint32_t *h_col_idx, uint32_t n,
                       uint64_t m, ccgpu_graph **out);
void ccgpu_graph_free(ccgpu_graph *g);
/* The CSC form of a .mat sparse matrix (column starts jc[ncols+1], row
 * indices ir[nnz], host arrays) transposed into a device-resident CSR graph
 * on the device: row r lists the columns c holding an entry (r, c) in
 * ascending order, and entries whose row index is not below nrows are
 * dropped - the count / prefix-sum / scatter of the reference's loader
 * (src/graph.c:91-117), done here as a radix sort of (row, column) keys.
 * Copy the result to the host with ccgpu_memcpy_d2h if needed. */
int ccgpu_graph_from_csc(const uint64_t *h_jc, const uint32_t *h_ir, uint32_t nrows,
                         uint32_t ncols, uint64_t nnz, ccgpu_graph **out);
const uint64_t *ccgpu_graph_row_ptr(const ccgpu_graph *g);
const uint32_t *ccgpu_graph_col_idx(const ccgpu_graph *g);
uint32_t ccgpu_graph_n(const ccgpu_graph *g);
uint64_t ccgpu_graph_m(const ccgpu_graph *g);
/* A device array of n labels that belongs to the graph: allocated on the
 * first call, kept with the graph's arrays by ccgpu_graph_free, so a load /
 * solve / free cycle with host output allocates it once. */
int ccgpu_graph_label_array(ccgpu_graph *g, uint32_t **d_labels);

/* ------------------------------------------------------------------------
 * Local CC (the kernel behind compute_connected_components_pthreads,
 * include/cc.h:27-28 of the reference).
 *
 * Algorithm: union-find over a CSR in HBM.  Roots are hooked larger-id
 * under smaller-id with atomicCAS, so each tree's root is its minimum id.
 *   1. sample   link every vertex with its first `sample_rounds` neighbours
 *   2. shortcut pointer-jump every vertex to its root
 *   3. giant    most frequent root of 1024 seeded samples
 *   4. finish   link the remaining neighbours of every vertex outside the
 *               giant tree; degree-binned: a CTA gathers the short rows and
 *               walks them edge-parallel, a warp takes each row of >= 32
 *               entries with 16-byte loads, rows above `heavy_degree` are
 *               queued and split across all CTAs
 *   5. shortcut labels[v] = root(v)
 * sample_rounds = 0 turns steps 1-3 off (every row is linked in step 4).
 * ---------------------------------------------------------------------- */
typedef struct {
    int chunk_size;     /* vertices a CTA takes per work grab in step 4;
                         * 1 = static blocks, <= 0 = 4096 (the reference's
                         * DEFAULT_CHUNK_SIZE, include/cc.h:7)               */
    int sample_rounds;  /* neighbours linked per vertex in step 1 (0..8);
                         * < 0 = default (2)                                  */
    int heavy_degree;   /* rows longer than this go to the grid-wide queue;
                         * <= 0 = default (8192)                              */
    int skip_giant;     /* 1 (default) = step 4 skips the giant tree;
                         * 0 = link every remaining neighbour               */
    int hook_mode;      /* bit mask, < 0 = default (CADENCE | MINHOOK):
                         *  1 FIRST: the init pass hooks v under its first
                         *    neighbour when that is smaller (plain store,
                         *    no walk); step 1 links the rest
                         *  2 LAZY: a root is hooked under the smaller
                         *    endpoint itself instead of walking to its root
                         *  4 CADENCE: one launch per sampled neighbour with a
                         *    shortcut pass after each
                         *  8 MINHOOK: sampling only builds a valid forest:
                         *    roots are lowered with fire-and-forget atomicMin
                         *    (no CAS retry), and step 4 links every entry of
                         *    each row outside the giant tree, sampled ones
                         *    included                                        */
} ccgpu_cc_opts;

#define CCGPU_HOOK_FIRST 1
#define CCGPU_HOOK_LAZY 2
#define CCGPU_HOOK_CADENCE 4
#define CCGPU_HOOK_MINHOOK 8

typedef struct {
    uint32_t giant_label;   /* root found in step 3 (UINT32_MAX if off)      */
    uint32_t heavy_rows;    /* rows handled by the grid-wide queue           */
    uint32_t components;    /* number of distinct labels (roots)             */
    uint32_t kernels;       /* kernel launches this call made                */
    uint64_t finish_rows;   /* rows step 4 linked (outside the giant tree)   */
    uint64_t finish_edges;  /* row entries step 4 linked                     */
} ccgpu_cc_stats;

/* Fills opts with the defaults. */
void ccgpu_cc_opts_default(ccgpu_cc_opts *opts);

/* labels[v] = min vertex id of v's component, for a device-resident CSR
 * (d_row_ptr[n+1], d_col_idx[m]).  opts may be NULL (defaults).  stats may be
 * NULL; when non-NULL the call synchronises `stream` to fill it.  Otherwise
 * the call is asynchronous on `stream`. */
int ccgpu_local_cc(ccgpu_ctx *ctx, const uint64_t *d_row_ptr, const uint32_t *d_col_idx,
                   uint32_t n, uint64_t m, uint32_t *d_labels,
                   const ccgpu_cc_opts *opts, ccgpu_cc_stats *stats, void *stream);

/* Same computation from host buffers: copies h_row_ptr/h_col_idx to HBM
 * (column copies pipelined with the sampling kernel), solves, and copies the
 * labels back to h_labels.  Synchronous.  Pinned host buffers go fastest. */
int ccgpu_local_cc_host(ccgpu_ctx *ctx, const uint64_t *h_row_ptr, const uint32_t *h_col_idx,
                        uint32_t n, uint64_t m, uint32_t *h_labels,
                        const ccgpu_cc_opts *opts, ccgpu_cc_stats *stats);

/* ------------------------------------------------------------------------
 * Partitioned CC (the kernels behind compute_connected_components_mpi_
 * advanced, reference include/cc_mpi.h:29-33 and src/cc_mpi.c:221-763).
 *
 * The graph is cut into `parts` contiguous vertex ranges exactly as the
 * reference cuts it over MPI ranks (src/graph_dist.c:22-92), and every range
 * stays resident in HBM:
 *   1. bounds   edge+vertex weighted cuts (or block ranges) on the device
 *   2. local    union-find CC of each range's local subgraph
 *   3. pairs    (rep, remote) for every cut edge, packed as sort keys
 *   4. sort     LSD radix sort of the keys, dedup, ghost ids, plan ranges
 *   5. merge    rounds of hook + pointer jumps; every `exchange_interval`
 *               rounds, or when nothing changed, the labels owners changed
 *               since the last exchange travel as (position, label) pairs
 *               between the ranges (the reference's delta exchange,
 *               src/exchange_plan.c:242-425)
 *   6. labels   labels[v] = min vertex id of v's component
 * The round and exchange schedule is the reference's (src/cc_mpi.c:535-710);
 * each round reads the previous round's labels, so the round count is
 * deterministic.
 * ---------------------------------------------------------------------- */
#define CCGPU_MAX_PARTS 256

typedef struct {
    int parts;              /* number of partitions (the reference's -np)   */
    int use_edge;           /* 1: edge-balanced bounds (the reference's
                             * benchmark), 0: block vertex ranges           */
    int chunk_size;         /* passed to the local CC as in the reference   */
    int exchange_interval;  /* merge rounds between exchanges (< 1 = 1)     */
    int verbose;            /* 1: print the reference's phase lines         */
} ccgpu_dist_opts;

typedef struct {
    int rounds;             /* merge rounds ("CC merge converged in N")     */
    int exchanges;          /* delta exchanges performed                    */
    int sort_passes;        /* radix passes over the boundary keys          */
    int pad;
    uint64_t boundary_raw;  /* cut edges (before dedup), all partitions     */
    uint64_t pair_count;    /* distinct (rep, remote) pairs                 */
    uint64_t ghost_count;   /* distinct remote vertices, summed             */
    uint64_t rep_count;     /* local components, summed                     */
    uint64_t roots;         /* components of the whole graph                */
    uint64_t sent_pairs;    /* (position, label) pairs moved in exchanges   */
    double ms_bounds, ms_local, ms_pairs, ms_sort, ms_ghosts, ms_merge, ms_total;
    uint64_t sorted_keys;   /* boundary keys the radix sort ordered         */
    uint64_t local_entries; /* entries of the partitions' local subgraphs   */
    int sorted_rows;        /* 1: the boundary pairs came from the sorted-row
                             * passes (rows strictly ascending), 0: from the
                             * gather pass                                  */
    int row_runs;           /* 1: the local subgraphs were read in place as
                             * each row's run inside its own partition (rows
                             * ascending, 2-8 partitions), 0: a local CSR
                             * was built                                    */
} ccgpu_dist_stats;

void ccgpu_dist_opts_default(ccgpu_dist_opts *opts);

/* d_labels (may be NULL) receives the labels; h_bounds (may be NULL,
 * parts+1 entries) the partition bounds.  Synchronous (the merge loop reads
 * two flags per round).  Needs n >= parts. */
int ccgpu_dist_cc(ccgpu_ctx *ctx, const uint64_t *d_row_ptr, const uint32_t *d_col_idx,
                  uint32_t n, uint64_t m, const ccgpu_dist_opts *opts, uint32_t *d_labels,
                  uint32_t *h_bounds, ccgpu_dist_stats *stats, void *stream);

/* Partition bounds only (step 1), into h_bounds[parts+1]. */
int ccgpu_partition_bounds(const uint64_t *d_row_ptr, uint32_t n, int parts, int use_edge,
                           uint32_t *h_bounds, void *stream);

/* Generic u64 key sort (the LSD radix sort behind the boundary sort): sorts
 * d_keys[0..count) ascending on bits [0, bits) (higher bits must be zero),
 * using d_alt (same size) as the other buffer; *in_alt = 1 when the result
 * ended in d_alt.  Asynchronous on `stream`. */
int ccgpu_sort_keys(ccgpu_ctx *ctx, uint64_t *d_keys, uint64_t *d_alt, uint64_t count, int bits,
                    int *in_alt, void *stream);
/* Writes the distinct values of the sorted d_keys[0..count) to d_out
 * (may not alias d_keys); *out_count receives their number.  Synchronous. */
int ccgpu_unique_keys(ccgpu_ctx *ctx, const uint64_t *d_keys, uint64_t count, uint64_t *d_out,
                      uint64_t *out_count, void *stream);

/* Sorts d_pairs[0..count) in place, ascending on (remote << 32 | rep) - the
 * reference's boundary edge order (src/boundary_sort.c:5-8,93-98) - where
 * each pair is {uint32 rep, uint32 remote}.  max_rep / max_remote bound the
 * values (UINT32_MAX if unknown) so that only the needed digits are sorted. */
int ccgpu_boundary_sort(ccgpu_ctx *ctx, uint32_t *d_pairs, uint64_t count, uint32_t max_rep,
                        uint32_t max_remote, void *stream);
/* Removes adjacent duplicates of a sorted pair array in place
 * (src/boundary_sort.c:100-119); *new_count receives the kept count. */
int ccgpu_boundary_dedup(ccgpu_ctx *ctx, uint32_t *d_pairs, uint64_t count, uint64_t *new_count,
                         void *stream);

/* Plans: the whole local-CC launch sequence for fixed arguments captured
 * once into a CUDA graph and replayed with one cudaGraphLaunch.  The plan
 * owns a private context (its scratch), so it stays valid whatever else the
 * caller runs; its arguments (pointers, sizes, options) are fixed at
 * creation.  ccgpu_plan_kernels() is the number of kernels one launch runs. */
typedef struct ccgpu_plan ccgpu_plan;
int ccgpu_local_cc_plan(const uint64_t *d_row_ptr, const uint32_t *d_col_idx, uint32_t n,
                        uint64_t m, uint32_t *d_labels, const ccgpu_cc_opts *opts,
                        ccgpu_plan **out);
int ccgpu_plan_launch(ccgpu_plan *plan, void *stream);
int ccgpu_plan_kernels(const ccgpu_plan *plan);
void ccgpu_plan_destroy(ccgpu_plan *plan);

/* ccgpu_local_cc without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory
 * (processes whose allocator reserved all of HBM up front; plug-ins that
 * must not own device memory; loops that must not take the device-wide
 * synchronisation of cudaMalloc/cudaFree).  Scratch lives in a fixed file-scope device array of
 * ccgpu_local_cc_noalloc_capacity() bytes (1 MiB), held by every GPU that
 * loads the library until the process exits; a solve needs
 * ccgpu_local_cc_noalloc_required(n, m, opts) bytes (about 4 bytes per
 * m/heavy_degree row of the heavy queue) and larger graphs are rejected
 * with CCGPU_ERR_LIMIT; _required returns SIZE_MAX for invalid options.
 * The first call on a device looks up the array with cudaGetSymbolAddress
 * and keeps the address; make it before any stream capture, and do not use
 * the call after cudaDeviceReset in the same process.  Calls share the
 * array: calls whose kernels overlap on the GPU race.  Asynchronous on
 * `stream`; no stats. */
int ccgpu_local_cc_noalloc(const uint64_t *d_row_ptr, const uint32_t *d_col_idx, uint32_t n,
                           uint64_t m, uint32_t *d_labels, const ccgpu_cc_opts *opts,
                           void *stream);
size_t ccgpu_local_cc_noalloc_capacity(void);
size_t ccgpu_local_cc_noalloc_required(uint32_t n, uint64_t m, const ccgpu_cc_opts *opts);

/* ------------------------------------------------------------------------
 * Batched CC: many independent graphs in one solve.  No counterpart in the
 * reference, which solves one graph per call
 * (compute_connected_components_pthreads, include/cc.h:27-28); every graph
 * of a batch gets exactly that call's labels (minimum local vertex id of
 * each component of its own graph).
 *
 * Packed CSR-of-CSRs, G graphs:
 *   h_vtx_off[G+1], h_edge_off[G+1]  host prefix sums of n_g and m_g
 *   d_row_ptr  graph g's n_g + 1 local row pointers (0 .. m_g) at
 *              d_row_ptr[vtx_off[g] + g]
 *   d_col      graph g's local neighbour ids at d_col[edge_off[g]]
 *   d_labels   out: graph g's labels at d_labels[vtx_off[g]]
 * Graphs are grouped into CCGPU_BATCH_CLASSES degree classes by mean row
 * length (m_g / n_g against class_bounds); each class has its own schedule
 * (sampled neighbours, shortcut cadence, tile size, warp-row threshold),
 * tile list and stream, so classes run concurrently.  A plan's launch
 * replays the whole batch as one CUDA graph (captured on the first launch).
 * ---------------------------------------------------------------------- */
#define CCGPU_BATCH_CLASSES 3

typedef struct {
    uint32_t graphs;
    const uint64_t *h_vtx_off;
    const uint64_t *h_edge_off;
    const uint64_t *d_row_ptr;
    const uint32_t *d_col;
    uint32_t *d_labels;
} ccgpu_batch;

typedef struct {
    int sample_rounds; /* neighbours linked per vertex before the giant skip (0..4) */
    int cadence;       /* 1: shortcut pass after every sampled neighbour            */
    int tile;          /* vertices per tile, power of two in 256..2^20              */
    int warp_degree;   /* rows with at least this many entries get a whole warp     */
} ccgpu_batch_class_opts;

typedef struct {
    float class_bounds[CCGPU_BATCH_CLASSES - 1]; /* mean-row-length cut points (6, 16) */
    int heavy_degree;                            /* rows above it are queued (8192)    */
    ccgpu_batch_class_opts cls[CCGPU_BATCH_CLASSES];
    int persistent;   /* 1: each class is one persistent launch that moves every
                       * graph through init, sampling, shortcuts, giant, finish and
                       * final by per-graph phase counters (0: one launch per
                       * phase)                                                  */
    int wait_ms;      /* persistent: limit of one wait on a graph's previous phase
                       * (0 = 2000); a wait that runs out ends the launch and the
                       * results call returns CCGPU_ERR_TIMEOUT                   */
    int stall_graph;  /* test aid, -1 = off: graph whose first wait can never be
                       * met, to exercise the bounded wait                        */
} ccgpu_batch_tuning;

void ccgpu_batch_tuning_default(ccgpu_batch_tuning *t);

typedef struct ccgpu_batch_plan ccgpu_batch_plan;
/* Validates the offsets, builds the classes' tile lists and scratch (owned
 * by the plan).  tuning NULL = defaults. */
int ccgpu_batch_plan_create(ccgpu_ctx *ctx, const ccgpu_batch *b, const ccgpu_batch_tuning *tuning,
                            ccgpu_batch_plan **out);
/* Enqueues the solve kernel by kernel on `stream` (asynchronous). */
int ccgpu_batch_plan_run(ccgpu_batch_plan *p, void *stream);
/* Enqueues the solve as one CUDA graph launch on `stream` (asynchronous). */
int ccgpu_batch_plan_launch(ccgpu_batch_plan *p, void *stream);
/* Kernels one graph launch runs (0 before the first launch). */
int ccgpu_batch_plan_kernels(const ccgpu_batch_plan *p);
/* Times candidate schedules per class on the device (coordinate descent over
 * sample_rounds, cadence, tile, warp_degree) and keeps the fastest; the
 * chosen tuning is written to *chosen (may be NULL).  Synchronous. */
int ccgpu_batch_plan_autotune(ccgpu_batch_plan *p, void *stream, ccgpu_batch_tuning *chosen);
int ccgpu_batch_plan_tuning(const ccgpu_batch_plan *p, ccgpu_batch_tuning *out);
/* Graphs per class (array of CCGPU_BATCH_CLASSES). */
int ccgpu_batch_plan_class_graphs(const ccgpu_batch_plan *p, uint32_t *counts);
/* Per-graph component counts and done flags of the last solve (host arrays
 * of G entries, either may be NULL).  Synchronous on `stream`.
 * CCGPU_ERR_TIMEOUT when a persistent launch gave up a wait (graphs whose
 * done flag is 0 were not solved). */
int ccgpu_batch_plan_results(ccgpu_batch_plan *p, uint32_t *h_components, uint32_t *h_done,
                             void *stream);
void ccgpu_batch_plan_destroy(ccgpu_batch_plan *p);
/* One-shot: plan, solve, per-graph component counts (may be NULL).  The
 * context keeps the plan (and its device arrays, which only grow) for its
 * next call, and frees it in ccgpu_ctx_destroy; a context serves one host
 * thread at a time.  Synchronous on `stream`. */
int ccgpu_batch_cc(ccgpu_ctx *ctx, const ccgpu_batch *b, const ccgpu_batch_tuning *tuning,
                   uint32_t *h_components, void *stream);

/* ------------------------------------------------------------------------
 * Served CC: a request server with continuous batching.  No counterpart in
 * the reference; each request's labels are those of
 * compute_connected_components_pthreads on its graph alone.
 *
 * A worker thread admits submitted requests, oldest first, while a slot
 * (max_graphs) is free and the request's CSR and labels fit in the server's
 * HBM pool (hbm_bytes; 0 = half of the free device memory at creation).
 * Whenever one of `streams` batch slots is idle, up to max_batch admitted
 * requests become one batched solve on that slot's stream, so batches that
 * form while others run overlap them on the device.  CSRs and labels stay in
 * HBM from admission to completion.  Host buffers passed to submit must
 * stay valid until its wait returns; pinned buffers let the copies run
 * asynchronously.  Times are seconds on the server's clock.
 * ---------------------------------------------------------------------- */
typedef struct {
    size_t hbm_bytes;    /* pool for request data; 0 = half the free HBM  */
    uint32_t max_graphs; /* requests resident in HBM at once (8192)       */
    uint32_t max_batch;  /* requests per batched solve (4096)             */
    int streams;         /* batches in flight at once, 1..8 (2)           */
} ccgpu_server_opts;

typedef struct {
    double t_submit, t_admit, t_start, t_done;
    uint32_t components;   /* components of the request's graph          */
    uint32_t batch_graphs; /* requests in the batch it was solved in     */
    int status;
} ccgpu_request_info;

typedef struct {
    uint64_t submitted, completed, batches;
    uint32_t in_flight, max_in_flight, max_batch_seen, pending, resident;
    size_t pool_bytes, pool_used, pool_peak;
} ccgpu_server_stats;

typedef struct ccgpu_server ccgpu_server;
void ccgpu_server_opts_default(ccgpu_server_opts *o);
/* Creates the pool, the batch slots and the worker thread on the current
 * device.  tuning NULL = the batched solver's defaults. */
int ccgpu_server_create(const ccgpu_server_opts *opts, const ccgpu_batch_tuning *tuning,
                        ccgpu_server **out);
/* Queues one symmetric CSR (host arrays); h_labels (n entries) receives the
 * labels.  CCGPU_ERR_LIMIT if the graph can never fit in the pool. */
int ccgpu_server_submit(ccgpu_server *s, const uint64_t *h_row_ptr, const uint32_t *h_col_idx,
                        uint32_t n, uint64_t m, uint32_t *h_labels, uint64_t *ticket);
/* Waits for a request (timeout_s < 0: no limit), copies its labels from
 * HBM into the buffer given at submission, returns its blocks to the pool
 * and releases the ticket (t_done = labels in that buffer).  One wait per
 * ticket at a time; CCGPU_ERR_TIMEOUT leaves the ticket valid.  A solved
 * request keeps its pool blocks until it is waited for. */
int ccgpu_server_wait(ccgpu_server *s, uint64_t ticket, double timeout_s,
                      ccgpu_request_info *info);
int ccgpu_server_stats_get(ccgpu_server *s, ccgpu_server_stats *out);
double ccgpu_server_now(ccgpu_server *s);
/* Lets the batches in flight finish, drops requests not yet in a batch,
 * stops the worker and frees the pool (labels not yet waited for are lost). */
void ccgpu_server_destroy(ccgpu_server *s);

/* Number of v with d_labels[v] == v (one root per component when the labels
 * are min-id labels).  Synchronous; result in *count. */
int ccgpu_count_roots(ccgpu_ctx *ctx, const uint32_t *d_labels, uint32_t n,
                      uint64_t *count, void *stream);

/* Checks, on the device, the invariants a min-id labelling satisfies:
 * labels[u] == labels[v] for every edge, labels[v] <= v, and
 * labels[labels[v]] == labels[v].  *violations counts failing vertices/edges.
 * (With an independent component count this pins the labelling exactly.) */
int ccgpu_check_labels(ccgpu_ctx *ctx, const uint64_t *d_row_ptr, const uint32_t *d_col_idx,
                       uint32_t n, uint64_t m, const uint32_t *d_labels,
                       uint64_t *violations, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CCGPU_H */
