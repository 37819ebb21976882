/*
 * Internal helpers shared by the CUDA translation units: status/error
 * plumbing, the per-context scratch arena, launch geometry and the
 * union-find device primitives every solver uses.
 */
#ifndef CCGPU_INTERNAL_H
#define CCGPU_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "ccgpu.h"

/* ---------------------------------------------------------------- errors */

int ccgpu_set_error(int status, const char *fmt, ...);
int ccgpu_cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define CC_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess)                                                 \
            return ccgpu_cuda_fail(e_, #call, __FILE__, __LINE__);             \
    } while (0)

#define CC_TRY(call)                                                           \
    do {                                                                       \
        int s_ = (call);                                                       \
        if (s_ != CCGPU_OK)                                                    \
            return s_;                                                         \
    } while (0)

#define CC_LAUNCH_CHECK() CC_CUDA(cudaGetLastError())

/* ----------------------------------------------------------------- arena */

/* A context's scratch: one grow-only device block carved into aligned
 * pieces per call.  Growing frees and reallocates (a device-wide sync). */
struct ccgpu_ctx {
    int device;
    void *base;
    size_t cap;
    size_t used;      /* bump pointer of the current call */
    void *host_pinned; /* small pinned staging for stats read-back */
    size_t host_cap;
    int sm_count;
    int owned_by_default;
    unsigned long long *cell; /* 256-byte device cell for small reductions */
    unsigned long long launches; /* kernels this context has launched */
    struct cc_prof *prof;        /* per-kernel event timing, NULL = off */
    struct ccgpu_batch_plan *batch_cache; /* the plan ccgpu_batch_cc reuses */
};

/* Frees the context's cached batch plan (batch_cc.cu). */
void cc_batch_cache_free(ccgpu_ctx *ctx);

/* Kernel ids for the launch profiler (names in runtime.cu). */
enum {
    CCK_INIT = 0,
    CCK_SAMPLE,
    CCK_COMPRESS,
    CCK_GIANT,
    CCK_LINK_ROWS,
    CCK_LINK_HEAVY,
    CCK_FINAL_COMPRESS,
    CCK_COUNT_ROOTS,
    CCK_CHECK,
    CCK_DIST_SPLIT,
    CCK_DIST_FILL,
    CCK_DIST_REPS,
    CCK_DIST_PAIRS,
    CCK_SORT_HIST,
    CCK_SORT_SCAN,
    CCK_SORT_SCATTER,
    CCK_DIST_DEDUP,
    CCK_DIST_GHOSTS,
    CCK_DIST_PLAN,
    CCK_MERGE_INIT,
    CCK_MERGE_HOOK,
    CCK_MERGE_UPD,
    CCK_MERGE_EXCH_PACK,
    CCK_MERGE_EXCH_SCATTER,
    CCK_DIST_LABELS,
    CCK_DIST_BOUNDS,
    CCK_SCAN,
    CCK_BATCH,
    CCK_MISC,
    CCK_DIST_PAIRS_HEAVY,
    CCK_DIST_PAIRS_BITMAP,
    CCK_BATCH_INIT,
    CCK_BATCH_SAMPLE,
    CCK_BATCH_COMPRESS,
    CCK_BATCH_GIANT,
    CCK_BATCH_LINK,
    CCK_BATCH_HEAVY,
    CCK_BATCH_FINAL,
    CCK_DIST_LOCAL_COUNT,
    CCK_DIST_LOCAL_FILL,
    CCK_DIST_TILES,
    CCK_DIST_GFLAG,
    CCK_DIST_MERGE_KEYS,
    CCK_MERGE_EXCH_PULL,
    CCK_DIST_PAIRS_LOCAL,
    CCK_NUM
};

/* Records events around a launch when the context's profiler is on. */
void cc_prof_mark(ccgpu_ctx *ctx, int kid, int end, cudaStream_t st);

#define CC_KLAUNCH(ctx, kid, kernel, grid, block, smem, st, ...)               \
    do {                                                                       \
        if ((ctx)->prof)                                                       \
            cc_prof_mark((ctx), (kid), 0, (st));                               \
        kernel<<<(grid), (block), (smem), (st)>>>(__VA_ARGS__);                \
        CC_LAUNCH_CHECK();                                                     \
        (ctx)->launches++;                                                     \
        if ((ctx)->prof)                                                       \
            cc_prof_mark((ctx), (kid), 1, (st));                               \
    } while (0)

/* Layout helper: first pass (base == NULL) sums sizes, second pass hands
 * out pointers.  Pieces are 256-byte aligned. */
typedef struct {
    char *base;
    size_t off;
} cc_carve;

static inline void *cc_take(cc_carve *c, size_t bytes)
{
    size_t off = (c->off + 255) & ~(size_t)255;
    c->off = off + bytes;
    return c->base ? (void *)(c->base + off) : NULL;
}

int ccgpu_ctx_resolve(ccgpu_ctx **ctx);
/* Ensures the context holds at least `bytes` of scratch; returns its base. */
int ccgpu_ctx_reserve(ccgpu_ctx *ctx, size_t bytes, void **base);
int ccgpu_ctx_pinned(ccgpu_ctx *ctx, size_t bytes, void **host);
/* The context's 256-byte device cell (allocated on first use). */
int ccgpu_ctx_cell(ccgpu_ctx *ctx, unsigned long long **cell);

/* ------------------------------------------------------------ geometry */

static inline unsigned cc_blocks(uint64_t work, unsigned per_block, unsigned cap)
{
    uint64_t b = (work + per_block - 1) / per_block;
    if (b == 0)
        b = 1;
    if (b > cap)
        b = cap;
    return (unsigned)b;
}

/* ----------------------------------------------- union-find primitives */
#ifdef __CUDACC__

/* Parent reads are weak loads cached in L1 (ld.global.ca).  L1 is not
 * coherent across SMs, so a read may return an older value of parent[i];
 * that is harmless here: every value parent[i] ever held is an ancestor of
 * i with parent[i] <= i, so walks still end, and a stale "root" only makes a
 * hook CAS fail and retry from the fresher value the CAS returns.  Caching
 * matters because every find ends on the few lines near the giant root:
 * served from L2 they turn one L2 slice into a hot spot.  The asm is
 * volatile so the compiler cannot merge or hoist the reads. */
#ifndef CC_PARENT_LOAD_L2
#define CC_PARENT_LOAD_L2 0
#endif
#ifndef CC_FIND_HALVING
#define CC_FIND_HALVING 1
#endif
__device__ __forceinline__ uint32_t cc_ldp(const uint32_t *p, uint32_t i)
{
    uint32_t v;
#if CC_PARENT_LOAD_L2
    asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p + i));
#else
    asm volatile("ld.global.ca.u32 %0, [%1];" : "=r"(v) : "l"(p + i));
#endif
    return v;
}

/* Root of x with path halving.  Invariant parent[x] <= x, so the walk is
 * strictly decreasing and ends.  Halving writes only touch non-roots and
 * always store an ancestor, so they never break a concurrent hook.  They
 * are atomicMin (a fire-and-forget red.min): ancestors have smaller ids
 * than their descendants, so a pointer only ever moves towards the root.
 * A plain store here would let a slow thread put an intermediate ancestor
 * back over the root pointer another thread just wrote in the final
 * shortcut pass, leaving a label that is not the component minimum. */
__device__ __forceinline__ uint32_t cc_find(uint32_t *parent, uint32_t x)
{
    uint32_t p = cc_ldp(parent, x);
    while (p != x) {
        uint32_t gp = cc_ldp(parent, p);
        if (gp == p)
            return p;
        if (CC_FIND_HALVING)
            atomicMin(parent + x, gp);
        x = gp;
        p = cc_ldp(parent, x);
    }
    return x;
}

/* Root of x without writes (for read-only passes). */
__device__ __forceinline__ uint32_t cc_find_ro(const uint32_t *parent, uint32_t x)
{
    uint32_t p = cc_ldp(parent, x);
    while (p != x) {
        x = p;
        p = cc_ldp(parent, x);
    }
    return x;
}

/* Union of the trees of a and b: the larger root is hooked under the
 * smaller with a CAS that only succeeds while it is still a root.  A failed
 * CAS means another thread hooked it first; the retry starts from roots
 * strictly below the failed one, so the loop ends. */
__device__ __forceinline__ void cc_link_roots(uint32_t *parent, uint32_t ra, uint32_t rb)
{
    while (ra != rb) {
        uint32_t hi = ra > rb ? ra : rb;
        uint32_t lo = ra ^ rb ^ hi;
        uint32_t old = atomicCAS(parent + hi, hi, lo);
        if (old == hi)
            return;
        ra = cc_find(parent, old);
        rb = cc_find(parent, lo);
    }
}

__device__ __forceinline__ void cc_link(uint32_t *parent, uint32_t a, uint32_t b)
{
    cc_link_roots(parent, cc_find(parent, a), cc_find(parent, b));
}

/* Union of the trees of a and b that skips walking b's path when b is
 * smaller than a's root: the root ra is then hooked directly under b.  That
 * is safe because a root is the minimum of its tree, so b < ra means b lies
 * in another tree and no cycle can form.  It trades a longer path later
 * (ra hangs under b, not under b's root) for one walk fewer now. */
__device__ __forceinline__ void cc_link_lazy(uint32_t *parent, uint32_t a, uint32_t b)
{
    uint32_t ra = cc_find(parent, a);
    while (b < ra) {
        uint32_t old = atomicCAS(parent + ra, ra, b);
        if (old == ra)
            return;
        ra = cc_find(parent, old);
    }
    cc_link_roots(parent, ra, cc_find(parent, b));
}

template <bool LAZY>
__device__ __forceinline__ void cc_union(uint32_t *parent, uint32_t a, uint32_t b)
{
    if (LAZY)
        cc_link_lazy(parent, a, b);
    else
        cc_link(parent, a, b);
}

__device__ __forceinline__ uint32_t cc_warp_min(uint32_t v)
{
    return __reduce_min_sync(0xffffffffu, v);
}

/* Spreads the rows of a heavy-row list over every warp of the grid in
 * pieces of `chunk` entries: rows are taken 256 at a time, the block scans
 * their piece counts in shared memory, and piece g of the batch goes to
 * warp g mod (all warps).  fn(v, jb, je) is called by all 32 lanes of a
 * warp together.  Rows are [row_ptr[v] + skip, row_ptr[v+1]) clamped to m,
 * or [row_ptr[v] + skip, row_end[v]) when row_end is given.  Must be called
 * by every thread of a 256-thread block. */
template <typename Fn>
__device__ __forceinline__ void cc_for_heavy_pieces(const uint32_t *list, uint32_t count,
                                                    const uint64_t *row_ptr,
                                                    const uint64_t *row_end, uint64_t m,
                                                    uint32_t skip, uint64_t chunk, Fn fn)
{
    __shared__ uint64_t s_pre[257];
    __shared__ uint64_t s_beg[256], s_end[256];
    __shared__ uint32_t s_v[256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t gwarp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp;
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint32_t b0 = 0; b0 < count; b0 += 256) {
        const uint32_t h = b0 + threadIdx.x;
        uint64_t pieces = 0;
        if (h < count) {
            uint32_t v = list[h];
            uint64_t e = row_end ? row_end[v] : row_ptr[v + 1], b = row_ptr[v];
            if (e > m)
                e = m;
            if (b > e)
                b = e;
            b = b + skip < e ? b + skip : e;
            s_v[threadIdx.x] = v;
            s_beg[threadIdx.x] = b;
            s_end[threadIdx.x] = e;
            pieces = (e - b + chunk - 1) / chunk;
        }
        /* block-wide exclusive scan of the piece counts (256 threads) */
        uint64_t incl = pieces;
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += y;
        }
        __shared__ uint64_t s_w[8];
        if (lane == 31)
            s_w[warp] = incl;
        __syncthreads();
        uint64_t pre = 0, total = 0;
        for (int w = 0; w < 8; ++w) {
            pre += (w < warp) ? s_w[w] : 0ull;
            total += s_w[w];
        }
        s_pre[threadIdx.x] = pre + incl - pieces;
        if (threadIdx.x == 0)
            s_pre[256] = total;
        __syncthreads();
        const int rows = count - b0 < 256u ? (int)(count - b0) : 256;
        for (uint64_t g = gwarp; g < total; g += nwarps) {
            int lo = 0, hi = rows; /* last row whose first piece is <= g */
            while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (s_pre[mid] <= g)
                    lo = mid;
                else
                    hi = mid;
            }
            uint64_t jb = s_beg[lo] + (g - s_pre[lo]) * chunk;
            uint64_t je = jb + chunk < s_end[lo] ? jb + chunk : s_end[lo];
            fn(s_v[lo], jb, je);
        }
        __syncthreads();
    }
    (void)lane;
}

/* MurmurHash3 fmix32 finaliser (Appleby, public domain) as a sample mixer. */
__device__ __forceinline__ uint32_t cc_mix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

/* Most frequent value among the 1024 values of a 1024-thread block (one per
 * thread, `val`); ties go to the smaller value, so the choice is
 * deterministic.  Bitonic sort in shared memory, run lengths by binary
 * search, then a max-reduction of (count, ~value).  Every thread must call
 * it; all of them get the result. */
__device__ __forceinline__ uint32_t cc_block_mode1024(uint32_t val, uint32_t *s,
                                                      unsigned long long *s_best)
{
    const uint32_t i = threadIdx.x;
    s[i] = val;
    __syncthreads();
    for (uint32_t k = 2; k <= 1024; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            uint32_t ij = i ^ j;
            if (ij > i) {
                uint32_t a = s[i], b = s[ij];
                bool up = (i & k) == 0;
                if ((a > b) == up) {
                    s[i] = b;
                    s[ij] = a;
                }
            }
            __syncthreads();
        }
    }
    uint32_t cnt = 0;
    val = s[i];
    if (i == 0 || s[i - 1] != val) {
        uint32_t a = i, b = 1024;
        while (a < b) {
            uint32_t mid = (a + b) >> 1;
            if (s[mid] <= val)
                a = mid + 1;
            else
                b = mid;
        }
        cnt = a - i;
    }
    unsigned long long key = ((unsigned long long)cnt << 32) | (uint32_t)~val;
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if ((i & 31) == 0)
        s_best[i >> 5] = key;
    __syncthreads();
    key = s_best[i & 31];
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    __syncthreads();
    return ~(uint32_t)key;
}

/* Warp-cooperative link of v with up to K entries per lane (all 32 lanes
 * call it).  Hooking every entry's root under v's root one by one piles the
 * CAS attempts of the whole row onto v's root (a herd: one wins per round,
 * the rest retry).  Instead the warp first hooks v's tree under the
 * smallest root among its entries; v's root is then no larger than any
 * entry's root, so the remaining hooks go to each entry's own root. */
template <int K>
__device__ __forceinline__ void cc_warp_link_min_first(uint32_t *parent, uint32_t v,
                                                       const uint32_t *u, const bool *ok,
                                                       int lane)
{
    uint32_t r[K];
    uint32_t mn = 0xffffffffu;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        r[i] = ok[i] ? cc_find(parent, u[i]) : 0xffffffffu;
        mn = r[i] < mn ? r[i] : mn;
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    if (mn == 0xffffffffu)
        return;
    if (lane == 0) {
        uint32_t rv = cc_find(parent, v);
        if (rv != mn)
            cc_link_roots(parent, rv, mn);
    }
    __syncwarp();
    uint32_t rv = cc_find(parent, v);
#pragma unroll
    for (int i = 0; i < K; ++i)
        if (ok[i] && r[i] != rv)
            cc_link_roots(parent, r[i], rv);
}

/* Generalisation of cc_for_heavy_pieces to rows whose bounds come from a
 * functor: bounds(h, &beg, &end) gives the entry range of list item h,
 * fn(h, jb, je) is called by all 32 lanes of a warp for each piece.  Piece g
 * of a batch of 256 items goes to warp g mod (all warps).  Must be called
 * by every thread of a 256-thread block. */
template <typename Bounds, typename Fn>
__device__ __forceinline__ void cc_for_pieces(uint32_t count, uint64_t chunk, Bounds bounds,
                                              Fn fn)
{
    __shared__ uint64_t s_pre[257];
    __shared__ uint64_t s_beg[256], s_end[256];
    __shared__ uint64_t s_w[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t gwarp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp;
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint32_t b0 = 0; b0 < count; b0 += 256) {
        const uint32_t h = b0 + threadIdx.x;
        uint64_t pieces = 0;
        if (h < count) {
            uint64_t b = 0, e = 0;
            bounds(h, b, e);
            s_beg[threadIdx.x] = b;
            s_end[threadIdx.x] = e;
            pieces = (e - b + chunk - 1) / chunk;
        }
        uint64_t incl = pieces;
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += y;
        }
        if (lane == 31)
            s_w[warp] = incl;
        __syncthreads();
        uint64_t pre = 0, total = 0;
        for (int w = 0; w < 8; ++w) {
            pre += (w < warp) ? s_w[w] : 0ull;
            total += s_w[w];
        }
        s_pre[threadIdx.x] = pre + incl - pieces;
        if (threadIdx.x == 0)
            s_pre[256] = total;
        __syncthreads();
        const int rows = count - b0 < 256u ? (int)(count - b0) : 256;
        for (uint64_t g = gwarp; g < total; g += nwarps) {
            int lo = 0, hi = rows;
            while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (s_pre[mid] <= g)
                    lo = mid;
                else
                    hi = mid;
            }
            uint64_t jb = s_beg[lo] + (g - s_pre[lo]) * chunk;
            uint64_t je = jb + chunk < s_end[lo] ? jb + chunk : s_end[lo];
            fn(b0 + (uint32_t)lo, jb, je);
        }
        __syncthreads();
    }
    (void)lane;
}

#endif /* __CUDACC__ */

#endif /* CCGPU_INTERNAL_H */
