/*
 * Batched connected components: many independent graphs solved by one
 * sequence of grid-wide kernels, replayed as one CUDA graph.
 *
 * The reference solves one graph per call (src/cc_pthreads.c:152-229); a
 * batch keeps that result for every graph - labels[v] is the minimum local
 * vertex id of v's component in its own graph - and removes the per-graph
 * launch and synchronisation cost that dominates small graphs.
 *
 * Layout (packed CSR-of-CSRs in HBM):
 *   vtx_off[G+1], edge_off[G+1]  prefix sums of vertex and entry counts
 *   row_ptr   graph g's n_g + 1 local row pointers at row_ptr[vtx_off[g] + g]
 *   col       graph g's local (int32) neighbour ids at col[edge_off[g]]
 *   labels    graph g's labels at labels[vtx_off[g]]
 *
 * Work is cut into tiles - up to `tile` consecutive vertices of one graph -
 * so a CTA reads its graph's bases once per tile and then runs exactly the
 * single-graph union-find (roots hooked larger-id under smaller-id) on the
 * graph's own slice of the label array in local ids.  Graphs are grouped
 * into degree classes by their mean row length; each class has its own
 * tile size, sampled neighbours, shortcut cadence and warp-row threshold
 * (the autotuner picks them), its own tile list and counters, and its own
 * branch of the CUDA graph, so classes run concurrently.
 *
 * Per class, one solve is:
 *   kb_init      parent[v] = v
 *   kb_sample    r = 0..k-1: link v with its r-th neighbour (atomicMin on
 *                the larger root: the forest stays valid; anything lost is
 *                relinked by the finish pass), kb_compress after each round
 *                when the cadence is on, and always before kb_giant
 *   kb_giant     one CTA per graph: most frequent root of 1024 samples
 *   kb_link      finish pass over the rows of vertices outside their graph's
 *                giant tree: short rows gathered per CTA and walked
 *                edge-parallel, rows of >= warp_degree entries by a warp,
 *                rows above heavy_degree queued
 *   kb_heavy     queued rows in 512-entry pieces over every warp
 *   kb_final     labels[v] = root(v); per-graph root count, and the graph's
 *                done flag set by its last tile
 */
#include <cstdio>
#include <cstring>
#include <vector>

#include "batch_core.h"

namespace {

constexpr int kB = 256;
constexpr int kWarpsB = kB / 32;
constexpr uint64_t kPiece = 512;
constexpr uint32_t kNone = 0xffffffffu;

struct BatchK {
    const BGraph *gr;         /* [G] graph descriptors           */
    const uint64_t *row_ptr;
    const uint32_t *col;
    uint32_t *labels;
    const uint32_t *tile_g;   /* [tiles] graph of each tile      */
    const uint32_t *tile_v0;  /* [tiles] first local vertex      */
    uint32_t tiles;
    uint32_t tile;            /* vertices per tile               */
    const uint32_t *graphs;   /* [ngraphs] graphs of this class  */
    uint32_t ngraphs;
    uint32_t *giants;         /* [G] giant root (local id)       */
    uint32_t *comps;          /* [G] components                  */
    uint32_t *tiles_done;     /* [G] finished tiles of kb_final  */
    uint32_t *done;           /* [G] 1 once the graph is solved  */
    unsigned long long *grab; /* tile counter of kb_link         */
    uint32_t *heavy_count;
    uint64_t *heavy_list;     /* (g << 32) | v                   */
    uint32_t heavy_cap;
    uint32_t heavy_deg;
    uint32_t warp_deg;
    int skip;                 /* finish pass skips giant trees   */
    uint32_t *stash;          /* second neighbours (like labels), NULL = off */
};

struct Tile {
    uint32_t g, v0, v1, n;
    uint64_t m;
    const uint64_t *rp;
    uint32_t *parent;
    const uint32_t *col;
};

__device__ __forceinline__ Tile tile_of(const BatchK &K, uint32_t t)
{
    Tile T;
    T.g = __ldg(K.tile_g + t);
    T.v0 = __ldg(K.tile_v0 + t);
    const BGraph *d = K.gr + T.g;
    T.n = __ldg(&d->n);
    T.v1 = T.v0 + K.tile < T.n ? T.v0 + K.tile : T.n;
    T.m = __ldg(&d->m);
    T.rp = K.row_ptr + __ldg(&d->rp);
    T.parent = K.labels + __ldg(&d->lab);
    T.col = K.col + __ldg(&d->col);
    return T;
}

__device__ __forceinline__ void row_bounds(const Tile &T, uint32_t v, uint64_t &b, uint64_t &e)
{
    b = __ldg(T.rp + v);
    e = __ldg(T.rp + v + 1);
    if (e > T.m)
        e = T.m;
    if (b > e)
        b = e;
}

__device__ __forceinline__ void tile_init(const Tile &T)
{
    for (uint32_t v = T.v0 + threadIdx.x; v < T.v1; v += kB)
        T.parent[v] = v;
}

/* Links row entry r of every vertex of the tile (MINHOOK sampling). */
__device__ __forceinline__ void tile_sample(const BatchK &K, const Tile &T, int r)
{
    uint32_t *stash = K.stash ? K.stash + (T.parent - K.labels) : nullptr;
    for (uint32_t v = T.v0 + threadIdx.x; v < T.v1; v += kB) {
        uint32_t u;
        if (stash && r == 1) {
            u = stash[v]; /* written by round 0 */
        } else {
            uint64_t b, e;
            row_bounds(T, v, b, e);
            u = b + (uint64_t)r < e ? __ldg(T.col + b + r) : 0xffffffffu;
            if (stash && r == 0)
                stash[v] = b + 1 < e ? __ldg(T.col + b + 1) : 0xffffffffu;
        }
        if (u >= T.n)
            continue;
        const uint32_t rv = cc_find(T.parent, v), ru = cc_find(T.parent, u);
        if (rv != ru)
            atomicMin(T.parent + (rv > ru ? rv : ru), rv < ru ? rv : ru);
    }
}

__device__ __forceinline__ void tile_compress(const Tile &T)
{
    for (uint32_t v = T.v0 + threadIdx.x; v < T.v1; v += kB) {
        const uint32_t r = cc_find(T.parent, v);
        if (r != v)
            T.parent[v] = r;
    }
}

__global__ void __launch_bounds__(kB) kb_init(BatchK K)
{
    for (uint32_t t = blockIdx.x; t < K.tiles; t += gridDim.x)
        tile_init(tile_of(K, t));
}

__global__ void __launch_bounds__(kB) kb_sample(BatchK K, int r)
{
    for (uint32_t t = blockIdx.x; t < K.tiles; t += gridDim.x)
        tile_sample(K, tile_of(K, t), r);
}

__global__ void __launch_bounds__(kB) kb_compress(BatchK K)
{
    for (uint32_t t = blockIdx.x; t < K.tiles; t += gridDim.x)
        tile_compress(tile_of(K, t));
}

/* One CTA per graph of the class: most frequent root of 1024 samples. */
__global__ void __launch_bounds__(1024) kb_giant(BatchK K, uint32_t seed)
{
    __shared__ uint32_t s[1024];
    __shared__ unsigned long long s_best[32];
    for (uint32_t i = blockIdx.x; i < K.ngraphs; i += gridDim.x) {
        const uint32_t g = __ldg(K.graphs + i);
        const uint32_t n = __ldg(&K.gr[g].n);
        if (n == 0) {
            if (threadIdx.x == 0)
                K.giants[g] = kNone;
            continue;
        }
        const uint32_t h = cc_mix32(threadIdx.x * 0x9e3779b9u + seed + g);
        const uint32_t v = (uint32_t)(((uint64_t)h * n) >> 32);
        const uint32_t mode = cc_block_mode1024(cc_find_ro(K.labels + __ldg(&K.gr[g].lab), v), s, s_best);
        if (threadIdx.x == 0)
            K.giants[g] = mode;
    }
}

/* A warp links v with entries [b, e) of its graph: 16-byte column loads on
 * the aligned body when the graph's columns are 16-byte aligned. */
__device__ __forceinline__ void warp_row(const Tile &T, uint32_t v, uint64_t b, uint64_t e,
                                         int lane)
{
    uint64_t a = b, body_end = b; /* unaligned columns: every entry scalar */
    if ((((uintptr_t)T.col) & 15) == 0) {
        a = (b + 3) & ~3ull;
        if (a > e)
            a = e;
        body_end = e & ~3ull;
        if (body_end < a)
            body_end = a;
    }
    const uint64_t head = a - b, scalars = head + (e - body_end);
    for (uint64_t s0 = 0; s0 < scalars; s0 += 32) {
        const uint64_t s = s0 + lane;
        uint32_t u[1] = {0};
        bool ok[1] = {false};
        if (s < scalars) {
            u[0] = __ldg(T.col + (s < head ? b + s : body_end + (s - head)));
            ok[0] = u[0] < T.n;
        }
        cc_warp_link_min_first<1>(T.parent, v, u, ok, lane);
    }
    const uint4 *c4 = reinterpret_cast<const uint4 *>(T.col);
    for (uint64_t q0 = a / 4; q0 < body_end / 4; q0 += 32) {
        const uint64_t q = q0 + lane;
        uint32_t u[4] = {0, 0, 0, 0};
        bool ok[4] = {false, false, false, false};
        if (q < body_end / 4) {
            const uint4 x = __ldg(c4 + q);
            u[0] = x.x;
            u[1] = x.y;
            u[2] = x.z;
            u[3] = x.w;
#pragma unroll
            for (int i = 0; i < 4; ++i)
                ok[i] = u[i] < T.n;
        }
        cc_warp_link_min_first<4>(T.parent, v, u, ok, lane);
    }
}

/* Vertices a thread takes per step of the finish pass (consecutive), so
 * the step's barriers are paid once per kVPT vertices per thread. */
constexpr int kVPT = 4;
constexpr int kStep = kB * kVPT;

/* Shared memory of one tile of the finish pass. */
struct LinkSmem {
    uint32_t off[kStep + 1];
    uint64_t beg[kStep];
    uint32_t wsum[kWarpsB];
    uint32_t heavy_n;
    uint32_t heavy_v[kStep];
    uint64_t heavy_b[kStep], heavy_e[kStep];
};

/* Finish pass over one tile: rows of vertices outside the graph's giant tree
 * (valid for symmetric graphs: every edge leaving the tree is seen from its
 * other end).  Short rows are gathered per CTA and walked edge-parallel,
 * rows of at least warp_deg entries by a warp; rows above heavy_deg go to
 * the class's heavy queue, or, with inline_heavy, are walked by the whole
 * CTA once the tile's other rows are done. */
__device__ __forceinline__ void tile_link(const BatchK &K, const Tile &T, LinkSmem &S,
                                          bool inline_heavy)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t giant = K.skip ? __ldg(K.giants + T.g) : kNone;
    if (threadIdx.x == 0)
        S.heavy_n = 0;
    __syncthreads();
    for (uint32_t t0 = T.v0; t0 < T.v1; t0 += kStep) {
        uint64_t beg[kVPT], end[kVPT];
        uint32_t small[kVPT], mine = 0;
#pragma unroll
        for (int k = 0; k < kVPT; ++k) {
            const uint32_t v = t0 + threadIdx.x * kVPT + k;
            beg[k] = end[k] = 0;
            if (v < T.v1 && (giant == kNone || cc_ldp(T.parent, v) != giant))
                row_bounds(T, v, beg[k], end[k]);
            uint64_t deg = end[k] - beg[k];
            if (deg > K.heavy_deg) {
                if (inline_heavy) {
                    const uint32_t slot = atomicAdd(&S.heavy_n, 1u);
                    S.heavy_v[slot] = v;
                    S.heavy_b[slot] = beg[k];
                    S.heavy_e[slot] = end[k];
                    deg = 0;
                    end[k] = beg[k];
                } else {
                    const uint32_t slot = atomicAdd(K.heavy_count, 1u);
                    if (slot < K.heavy_cap) {
                        K.heavy_list[slot] = ((uint64_t)T.g << 32) | v;
                        deg = 0;
                        end[k] = beg[k];
                    }
                }
            }
            unsigned big = __ballot_sync(0xffffffffu, deg >= K.warp_deg);
            while (big) {
                const int src = __ffs(big) - 1;
                big &= big - 1;
                const uint32_t vv = __shfl_sync(0xffffffffu, v, src);
                const uint64_t bb = __shfl_sync(0xffffffffu, beg[k], src);
                const uint64_t ee = __shfl_sync(0xffffffffu, end[k], src);
                warp_row(T, vv, bb, ee, lane);
            }
            small[k] = deg < K.warp_deg ? (uint32_t)deg : 0u;
            mine += small[k];
            S.beg[threadIdx.x * kVPT + k] = beg[k];
        }
        uint32_t incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += y;
        }
        if (lane == 31)
            S.wsum[warp] = incl;
        __syncthreads();
        uint32_t wpre = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kWarpsB; ++w) {
            const uint32_t x = S.wsum[w];
            wpre += (w < warp) ? x : 0u;
            total += x;
        }
        uint32_t run = wpre + incl - mine;
#pragma unroll
        for (int k = 0; k < kVPT; ++k) {
            S.off[threadIdx.x * kVPT + k] = run;
            run += small[k];
        }
        if (threadIdx.x == 0)
            S.off[kStep] = total;
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < total; e += kB) {
            int lo = 0, hi = kStep;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (S.off[mid] <= e)
                    lo = mid;
                else
                    hi = mid;
            }
            const uint32_t u = __ldg(T.col + S.beg[lo] + (e - S.off[lo]));
            if (u < T.n)
                cc_link(T.parent, t0 + (uint32_t)lo, u);
        }
        if (inline_heavy) { /* this step's heavy rows (at most kStep) */
            const uint32_t nh = S.heavy_n;
            for (uint32_t h = 0; h < nh; ++h) {
                const uint32_t v = S.heavy_v[h];
                for (uint64_t j = S.heavy_b[h] + threadIdx.x; j < S.heavy_e[h]; j += kB) {
                    const uint32_t u = __ldg(T.col + j);
                    if (u < T.n)
                        cc_link(T.parent, v, u);
                }
            }
        }
        __syncthreads();
        if (inline_heavy && threadIdx.x == 0)
            S.heavy_n = 0;
        __syncthreads();
    }
}

/* Finish pass: tiles grabbed with an atomic counter. */
__global__ void __launch_bounds__(kB, 4) kb_link(BatchK K)
{
    __shared__ LinkSmem S;
    __shared__ unsigned long long s_t;
    for (;;) {
        if (threadIdx.x == 0)
            s_t = atomicAdd(K.grab, 1ull);
        __syncthreads();
        const unsigned long long t = s_t;
        __syncthreads();
        if (t >= K.tiles)
            break;
        tile_link(K, tile_of(K, (uint32_t)t), S, false);
    }
}

__global__ void __launch_bounds__(kB) kb_heavy(BatchK K)
{
    uint32_t cnt = *K.heavy_count;
    if (cnt > K.heavy_cap)
        cnt = K.heavy_cap;
    const int lane = threadIdx.x & 31;
    cc_for_pieces(
        cnt, kPiece,
        [&](uint32_t h, uint64_t &b, uint64_t &e) {
            const uint64_t gv = K.heavy_list[h];
            const uint32_t g = (uint32_t)(gv >> 32), v = (uint32_t)gv;
            const uint64_t m = __ldg(&K.gr[g].m);
            const uint64_t *rp = K.row_ptr + __ldg(&K.gr[g].rp);
            b = __ldg(rp + v);
            e = __ldg(rp + v + 1);
            if (e > m)
                e = m;
            if (b > e)
                b = e;
        },
        [&](uint32_t h, uint64_t jb, uint64_t je) {
            const uint64_t gv = K.heavy_list[h];
            const uint32_t g = (uint32_t)(gv >> 32), v = (uint32_t)gv;
            const uint32_t n = __ldg(&K.gr[g].n);
            const uint32_t *col = K.col + __ldg(&K.gr[g].col);
            uint32_t *parent = K.labels + __ldg(&K.gr[g].lab);
            for (uint64_t j0 = jb; j0 < je; j0 += 32) {
                const uint64_t j = j0 + lane;
                uint32_t u[1] = {0};
                bool ok[1] = {false};
                if (j < je) {
                    u[0] = __ldg(col + j);
                    ok[0] = u[0] < n;
                }
                cc_warp_link_min_first<1>(parent, v, u, ok, lane);
            }
        });
}

/* Root of x read through L2 (ld.global.cg): in a persistent launch a
 * block's L1 may hold parent values written before other blocks' links,
 * and a stale "root" must not become a final label. */
__device__ __forceinline__ uint32_t find_coherent(uint32_t *parent, uint32_t x)
{
    uint32_t p;
    asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(p) : "l"(parent + x));
    while (p != x) {
        uint32_t gp;
        asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(gp) : "l"(parent + p));
        if (gp == p)
            return p;
        atomicMin(parent + x, gp);
        x = gp;
        asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(p) : "l"(parent + x));
    }
    return x;
}

/* labels[v] = root(v) over the tile; the graph's component count, and its
 * done flag set by its last tile. */
__device__ __forceinline__ void tile_final(const BatchK &K, const Tile &T, uint32_t *s_c,
                                           bool coherent)
{
    uint32_t c = 0;
    for (uint32_t v = T.v0 + threadIdx.x; v < T.v1; v += kB) {
        const uint32_t r = coherent ? find_coherent(T.parent, v) : cc_find(T.parent, v);
        if (r != v)
            T.parent[v] = r;
        c += r == v;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0)
        s_c[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t sum = 0;
        for (int w = 0; w < kWarpsB; ++w)
            sum += s_c[w];
        if (sum)
            atomicAdd(K.comps + T.g, sum);
        const uint32_t ntiles = (T.n + K.tile - 1) / K.tile;
        __threadfence();
        if (atomicAdd(K.tiles_done + T.g, 1u) + 1 == ntiles)
            atomicExch(K.done + T.g, 1u);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kB) kb_final(BatchK K)
{
    __shared__ uint32_t s_c[kWarpsB];
    for (uint32_t t = blockIdx.x; t < K.tiles; t += gridDim.x)
        tile_final(K, tile_of(K, t), s_c, false);
}

/* ------------------------------------------------- persistent launch */

/* One launch moves every graph of every degree class through the solve's
 * phases.  Each class's solve is a program of phases (init, sample rounds
 * and compressions, giant, link, final); a phase's work items are its
 * class's tiles - or graphs, for the giant phase.  The launch's items are
 * the segments (class, phase) in phase-major order across the classes, so
 * the classes advance together; blocks take items from one counter in that
 * order.  An item of phase k of a class waits until its graph's counter of
 * phase k-1 shows all of that phase's items done.  Items are taken in
 * order and every item depends only on items before it, so the oldest
 * unfinished item never waits and the launch always progresses; each wait
 * is still bounded (wait_ns of the global timer), and one that runs out
 * sets *err, after which every block stops taking items. */
constexpr int kMaxPhases = 12;
constexpr int kMaxSegs = CCGPU_BATCH_CLASSES * kMaxPhases;
enum { PH_INIT = 0, PH_SAMPLE = 1, PH_COMPRESS = 2, PH_GIANT = 3, PH_LINK = 4, PH_FINAL = 5 };

struct PersistK {
    BatchK K[CCGPU_BATCH_CLASSES];
    int nseg;
    int cls[kMaxSegs];             /* class of the segment                  */
    int kind[kMaxSegs];
    int round[kMaxSegs];           /* sample round                          */
    int phase[kMaxSegs];           /* phase index within its class          */
    int prev_kind[kMaxSegs];       /* kind of the class's previous phase    */
    uint64_t off[kMaxSegs + 1];    /* first item of each segment            */
    uint32_t *pcnt;                /* [G * kMaxPhases] items done per graph */
    unsigned long long *grab;
    int *err;
    unsigned long long wait_ns;
    uint32_t stall_graph;          /* kNone = off                           */
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

/* The giant phase of one graph with 256 threads: the same 1024 seeded
 * samples as kb_giant, sorted bitonically 4 per thread, and the most
 * frequent root (ties to the smaller). */
__device__ __forceinline__ void graph_giant(const BatchK &K, uint32_t g, uint32_t seed,
                                            uint32_t *s, unsigned long long *s_best)
{
    const uint32_t n = __ldg(&K.gr[g].n);
    const uint32_t *parent = K.labels + __ldg(&K.gr[g].lab);
    if (n == 0) {
        if (threadIdx.x == 0)
            K.giants[g] = kNone;
        return;
    }
    for (uint32_t i = threadIdx.x; i < 1024; i += kB) {
        const uint32_t h = cc_mix32(i * 0x9e3779b9u + seed + g);
        const uint32_t v = (uint32_t)(((uint64_t)h * n) >> 32);
        s[i] = cc_find_ro(parent, v);
    }
    __syncthreads();
    for (uint32_t k = 2; k <= 1024; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < 1024; i += kB) {
                const uint32_t ij = i ^ j;
                if (ij > i) {
                    const uint32_t a = s[i], b = s[ij];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        s[i] = b;
                        s[ij] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    unsigned long long key = 0;
    for (uint32_t i = threadIdx.x; i < 1024; i += kB) {
        const uint32_t val = s[i];
        if (i == 0 || s[i - 1] != val) {
            uint32_t a = i, b = 1024;
            while (a < b) {
                const uint32_t mid = (a + b) >> 1;
                if (s[mid] <= val)
                    a = mid + 1;
                else
                    b = mid;
            }
            const unsigned long long kk = ((unsigned long long)(a - i) << 32) | (uint32_t)~val;
            key = kk > key ? kk : key;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if ((threadIdx.x & 31) == 0)
        s_best[threadIdx.x >> 5] = key;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long best = 0;
        for (int w = 0; w < kWarpsB; ++w)
            best = s_best[w] > best ? s_best[w] : best;
        K.giants[g] = ~(uint32_t)best;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kB) kb_persist(const __grid_constant__ PersistK Q)
{
    __shared__ LinkSmem S;
    __shared__ uint32_t s_g[1024];
    __shared__ unsigned long long s_best[kWarpsB];
    __shared__ uint32_t s_c[kWarpsB];
    __shared__ unsigned long long s_item;
    __shared__ int s_seg, s_stop;
    const uint64_t total = Q.off[Q.nseg];
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned long long item =
                *(volatile int *)Q.err ? ~0ull : atomicAdd(Q.grab, 1ull);
            int sg = 0;
            while (sg + 1 < Q.nseg && Q.off[sg + 1] <= item)
                ++sg;
            s_item = item;
            s_seg = sg;
            s_stop = 0;
        }
        __syncthreads();
        const unsigned long long item = s_item;
        if (item >= total)
            break;
        const int sg = s_seg;
        const BatchK &K = Q.K[Q.cls[sg]];
        const uint64_t idx = item - Q.off[sg];
        const int kind = Q.kind[sg], ph = Q.phase[sg];
        Tile T;
        uint32_t g;
        if (kind == PH_GIANT) {
            g = __ldg(K.graphs + idx);
        } else {
            T = tile_of(K, (uint32_t)idx);
            g = T.g;
        }
        if (ph > 0 && threadIdx.x == 0) {
            /* items of the class's previous phase for this graph: one giant
             * item, or one per tile */
            const uint32_t n = __ldg(&K.gr[g].n);
            uint32_t need = Q.prev_kind[sg] == PH_GIANT ? 1u : (n + K.tile - 1) / K.tile;
            if (g == Q.stall_graph && ph == 1)
                need += 1; /* never met: exercises the bounded wait */
            const uint32_t *c = Q.pcnt + (uint64_t)g * kMaxPhases + (ph - 1);
            if (ld_acquire(c) < need) {
                const unsigned long long t0 = global_ns();
                while (ld_acquire(c) < need) {
                    if (*(volatile int *)Q.err || global_ns() - t0 > Q.wait_ns) {
                        atomicExch(Q.err, 1);
                        s_stop = 1;
                        break;
                    }
                    __nanosleep(256);
                }
            }
        }
        __syncthreads();
        if (s_stop)
            break;
        switch (kind) {
        case PH_INIT: tile_init(T); break;
        case PH_SAMPLE: tile_sample(K, T, Q.round[sg]); break;
        case PH_COMPRESS: tile_compress(T); break;
        case PH_GIANT: graph_giant(K, g, 0x5eed1234u, s_g, s_best); break;
        case PH_LINK: tile_link(K, T, S, true); break;
        default: tile_final(K, T, s_c, true); break;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(Q.pcnt + (uint64_t)g * kMaxPhases + ph, 1u);
        }
    }
}

/* ------------------------------------------------------------- the core */

/* Grows the pair of tile arrays of a class together (one capacity). */
int grow_tiles(BatchClass &C, size_t need)
{
    if (need <= C.tile_cap && C.d_tile_g)
        return CCGPU_OK;
    cudaFree(C.d_tile_g);
    cudaFree(C.d_tile_v0);
    C.d_tile_g = C.d_tile_v0 = nullptr;
    C.tile_cap = 0;
    const size_t want = need + need / 2 + 64;
    CC_CUDA(cudaMalloc((void **)&C.d_tile_g, want * sizeof(uint32_t)));
    CC_CUDA(cudaMalloc((void **)&C.d_tile_v0, want * sizeof(uint32_t)));
    C.tile_cap = want;
    return CCGPU_OK;
}

template <typename T>
int grow(T **p, size_t *cap, size_t need)
{
    if (need <= *cap && *p)
        return CCGPU_OK;
    size_t want = need + need / 2 + 64;
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    CC_CUDA(cudaMalloc((void **)p, want * sizeof(T)));
    *cap = want;
    return CCGPU_OK;
}

BatchK kargs(BatchCore *c, int k)
{
    BatchClass &C = c->cls[k];
    BatchK K;
    K.gr = c->d_gr;
    K.row_ptr = c->row_ptr;
    K.col = c->col;
    K.labels = c->labels;
    K.tile_g = C.d_tile_g;
    K.tile_v0 = C.d_tile_v0;
    K.tiles = C.tiles;
    K.tile = (uint32_t)C.o.tile;
    K.graphs = C.d_graphs;
    K.ngraphs = (uint32_t)C.graphs.size();
    K.giants = c->d_giants;
    K.comps = c->d_comps;
    K.tiles_done = c->d_tiles_done;
    K.done = c->d_done;
    K.grab = C.d_cnt;
    K.heavy_count = (uint32_t *)(C.d_cnt + 1);
    K.heavy_list = C.d_heavy;
    K.heavy_cap = C.heavy_used;
    K.heavy_deg = (uint32_t)c->tune.heavy_degree;
    K.warp_deg = (uint32_t)C.o.warp_degree;
    K.skip = C.o.sample_rounds > 0;
    K.stash = (c->stash && C.o.sample_rounds >= 2 && C.entries >= 8ull * C.vertices) ? c->stash
                                                                                    : nullptr;
    return K;
}

/* Tile list of class k into `tg`/`tv` (host). */
void tiles_of(const BatchCore *c, int k, std::vector<uint32_t> &tg, std::vector<uint32_t> &tv)
{
    const BatchClass &C = c->cls[k];
    const uint32_t T = (uint32_t)C.o.tile;
    tg.clear();
    tv.clear();
    for (uint32_t g : C.graphs)
        for (uint64_t v0 = 0; v0 < c->gr[g].n; v0 += T) {
            tg.push_back(g);
            tv.push_back((uint32_t)v0);
        }
}

int stage(BatchCore *c, size_t bytes)
{
    if (bytes <= c->stage_cap && c->h_stage)
        return CCGPU_OK;
    if (c->h_stage)
        CC_CUDA(cudaFreeHost(c->h_stage));
    c->h_stage = nullptr;
    c->stage_cap = 0;
    const size_t want = bytes + bytes / 2 + 4096;
    CC_CUDA(cudaMallocHost(&c->h_stage, want));
    c->stage_cap = want;
    return CCGPU_OK;
}

} // namespace

int batch_class_of(const ccgpu_batch_tuning &t, uint64_t n, uint64_t m)
{
    const double avg = n ? (double)m / (double)n : 0.0;
    int c = 0;
    while (c < CCGPU_BATCH_CLASSES - 1 && avg >= t.class_bounds[c])
        ++c;
    return c;
}

int batch_check_tuning(ccgpu_batch_tuning *t)
{
    if (t->heavy_degree < 32)
        t->heavy_degree = 32;
    if (t->wait_ms < 0)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "batch: wait_ms %d is negative", t->wait_ms);
    for (int c = 0; c < CCGPU_BATCH_CLASSES; ++c) {
        const ccgpu_batch_class_opts &o = t->cls[c];
        if (o.sample_rounds < 0 || o.sample_rounds > 4)
            return ccgpu_set_error(CCGPU_ERR_INVALID, "batch: sample_rounds %d not in 0..4",
                                   o.sample_rounds);
        if (o.tile < 256 || o.tile > (1 << 20) || (o.tile & (o.tile - 1)))
            return ccgpu_set_error(CCGPU_ERR_INVALID,
                                   "batch: tile %d is not a power of two in 256..2^20", o.tile);
        if (o.warp_degree < 2 || o.warp_degree > 1024)
            return ccgpu_set_error(CCGPU_ERR_INVALID, "batch: warp_degree %d not in 2..1024",
                                   o.warp_degree);
    }
    return CCGPU_OK;
}

int batch_core_init(BatchCore *c, ccgpu_ctx *ctx, const ccgpu_batch_tuning *tuning)
{
    c->ctx = ctx;
    c->sms = ctx->sm_count;
    if (tuning)
        c->tune = *tuning;
    else
        ccgpu_batch_tuning_default(&c->tune);
    CC_TRY(batch_check_tuning(&c->tune));
    CC_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
    CC_CUDA(cudaMalloc((void **)&c->d_err, sizeof(int)));
    CC_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
    CC_CUDA(cudaMalloc((void **)&c->d_grab, sizeof(unsigned long long)));
    for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k) {
        c->cls[k].o = c->tune.cls[k];
        CC_CUDA(cudaStreamCreateWithFlags(&c->cls[k].st, cudaStreamNonBlocking));
        CC_CUDA(cudaEventCreateWithFlags(&c->cls[k].ev, cudaEventDisableTiming));
        CC_CUDA(cudaMalloc((void **)&c->cls[k].d_cnt, 256));
    }
    return CCGPU_OK;
}

void batch_core_free(BatchCore *c)
{
    for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k) {
        BatchClass &C = c->cls[k];
        cudaFree(C.d_graphs);
        cudaFree(C.d_tile_g);
        cudaFree(C.d_tile_v0);
        cudaFree(C.d_cnt);
        cudaFree(C.d_heavy);
        if (C.st)
            cudaStreamDestroy(C.st);
        if (C.ev)
            cudaEventDestroy(C.ev);
        C = BatchClass();
    }
    if (c->fork)
        cudaEventDestroy(c->fork);
    cudaFree(c->d_gr);
    cudaFree(c->d_giants);
    cudaFree(c->d_comps);
    cudaFree(c->d_tiles_done);
    cudaFree(c->d_done);
    cudaFree(c->d_pcnt);
    cudaFree(c->d_err);
    cudaFree(c->d_grab);
    if (c->h_stage)
        cudaFreeHost(c->h_stage);
    cudaFree(c->stash);
    *c = BatchCore();
}

int batch_core_stash(BatchCore *c, size_t entries)
{
    return grow(&c->stash, &c->stash_cap, entries ? entries : 1);
}

int batch_core_reserve(BatchCore *c, size_t graphs, size_t tiles, size_t heavy)
{
    if (graphs > c->g_cap || !c->d_gr) {
        cudaFree(c->d_gr);
        cudaFree(c->d_giants);
        cudaFree(c->d_comps);
        cudaFree(c->d_tiles_done);
        cudaFree(c->d_done);
        cudaFree(c->d_pcnt);
        c->d_gr = nullptr;
        c->d_giants = c->d_comps = c->d_tiles_done = c->d_done = c->d_pcnt = nullptr;
        c->g_cap = 0;
        CC_CUDA(cudaMalloc((void **)&c->d_gr, graphs * sizeof(BGraph)));
        CC_CUDA(cudaMalloc((void **)&c->d_giants, graphs * sizeof(uint32_t)));
        CC_CUDA(cudaMalloc((void **)&c->d_comps, graphs * sizeof(uint32_t)));
        CC_CUDA(cudaMalloc((void **)&c->d_tiles_done, graphs * sizeof(uint32_t)));
        CC_CUDA(cudaMalloc((void **)&c->d_done, graphs * sizeof(uint32_t)));
        CC_CUDA(cudaMalloc((void **)&c->d_pcnt, graphs * kMaxPhases * sizeof(uint32_t)));
        c->g_cap = graphs;
    }
    for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k) {
        BatchClass &C = c->cls[k];
        CC_TRY(grow(&C.d_graphs, &C.graphs_cap, graphs));
        CC_TRY(grow_tiles(C, tiles));
        CC_TRY(grow(&C.d_heavy, &C.heavy_cap, heavy));
    }
    return stage(c, graphs * sizeof(BGraph) +
                        CCGPU_BATCH_CLASSES * ((graphs + 2 * tiles) * sizeof(uint32_t) + 64));
}

int batch_core_set(BatchCore *c, const uint64_t *row_ptr, const uint32_t *col, uint32_t *labels,
                   const BGraph *gr, uint32_t G, cudaStream_t st, int sync)
{
    c->row_ptr = row_ptr;
    c->col = col;
    c->labels = labels;
    c->gr.assign(gr, gr + G);
    for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k) {
        BatchClass &C = c->cls[k];
        C.graphs.clear();
        C.vertices = C.entries = 0;
    }
    for (uint32_t g = 0; g < G; ++g) {
        BatchClass &C = c->cls[batch_class_of(c->tune, gr[g].n, gr[g].m)];
        C.graphs.push_back(g);
        C.vertices += gr[g].n;
        C.entries += gr[g].m;
    }
    if (G > c->g_cap || !c->d_gr) { /* per-graph arrays grow together */
        cudaFree(c->d_gr);
        cudaFree(c->d_giants);
        cudaFree(c->d_comps);
        cudaFree(c->d_tiles_done);
        cudaFree(c->d_done);
        cudaFree(c->d_pcnt);
        c->d_gr = nullptr;
        c->d_giants = c->d_comps = c->d_tiles_done = c->d_done = c->d_pcnt = nullptr;
        c->g_cap = 0;
        const size_t want = (size_t)G + G / 2 + 64;
        CC_CUDA(cudaMalloc((void **)&c->d_gr, want * sizeof(BGraph)));
        CC_CUDA(cudaMalloc((void **)&c->d_giants, want * sizeof(uint32_t)));
        CC_CUDA(cudaMalloc((void **)&c->d_comps, want * sizeof(uint32_t)));
        CC_CUDA(cudaMalloc((void **)&c->d_tiles_done, want * sizeof(uint32_t)));
        CC_CUDA(cudaMalloc((void **)&c->d_done, want * sizeof(uint32_t)));
        CC_CUDA(cudaMalloc((void **)&c->d_pcnt, want * kMaxPhases * sizeof(uint32_t)));
        c->g_cap = want;
    }
    /* staging: descriptors, then per class graph list and tile list */
    std::vector<uint32_t> tg[CCGPU_BATCH_CLASSES], tv[CCGPU_BATCH_CLASSES];
    size_t bytes = (size_t)G * sizeof(BGraph);
    for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k) {
        tiles_of(c, k, tg[k], tv[k]);
        bytes += (c->cls[k].graphs.size() + 2 * tg[k].size()) * sizeof(uint32_t) + 64;
    }
    CC_TRY(stage(c, bytes));
    char *h = (char *)c->h_stage;
    size_t off = 0;
    auto put = [&](const void *src, size_t n) -> char * {
        char *dst = h + off;
        if (n)
            memcpy(dst, src, n);
        off = (off + n + 15) & ~(size_t)15;
        return dst;
    };
    char *hg = put(gr, (size_t)G * sizeof(BGraph));
    if (G)
        CC_CUDA(cudaMemcpyAsync(c->d_gr, hg, (size_t)G * sizeof(BGraph), cudaMemcpyHostToDevice,
                                st));
    for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k) {
        BatchClass &C = c->cls[k];
        const size_t ng = C.graphs.size(), nt = tg[k].size();
        CC_TRY(grow(&C.d_graphs, &C.graphs_cap, ng ? ng : 1));
        CC_TRY(grow_tiles(C, nt ? nt : 1));
        uint64_t hc = C.entries / (uint64_t)c->tune.heavy_degree + 1;
        if (hc > C.vertices + 1)
            hc = C.vertices + 1;
        if (hc > 0xffffffffull)
            hc = 0xffffffffull;
        CC_TRY(grow(&C.d_heavy, &C.heavy_cap, (size_t)hc));
        C.heavy_used = (uint32_t)hc;
        C.tiles = (uint32_t)nt;
        if (ng) {
            char *p = put(C.graphs.data(), ng * 4);
            CC_CUDA(cudaMemcpyAsync(C.d_graphs, p, ng * 4, cudaMemcpyHostToDevice, st));
        }
        if (nt) {
            char *p = put(tg[k].data(), nt * 4);
            CC_CUDA(cudaMemcpyAsync(C.d_tile_g, p, nt * 4, cudaMemcpyHostToDevice, st));
            p = put(tv[k].data(), nt * 4);
            CC_CUDA(cudaMemcpyAsync(C.d_tile_v0, p, nt * 4, cudaMemcpyHostToDevice, st));
        }
    }
    if (sync)
        CC_CUDA(cudaStreamSynchronize(st));
    return CCGPU_OK;
}

int batch_core_retile(BatchCore *c, int k)
{
    BatchClass &C = c->cls[k];
    std::vector<uint32_t> tg, tv;
    tiles_of(c, k, tg, tv);
    const size_t nt = tg.size();
    CC_TRY(grow_tiles(C, nt ? nt : 1));
    if (nt) {
        CC_CUDA(cudaMemcpy(C.d_tile_g, tg.data(), nt * 4, cudaMemcpyHostToDevice));
        CC_CUDA(cudaMemcpy(C.d_tile_v0, tv.data(), nt * 4, cudaMemcpyHostToDevice));
    }
    C.tiles = (uint32_t)nt;
    return CCGPU_OK;
}

int batch_core_enqueue_class(BatchCore *c, int k, cudaStream_t st, int *kernels)
{
    BatchClass &C = c->cls[k];
    if (C.graphs.empty() || C.tiles == 0)
        return CCGPU_OK;
    ccgpu_ctx *ctx = c->ctx;
    const BatchK K = kargs(c, k);
    const unsigned tb = cc_blocks(C.tiles, 1, (unsigned)c->sms * 8);
    int n = 0;
    CC_CUDA(cudaMemsetAsync(C.d_cnt, 0, 2 * sizeof(unsigned long long), st));
    CC_KLAUNCH(ctx, CCK_BATCH_INIT, kb_init, tb, kB, 0, st, K);
    ++n;
    const int rounds = C.o.sample_rounds;
    for (int r = 0; r < rounds; ++r) {
        CC_KLAUNCH(ctx, CCK_BATCH_SAMPLE, kb_sample, tb, kB, 0, st, K, r);
        ++n;
        if (C.o.cadence || r + 1 == rounds) {
            CC_KLAUNCH(ctx, CCK_BATCH_COMPRESS, kb_compress, tb, kB, 0, st, K);
            ++n;
        }
    }
    if (rounds > 0) {
        const unsigned gb = cc_blocks(C.graphs.size(), 1, (unsigned)c->sms * 2);
        CC_KLAUNCH(ctx, CCK_BATCH_GIANT, kb_giant, gb, 1024, 0, st, K, 0x5eed1234u);
        ++n;
    }
    CC_KLAUNCH(ctx, CCK_BATCH_LINK, kb_link, (unsigned)c->sms * 4, kB, 0, st, K);
    CC_KLAUNCH(ctx, CCK_BATCH_HEAVY, kb_heavy, (unsigned)c->sms * 4, kB, 0, st, K);
    CC_KLAUNCH(ctx, CCK_BATCH_FINAL, kb_final, tb, kB, 0, st, K);
    n += 3;
    if (kernels)
        *kernels += n;
    return CCGPU_OK;
}

/* The whole batch as one persistent launch (kb_persist). */
int batch_core_enqueue_persistent(BatchCore *c, cudaStream_t st, int *kernels)
{
    PersistK Q;
    memset(&Q, 0, sizeof(Q));
    struct Prog {
        int n = 0;
        int kind[kMaxPhases], round[kMaxPhases];
        uint64_t items[kMaxPhases];
    } prog[CCGPU_BATCH_CLASSES];
    int longest = 0;
    for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k) {
        BatchClass &C = c->cls[k];
        if (C.graphs.empty() || C.tiles == 0)
            continue;
        Q.K[k] = kargs(c, k);
        Prog &P = prog[k];
        auto add = [&](int kind, int round, uint64_t items) {
            P.kind[P.n] = kind;
            P.round[P.n] = round;
            P.items[P.n] = items;
            P.n++;
        };
        const int rounds = C.o.sample_rounds;
        add(PH_INIT, 0, C.tiles);
        for (int r = 0; r < rounds; ++r) {
            add(PH_SAMPLE, r, C.tiles);
            if (C.o.cadence || r + 1 == rounds)
                add(PH_COMPRESS, 0, C.tiles);
        }
        if (rounds > 0)
            add(PH_GIANT, 0, C.graphs.size());
        add(PH_LINK, 0, C.tiles);
        add(PH_FINAL, 0, C.tiles);
        longest = P.n > longest ? P.n : longest;
    }
    for (int ph = 0; ph < longest; ++ph)
        for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k) {
            const Prog &P = prog[k];
            if (ph >= P.n)
                continue;
            const int sg = Q.nseg++;
            Q.cls[sg] = k;
            Q.kind[sg] = P.kind[ph];
            Q.round[sg] = P.round[ph];
            Q.phase[sg] = ph;
            Q.prev_kind[sg] = ph ? P.kind[ph - 1] : -1;
            Q.off[sg + 1] = Q.off[sg] + P.items[ph];
        }
    if (Q.nseg == 0)
        return CCGPU_OK;
    Q.pcnt = c->d_pcnt;
    Q.grab = c->d_grab;
    Q.err = c->d_err;
    Q.wait_ns = (unsigned long long)(c->tune.wait_ms ? c->tune.wait_ms : 2000) * 1000000ull;
    Q.stall_graph = c->tune.stall_graph >= 0 ? (uint32_t)c->tune.stall_graph : kNone;
    if (!c->persist_blocks) {
        CC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->persist_blocks, kb_persist, kB,
                                                              0));
        if (c->persist_blocks < 1)
            c->persist_blocks = 1;
    }
    CC_CUDA(cudaMemsetAsync(c->d_grab, 0, sizeof(unsigned long long), st));
    const uint64_t items = Q.off[Q.nseg];
    uint64_t grid = (uint64_t)c->sms * (uint64_t)c->persist_blocks;
    if (grid > items)
        grid = items;
    CC_KLAUNCH(c->ctx, CCK_BATCH, kb_persist, (unsigned)(grid ? grid : 1), kB, 0, st, Q);
    if (kernels)
        *kernels += 1;
    return CCGPU_OK;
}

int batch_core_enqueue(BatchCore *c, cudaStream_t st, int *kernels)
{
    const size_t gbytes = (c->gr.empty() ? 1 : c->gr.size()) * sizeof(uint32_t);
    CC_CUDA(cudaMemsetAsync(c->d_comps, 0, gbytes, st));
    CC_CUDA(cudaMemsetAsync(c->d_tiles_done, 0, gbytes, st));
    CC_CUDA(cudaMemsetAsync(c->d_done, 0, gbytes, st));
    if (c->tune.persistent) {
        CC_CUDA(cudaMemsetAsync(c->d_pcnt, 0, gbytes * kMaxPhases, st));
        CC_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), st));
        return batch_core_enqueue_persistent(c, st, kernels);
    }
    CC_CUDA(cudaEventRecord(c->fork, st));
    for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k) {
        BatchClass &C = c->cls[k];
        if (C.graphs.empty())
            continue;
        CC_CUDA(cudaStreamWaitEvent(C.st, c->fork, 0));
        CC_TRY(batch_core_enqueue_class(c, k, C.st, kernels));
        CC_CUDA(cudaEventRecord(C.ev, C.st));
        CC_CUDA(cudaStreamWaitEvent(st, C.ev, 0));
    }
    return CCGPU_OK;
}

/* -------------------------------------------------- packed-batch plans */

struct ccgpu_batch_plan {
    BatchCore core;
    uint32_t G = 0;
    std::vector<uint64_t> vtx_off;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
};

namespace {

void drop_graph(ccgpu_batch_plan *p)
{
    if (p->exec)
        cudaGraphExecDestroy(p->exec);
    if (p->graph)
        cudaGraphDestroy(p->graph);
    p->exec = nullptr;
    p->graph = nullptr;
}

int capture(ccgpu_batch_plan *p)
{
    drop_graph(p);
    cudaStream_t cs = nullptr;
    CC_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    int kernels = 0;
    int rc = CCGPU_OK;
    /* the launch profiler would record events into the graph: off while
     * capturing */
    ccgpu_ctx *ctx = p->core.ctx;
    struct cc_prof *saved = ctx->prof;
    ctx->prof = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        rc = ccgpu_cuda_fail(e, "cudaStreamBeginCapture", __FILE__, __LINE__);
    } else {
        rc = batch_core_enqueue(&p->core, cs, &kernels);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(cs, &g);
        if (rc == CCGPU_OK && e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        if (rc == CCGPU_OK) {
            e = cudaGraphInstantiate(&p->exec, g, 0);
            if (e != cudaSuccess)
                rc = ccgpu_cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__);
            p->graph = g;
        } else if (g) {
            cudaGraphDestroy(g);
        }
    }
    ctx->prof = saved;
    cudaStreamDestroy(cs);
    if (rc == CCGPU_OK)
        p->kernels = kernels;
    return rc;
}

/* Device time of `reps` solves of class k alone (after one warm-up). */
int time_class(BatchCore *c, int k, cudaStream_t st, int reps, float *ms)
{
    cudaEvent_t a = nullptr, z = nullptr;
    CC_CUDA(cudaEventCreate(&a));
    CC_CUDA(cudaEventCreate(&z));
    int rc = batch_core_enqueue_class(c, k, st, nullptr);
    if (rc == CCGPU_OK && cudaEventRecord(a, st) != cudaSuccess)
        rc = ccgpu_set_error(CCGPU_ERR_CUDA, "batch autotune: event record failed");
    for (int i = 0; rc == CCGPU_OK && i < reps; ++i)
        rc = batch_core_enqueue_class(c, k, st, nullptr);
    if (rc == CCGPU_OK) {
        cudaEventRecord(z, st);
        cudaError_t e = cudaEventSynchronize(z);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(ms, a, z);
        if (e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "batch autotune timing", __FILE__, __LINE__);
        *ms /= (float)reps;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    return rc;
}

} // namespace

/* ------------------------------------------------------------------ API */

extern "C" void ccgpu_batch_tuning_default(ccgpu_batch_tuning *t)
{
    if (!t)
        return;
    memset(t, 0, sizeof(*t));
    t->class_bounds[0] = 6.0f;
    t->class_bounds[1] = 16.0f;
    t->heavy_degree = 8192;
    t->persistent = 0;
    t->wait_ms = 0;
    t->stall_graph = -1;
    for (int c = 0; c < CCGPU_BATCH_CLASSES; ++c) {
        t->cls[c].sample_rounds = 2;
        t->cls[c].cadence = 1;
        t->cls[c].tile = 4096;
        t->cls[c].warp_degree = 32;
    }
}

namespace {

/* Checks a batch and builds its per-graph descriptors. */
int batch_descs(const ccgpu_batch *b, std::vector<BGraph> &gr)
{
    if (b->graphs == 0)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_plan_create: empty batch");
    if (!b->d_row_ptr || !b->d_labels || (b->h_edge_off[b->graphs] && !b->d_col))
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_plan_create: NULL device array");
    const uint32_t G = b->graphs;
    const uint64_t *vo = b->h_vtx_off, *eo = b->h_edge_off;
    if (vo[0] != 0 || eo[0] != 0)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "batch: offsets must start at 0");
    gr.resize(G);
    for (uint32_t g = 0; g < G; ++g) {
        if (vo[g + 1] < vo[g] || eo[g + 1] < eo[g])
            return ccgpu_set_error(CCGPU_ERR_INVALID, "batch: offsets of graph %u decrease", g);
        if (vo[g + 1] - vo[g] >= 0xffffffffull)
            return ccgpu_set_error(CCGPU_ERR_LIMIT, "batch: graph %u has 2^32-1 or more vertices",
                                   g);
        gr[g].rp = vo[g] + g;
        gr[g].col = eo[g];
        gr[g].lab = vo[g];
        gr[g].n = (uint32_t)(vo[g + 1] - vo[g]);
        gr[g].m = eo[g + 1] - eo[g];
        gr[g].pad = 0;
    }
    return CCGPU_OK;
}

/* Points an initialised plan at a batch: tuning, descriptors, tiles and a
 * stash covering its labels.  Device arrays only grow. */
int plan_set(ccgpu_batch_plan *p, const ccgpu_batch *b, const ccgpu_batch_tuning &t,
             const std::vector<BGraph> &gr)
{
    drop_graph(p);
    p->G = b->graphs;
    p->vtx_off.assign(b->h_vtx_off, b->h_vtx_off + b->graphs + 1);
    p->core.tune = t;
    for (int k = 0; k < CCGPU_BATCH_CLASSES; ++k)
        p->core.cls[k].o = t.cls[k];
    CC_TRY(batch_core_stash(&p->core, (size_t)p->vtx_off[p->G]));
    return batch_core_set(&p->core, b->d_row_ptr, b->d_col, b->d_labels, gr.data(), p->G,
                          nullptr, 1);
}

} // namespace

extern "C" int ccgpu_batch_plan_create(ccgpu_ctx *ctx, const ccgpu_batch *b,
                                       const ccgpu_batch_tuning *tuning, ccgpu_batch_plan **out)
{
    if (!b || !out || !b->h_vtx_off || !b->h_edge_off)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_plan_create: NULL argument");
    *out = nullptr;
    std::vector<BGraph> gr;
    CC_TRY(batch_descs(b, gr));
    ccgpu_batch_tuning t;
    if (tuning)
        t = *tuning;
    else
        ccgpu_batch_tuning_default(&t);
    CC_TRY(batch_check_tuning(&t));
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    ccgpu_batch_plan *p = new ccgpu_batch_plan();
    int rc = batch_core_init(&p->core, ctx, &t);
    if (rc == CCGPU_OK)
        rc = plan_set(p, b, t, gr);
    if (rc != CCGPU_OK) {
        ccgpu_batch_plan_destroy(p);
        return rc;
    }
    *out = p;
    return CCGPU_OK;
}

extern "C" int ccgpu_batch_plan_run(ccgpu_batch_plan *p, void *stream)
{
    if (!p)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_plan_run: NULL plan");
    return batch_core_enqueue(&p->core, (cudaStream_t)stream, nullptr);
}

extern "C" int ccgpu_batch_plan_launch(ccgpu_batch_plan *p, void *stream)
{
    if (!p)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_plan_launch: NULL plan");
    if (!p->exec)
        CC_TRY(capture(p));
    CC_CUDA(cudaGraphLaunch(p->exec, (cudaStream_t)stream));
    return CCGPU_OK;
}

extern "C" int ccgpu_batch_plan_kernels(const ccgpu_batch_plan *p)
{
    return p ? p->kernels : 0;
}

extern "C" int ccgpu_batch_plan_tuning(const ccgpu_batch_plan *p, ccgpu_batch_tuning *out)
{
    if (!p || !out)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_plan_tuning: NULL argument");
    *out = p->core.tune;
    return CCGPU_OK;
}

extern "C" int ccgpu_batch_plan_class_graphs(const ccgpu_batch_plan *p, uint32_t *counts)
{
    if (!p || !counts)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_plan_class_graphs: NULL argument");
    for (int c = 0; c < CCGPU_BATCH_CLASSES; ++c)
        counts[c] = (uint32_t)p->core.cls[c].graphs.size();
    return CCGPU_OK;
}

/* Coordinate descent per class over sampled neighbours, cadence, tile size
 * and the warp-row threshold, each candidate timed on the class alone. */
extern "C" int ccgpu_batch_plan_autotune(ccgpu_batch_plan *p, void *stream,
                                         ccgpu_batch_tuning *chosen)
{
    if (!p)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_plan_autotune: NULL plan");
    cudaStream_t st = (cudaStream_t)stream;
    BatchCore *c = &p->core;
    struct cc_prof *saved = c->ctx->prof;
    c->ctx->prof = nullptr;
    int rc = CCGPU_OK;
    for (int k = 0; k < CCGPU_BATCH_CLASSES && rc == CCGPU_OK; ++k) {
        BatchClass &C = c->cls[k];
        if (C.graphs.empty())
            continue;
        ccgpu_batch_class_opts best = C.o;
        float best_ms = 0.f;
        rc = time_class(c, k, st, 3, &best_ms);
        const int rounds[] = {0, 1, 2, 3};
        const int tiles[] = {1024, 4096, 16384};
        const int wdeg[] = {8, 16, 32, 64};
        for (int axis = 0; axis < 4 && rc == CCGPU_OK; ++axis) {
            const int nv = axis == 0 ? 4 : axis == 1 ? 2 : axis == 2 ? 3 : 4;
            for (int i = 0; i < nv && rc == CCGPU_OK; ++i) {
                ccgpu_batch_class_opts cand = best;
                if (axis == 0)
                    cand.sample_rounds = rounds[i];
                else if (axis == 1)
                    cand.cadence = i;
                else if (axis == 2)
                    cand.tile = tiles[i];
                else
                    cand.warp_degree = wdeg[i];
                if (!memcmp(&cand, &best, sizeof(cand)))
                    continue;
                const bool retile = cand.tile != C.o.tile;
                C.o = cand;
                if (retile)
                    rc = batch_core_retile(c, k);
                float ms = 0.f;
                if (rc == CCGPU_OK)
                    rc = time_class(c, k, st, 3, &ms);
                if (rc == CCGPU_OK && ms < best_ms) {
                    best_ms = ms;
                    best = cand;
                }
            }
        }
        const bool retile = best.tile != C.o.tile;
        C.o = best;
        if (rc == CCGPU_OK && retile)
            rc = batch_core_retile(c, k);
        c->tune.cls[k] = best;
    }
    c->ctx->prof = saved;
    drop_graph(p);
    if (rc == CCGPU_OK && chosen)
        *chosen = c->tune;
    return rc;
}

extern "C" int ccgpu_batch_plan_results(ccgpu_batch_plan *p, uint32_t *h_components,
                                        uint32_t *h_done, void *stream)
{
    if (!p)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_plan_results: NULL plan");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t gb = (size_t)p->G * sizeof(uint32_t);
    if (h_components)
        CC_CUDA(cudaMemcpyAsync(h_components, p->core.d_comps, gb, cudaMemcpyDeviceToHost, st));
    if (h_done)
        CC_CUDA(cudaMemcpyAsync(h_done, p->core.d_done, gb, cudaMemcpyDeviceToHost, st));
    int err = 0;
    if (p->core.tune.persistent)
        CC_CUDA(cudaMemcpyAsync(&err, p->core.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
    /* a graph without vertices has no tile: it is solved, with 0 components */
    for (uint32_t g = 0; h_done && g < p->G; ++g)
        if (p->vtx_off[g + 1] == p->vtx_off[g])
            h_done[g] = 1;
    if (err)
        return ccgpu_set_error(CCGPU_ERR_TIMEOUT,
                               "batch: a persistent launch gave up waiting for a graph's "
                               "previous phase (wait_ms %d)",
                               p->core.tune.wait_ms ? p->core.tune.wait_ms : 2000);
    return CCGPU_OK;
}

extern "C" void ccgpu_batch_plan_destroy(ccgpu_batch_plan *p)
{
    if (!p)
        return;
    drop_graph(p);
    batch_core_free(&p->core);
    delete p;
}

/* One-shot solve.  The context keeps the plan of its last call and points
 * it at the next batch, so repeated calls allocate only when a batch
 * outgrows what earlier ones needed (a context serves one host thread at a
 * time). */
extern "C" int ccgpu_batch_cc(ccgpu_ctx *ctx, const ccgpu_batch *b,
                              const ccgpu_batch_tuning *tuning, uint32_t *h_components,
                              void *stream)
{
    if (!b || !b->h_vtx_off || !b->h_edge_off)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_batch_cc: NULL argument");
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    ccgpu_batch_plan *p = ctx->batch_cache;
    if (p) {
        std::vector<BGraph> gr;
        CC_TRY(batch_descs(b, gr));
        ccgpu_batch_tuning t;
        if (tuning)
            t = *tuning;
        else
            ccgpu_batch_tuning_default(&t);
        CC_TRY(batch_check_tuning(&t));
        int rc = plan_set(p, b, t, gr);
        if (rc != CCGPU_OK) {
            ctx->batch_cache = nullptr;
            ccgpu_batch_plan_destroy(p);
            return rc;
        }
    } else {
        CC_TRY(ccgpu_batch_plan_create(ctx, b, tuning, &p));
        ctx->batch_cache = p;
    }
    int rc = ccgpu_batch_plan_run(p, stream);
    if (rc == CCGPU_OK)
        rc = ccgpu_batch_plan_results(p, h_components, nullptr, stream);
    else
        cudaStreamSynchronize((cudaStream_t)stream);
    return rc;
}

void cc_batch_cache_free(ccgpu_ctx *ctx)
{
    if (ctx && ctx->batch_cache) {
        ccgpu_batch_plan_destroy(ctx->batch_cache);
        ctx->batch_cache = nullptr;
    }
}
