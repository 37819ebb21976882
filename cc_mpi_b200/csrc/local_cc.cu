/*
 * Local connected components on a device-resident CSR (sm_100a).
 *
 * Replaces the reference's pthreads label propagation
 * (src/cc_pthreads.c:32-73 relax, :76-150 round loop, :152-229 driver),
 * whose result - each label is the minimum vertex id of its component - is
 * kept bit for bit.  The method is union-find hooking (the larger root is
 * CAS-hooked under a smaller vertex, so every root is its tree's minimum id)
 * with Afforest-style neighbour sampling (Sutton, Ben-Nun and Barak, IPDPS
 * 2018): after linking each vertex with its first few neighbours, the most
 * frequent root is found and the remaining rows of its tree are never read.
 * That skip is valid for symmetric graphs, the reference's input contract.
 * The optional first hook in the init pass follows ECL-CC's initialisation
 * (Jaiganesh and Burtscher, HPDC 2018).
 *
 * Kernels (256 threads):
 *   k_init       parent[v] = v, or v's first neighbour when smaller
 *   k_sample     thread per vertex, links row entries [r0, r1)
 *   k_compress   parent[v] = root(v)
 *   k_giant      one CTA per segment: most frequent root of 1024 samples
 *   k_link_rows  degree-binned finish pass: a CTA gathers short rows and
 *                walks them edge-parallel, a warp takes rows of >= 32 entries
 *                with 16-byte column loads, rows above the heavy threshold go
 *                to a queue
 *   k_link_heavy queued rows split in 512-entry pieces over every warp
 *   k_count_roots, k_check_labels   reductions for stats and tests
 */
#include <cstdio>
#include <cstring>

#include "local_cc.h"

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr uint32_t kNoGiant = 0xffffffffu;
constexpr int kGiantSamples = 1024;
constexpr uint64_t kHeavyPiece = 512; /* entries per warp piece of a queued row */

struct Rows {
    uint64_t beg, end;
};

/* Row v: [row_ptr[v], row_ptr[v+1]), or [row_ptr[v], row_end[v]) when the
 * rows are sub-ranges of the column array (row_end given). */
__device__ __forceinline__ Rows row_of(const uint64_t *__restrict__ row_ptr,
                                       const uint64_t *__restrict__ row_end, uint32_t v,
                                       uint64_t m)
{
    uint64_t b = __ldg(row_ptr + v), e = row_end ? __ldg(row_end + v) : __ldg(row_ptr + v + 1);
    if (e > m)
        e = m;
    if (b > e)
        b = e;
    return {b, e};
}

/* Index s with seg[s] <= v < seg[s+1] (seg ascending, nseg >= 1). */
__device__ __forceinline__ uint32_t seg_of(const uint64_t *__restrict__ seg, uint32_t nseg,
                                           uint64_t v)
{
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(seg + mid) <= v)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

/* [lo, hi) of v's segment when edges are filtered to segments, else [0, n). */
struct Span {
    uint32_t lo, hi;
};

__device__ __forceinline__ Span span_of(const uint64_t *__restrict__ fseg, uint32_t nseg,
                                        uint32_t n, uint64_t v)
{
    if (!fseg)
        return {0u, n};
    uint32_t s = seg_of(fseg, nseg, v);
    return {(uint32_t)__ldg(fseg + s), (uint32_t)__ldg(fseg + s + 1)};
}

__device__ __forceinline__ bool in_span(Span sp, uint32_t u)
{
    return u >= sp.lo && u < sp.hi;
}

__global__ void __launch_bounds__(kBlock) k_init(uint32_t *__restrict__ parent, uint32_t n,
                                                 LocalCCCounters *counters, int vec,
                                                 const uint64_t *__restrict__ row_ptr,
                                                 const uint64_t *__restrict__ row_end,
                                                 const uint32_t *__restrict__ col, uint64_t m,
                                                 int first_hook, const uint64_t *__restrict__ fseg,
                                                 uint32_t nseg)
{
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    const uint64_t tid = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (tid == 0)
        memset(counters, 0, sizeof(LocalCCCounters));
    if (first_hook) {
        /* parent[v] = first neighbour if it is smaller: v is still a root
         * and only this thread writes parent[v], so a plain store hooks it */
        for (uint64_t v = tid; v < n; v += stride) {
            Rows r = row_of(row_ptr, row_end, (uint32_t)v, m);
            uint32_t p = (uint32_t)v;
            if (r.beg < r.end) {
                uint32_t u = __ldg(col + r.beg);
                if (u < p && in_span(span_of(fseg, nseg, n, v), u))
                    p = u;
            }
            parent[v] = p;
        }
        return;
    }
    uint64_t done = 0;
    if (vec) {
        uint4 *p4 = reinterpret_cast<uint4 *>(parent);
        uint64_t nq = n / 4;
        for (uint64_t q = tid; q < nq; q += stride) {
            uint32_t b = (uint32_t)(q * 4);
            p4[q] = make_uint4(b, b + 1, b + 2, b + 3);
        }
        done = nq * 4;
    }
    for (uint64_t v = done + tid; v < n; v += stride)
        parent[v] = (uint32_t)v;
}

/* Links row entries [r0, r1) of every vertex in [v_lo, v_hi).  With the
 * first hook done by k_init, entry 0 is skipped when it was smaller. */
template <bool LAZY>
__global__ void __launch_bounds__(kBlock) k_sample(const uint64_t *__restrict__ row_ptr,
                                                   const uint64_t *__restrict__ row_end,
                                                   const uint32_t *__restrict__ col, uint32_t n,
                                                   uint64_t m, uint32_t *parent, uint32_t v_lo,
                                                   uint32_t v_hi, int r0, int r1, int first_done,
                                                   const uint64_t *__restrict__ fseg, uint32_t nseg)
{
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    for (uint64_t v = (uint64_t)v_lo + (uint64_t)blockIdx.x * kBlock + threadIdx.x; v < v_hi;
         v += stride) {
        Rows r = row_of(row_ptr, row_end, (uint32_t)v, m);
        const Span sp = span_of(fseg, nseg, n, v);
        for (int k = r0; k < r1; ++k) {
            uint64_t j = r.beg + (uint64_t)k;
            if (j >= r.end)
                break;
            uint32_t u = __ldg(col + j);
            if (!in_span(sp, u) || (k == 0 && first_done && u < (uint32_t)v))
                continue;
            cc_union<LAZY>(parent, (uint32_t)v, u);
        }
    }
}

/* Sampling that only has to leave a valid forest (MINHOOK): the larger of
 * the two roots is lowered to the smaller with a fire-and-forget atomicMin.
 * If that root was hooked elsewhere meanwhile, its subtree moves to the new
 * parent and one earlier link is lost; the forest stays valid (parent < self,
 * every link inside one component) and the finish pass re-links every row
 * outside the giant tree from its first entry, which restores anything
 * lost. */
__global__ void __launch_bounds__(kBlock) k_sample_min(const uint64_t *__restrict__ row_ptr,
                                                       const uint64_t *__restrict__ row_end,
                                                       const uint32_t *__restrict__ col,
                                                       uint32_t n, uint64_t m, uint32_t *parent,
                                                       uint32_t v_lo, uint32_t v_hi, int r0,
                                                       int r1, const uint64_t *__restrict__ fseg,
                                                       uint32_t nseg)
{
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    for (uint64_t v = (uint64_t)v_lo + (uint64_t)blockIdx.x * kBlock + threadIdx.x; v < v_hi;
         v += stride) {
        Rows r = row_of(row_ptr, row_end, (uint32_t)v, m);
        const Span sp = span_of(fseg, nseg, n, v);
        for (int k = r0; k < r1; ++k) {
            uint64_t j = r.beg + (uint64_t)k;
            if (j >= r.end)
                break;
            uint32_t u = __ldg(col + j);
            if (!in_span(sp, u))
                continue;
            uint32_t rv = cc_find(parent, (uint32_t)v), ru = cc_find(parent, u);
            if (rv != ru)
                atomicMin(parent + (rv > ru ? rv : ru), rv < ru ? rv : ru);
        }
    }
}

/* k_sample_min for rounds 0 and 1 with a stash of each vertex's second
 * neighbour: round 0 reads entries 0 and 1 of the row (one column sector)
 * and keeps entry 1 in stash[v]; round 1 links v with stash[v] without
 * touching the row.  UINT32_MAX in the stash means no second entry. */
__global__ void __launch_bounds__(kBlock) k_sample_stash(const uint64_t *__restrict__ row_ptr,
                                                         const uint64_t *__restrict__ row_end,
                                                         const uint32_t *__restrict__ col,
                                                         uint32_t n, uint64_t m,
                                                         uint32_t *parent, uint32_t *stash,
                                                         int round)
{
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    for (uint64_t v = (uint64_t)blockIdx.x * kBlock + threadIdx.x; v < n; v += stride) {
        uint32_t u;
        if (round == 0) {
            Rows r = row_of(row_ptr, row_end, (uint32_t)v, m);
            u = r.beg < r.end ? __ldg(col + r.beg) : 0xffffffffu;
            stash[v] = r.beg + 1 < r.end ? __ldg(col + r.beg + 1) : 0xffffffffu;
        } else {
            u = stash[v];
        }
        if (u >= n)
            continue;
        uint32_t rv = cc_find(parent, (uint32_t)v), ru = cc_find(parent, u);
        if (rv != ru)
            atomicMin(parent + (rv > ru ? rv : ru), rv < ru ? rv : ru);
    }
}

__global__ void __launch_bounds__(kBlock) k_compress(uint32_t *parent, uint32_t n)
{
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    for (uint64_t v = (uint64_t)blockIdx.x * kBlock + threadIdx.x; v < n; v += stride) {
        uint32_t r = cc_find(parent, (uint32_t)v);
        if (r != (uint32_t)v)
            parent[v] = r;
    }
}

/* Most frequent root among kGiantSamples seeded samples of segment
 * blockIdx.x.  Ties go to the smaller root, so the choice is deterministic
 * for a given forest. */
__global__ void __launch_bounds__(kGiantSamples) k_giant(const uint32_t *parent, uint32_t n,
                                                         const uint64_t *seg, uint32_t seed,
                                                         uint32_t *out)
{
    __shared__ uint32_t s[kGiantSamples];
    __shared__ unsigned long long s_best[kGiantSamples / 32];
    const uint32_t i = threadIdx.x;
    uint64_t lo = seg ? seg[blockIdx.x] : 0, hi = seg ? seg[blockIdx.x + 1] : n;
    if (hi <= lo) {
        if (i == 0)
            out[blockIdx.x] = kNoGiant;
        return;
    }
    uint64_t size = hi - lo;
    uint32_t h = cc_mix32(i * 0x9e3779b9u + seed + blockIdx.x);
    uint32_t v = (uint32_t)(lo + (((uint64_t)h * size) >> 32));
    uint32_t mode = cc_block_mode1024(cc_find_ro(parent, v), s, s_best);
    if (i == 0)
        out[blockIdx.x] = mode;
}

struct LinkParams {
    const uint64_t *row_ptr;
    const uint64_t *row_end;   /* NULL, or the end of each row (row_of) */
    const uint32_t *col;
    uint32_t n;
    uint64_t m;
    uint32_t *parent;
    uint32_t skip_from;        /* first row entry the finish pass links   */
    const uint32_t *giants;    /* [nseg] giant roots, NULL = no skipping   */
    const uint64_t *seg;       /* segment offsets or NULL                  */
    uint32_t nseg;
    uint32_t chunk;            /* vertices per work grab, 0 = static       */
    LocalCCCounters *cnt;
    uint32_t *heavy_list;
    uint32_t heavy_cap;
    uint32_t heavy_deg;
    int vec;                   /* col is 16-byte aligned                    */
    const uint64_t *fseg;      /* segment filter offsets, NULL = off        */
};

/* One warp links v with row entries [beg, end) that fall in sp: 16-byte
 * column loads for the aligned body, scalar loads for head and tail, every
 * step taken by all 32 lanes together. */
template <bool LAZY>
__device__ __forceinline__ void warp_link_row(const LinkParams &P, uint32_t v, uint64_t beg,
                                              uint64_t end, int lane, Span sp)
{
    uint64_t a = beg, body_end = beg;
    if (P.vec) {
        a = (beg + 3) & ~3ull;
        if (a > end)
            a = end;
        body_end = end & ~3ull;
        if (body_end < a)
            body_end = a;
    }
    /* scalar entries: [beg, a) and [body_end, end) */
    const uint64_t head = a - beg, scalars = head + (end - body_end);
    for (uint64_t s0 = 0; s0 < scalars; s0 += 32) {
        uint64_t s = s0 + lane;
        uint32_t u[1] = {0};
        bool ok[1] = {false};
        if (s < scalars) {
            u[0] = __ldg(P.col + (s < head ? beg + s : body_end + (s - head)));
            ok[0] = in_span(sp, u[0]);
        }
        cc_warp_link_min_first<1>(P.parent, v, u, ok, lane);
    }
    const uint4 *c4 = reinterpret_cast<const uint4 *>(P.col);
    for (uint64_t q0 = a / 4; q0 < body_end / 4; q0 += 32) {
        uint64_t q = q0 + lane;
        uint32_t u[4] = {0, 0, 0, 0};
        bool ok[4] = {false, false, false, false};
        if (q < body_end / 4) {
            uint4 x = __ldg(c4 + q);
            u[0] = x.x;
            u[1] = x.y;
            u[2] = x.z;
            u[3] = x.w;
#pragma unroll
            for (int i = 0; i < 4; ++i)
                ok[i] = in_span(sp, u[i]);
        }
        cc_warp_link_min_first<4>(P.parent, v, u, ok, lane);
    }
}

/* Vertices a thread takes per step of the finish pass: consecutive, so a
 * step covers kBlock * kVPT vertices and its barriers are paid once per
 * kVPT vertices per thread. */
constexpr int kVPT = 4;
constexpr int kStep = kBlock * kVPT;

template <bool LAZY>
__global__ void __launch_bounds__(kBlock, 4) k_link_rows(LinkParams P)
{
    __shared__ uint32_t s_off[kStep + 1];
    __shared__ uint64_t s_beg[kStep];
    __shared__ uint32_t s_wsum[kWarps];
    __shared__ Span s_span[kStep];
    __shared__ unsigned long long s_base;

    const uint32_t giant0 = (P.giants && P.nseg == 1) ? P.giants[0] : kNoGiant;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t my_rows = 0;
    unsigned long long my_edges = 0;

    uint64_t st_lo = 0, st_hi = 0;
    if (P.chunk == 0) {
        uint64_t per = ((uint64_t)P.n + gridDim.x - 1) / gridDim.x;
        per = (per + kStep - 1) / kStep * kStep;
        st_lo = per * blockIdx.x;
        st_hi = st_lo + per;
        if (st_lo > P.n)
            st_lo = P.n;
        if (st_hi > P.n)
            st_hi = P.n;
    }

    for (int iter = 0;; ++iter) {
        uint64_t base, cend;
        if (P.chunk) {
            if (threadIdx.x == 0)
                s_base = atomicAdd(&P.cnt->grab, (unsigned long long)P.chunk);
            __syncthreads();
            base = s_base;
            __syncthreads();
            if (base >= P.n)
                break;
            cend = base + P.chunk;
            if (cend > P.n)
                cend = P.n;
        } else {
            if (iter > 0 || st_lo >= st_hi)
                break;
            base = st_lo;
            cend = st_hi;
        }
        for (uint64_t t0 = base; t0 < cend; t0 += kStep) {
            /* this thread's kVPT consecutive vertices: slots kVPT*t + k */
            uint64_t beg[kVPT], end[kVPT];
            uint32_t small[kVPT];
            uint32_t mine = 0;
#pragma unroll
            for (int k = 0; k < kVPT; ++k) {
                const uint64_t v64 = t0 + (uint64_t)threadIdx.x * kVPT + k;
                const uint32_t v = (uint32_t)v64;
                beg[k] = end[k] = 0;
                const Span sp = span_of(P.fseg, P.nseg, P.n, v64 < cend ? v64 : t0);
                if (v64 < cend) {
                    uint32_t giant = giant0;
                    if (P.giants && P.nseg > 1)
                        giant = P.giants[seg_of(P.seg, P.nseg, v64)];
                    if (giant == kNoGiant || cc_ldp(P.parent, v) != giant) {
                        Rows r = row_of(P.row_ptr, P.row_end, v, P.m);
                        beg[k] = r.beg + P.skip_from;
                        end[k] = r.end;
                        if (beg[k] > end[k])
                            beg[k] = end[k];
                        my_rows++;
                        my_edges += end[k] - beg[k];
                    }
                }
                uint64_t deg = end[k] - beg[k];
                if (deg > P.heavy_deg) {
                    uint32_t slot = atomicAdd(&P.cnt->heavy_count, 1u);
                    if (slot < P.heavy_cap) {
                        P.heavy_list[slot] = v;
                        deg = 0;
                        end[k] = beg[k];
                    }
                }
                /* warp-cooperative rows */
                unsigned big = __ballot_sync(0xffffffffu, deg >= 32);
                while (big) {
                    int src = __ffs(big) - 1;
                    big &= big - 1;
                    uint32_t vv = __shfl_sync(0xffffffffu, v, src);
                    uint64_t bb = __shfl_sync(0xffffffffu, beg[k], src);
                    uint64_t ee = __shfl_sync(0xffffffffu, end[k], src);
                    Span ss = {__shfl_sync(0xffffffffu, sp.lo, src),
                               __shfl_sync(0xffffffffu, sp.hi, src)};
                    warp_link_row<LAZY>(P, vv, bb, ee, lane, ss);
                }
                small[k] = deg < 32 ? (uint32_t)deg : 0u;
                mine += small[k];
                s_beg[threadIdx.x * kVPT + k] = beg[k];
                s_span[threadIdx.x * kVPT + k] = sp;
            }
            /* short rows: CTA-wide gather over the step's slots, walked
             * edge-parallel */
            uint32_t incl = mine;
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o)
                    incl += y;
            }
            if (lane == 31)
                s_wsum[warp] = incl;
            __syncthreads();
            uint32_t wpre = 0, total = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                uint32_t x = s_wsum[w];
                wpre += (w < warp) ? x : 0u;
                total += x;
            }
            uint32_t run = wpre + incl - mine;
#pragma unroll
            for (int k = 0; k < kVPT; ++k) {
                s_off[threadIdx.x * kVPT + k] = run;
                run += small[k];
            }
            if (threadIdx.x == 0)
                s_off[kStep] = total;
            __syncthreads();
            for (uint32_t e = threadIdx.x; e < total; e += kBlock) {
                int lo = 0, hi = kStep;
                while (hi - lo > 1) {
                    int mid = (lo + hi) >> 1;
                    if (s_off[mid] <= e)
                        lo = mid;
                    else
                        hi = mid;
                }
                uint64_t j = s_beg[lo] + (e - s_off[lo]);
                uint32_t u = __ldg(P.col + j);
                if (in_span(s_span[lo], u))
                    cc_union<LAZY>(P.parent, (uint32_t)(t0 + lo), u);
            }
            __syncthreads();
        }
    }
    unsigned long long rows = my_rows;
    for (int o = 16; o > 0; o >>= 1) {
        rows += __shfl_xor_sync(0xffffffffu, rows, o);
        my_edges += __shfl_xor_sync(0xffffffffu, my_edges, o);
    }
    if (lane == 0 && rows) {
        atomicAdd(&P.cnt->finish_rows, rows);
        atomicAdd(&P.cnt->finish_edges, my_edges);
    }
}

/* Queued rows in pieces of kHeavyPiece entries spread over every warp of
 * the grid (piece g of the list goes to warp g mod all warps), each piece
 * linked min-first like the warp rows. */
template <bool LAZY>
__global__ void __launch_bounds__(kBlock) k_link_heavy(LinkParams P)
{
    uint32_t cnt = P.cnt->heavy_count;
    if (cnt > P.heavy_cap)
        cnt = P.heavy_cap;
    const int lane = threadIdx.x & 31;
    cc_for_heavy_pieces(P.heavy_list, cnt, P.row_ptr, P.row_end, P.m, P.skip_from, kHeavyPiece,
                        [&](uint32_t v, uint64_t jb, uint64_t je) {
                            const Span sp = span_of(P.fseg, P.nseg, P.n, v);
                            for (uint64_t j0 = jb; j0 < je; j0 += 32) {
                                uint64_t j = j0 + lane;
                                uint32_t u[1] = {0};
                                bool ok[1] = {false};
                                if (j < je) {
                                    u[0] = __ldg(P.col + j);
                                    ok[0] = in_span(sp, u[0]);
                                }
                                cc_warp_link_min_first<1>(P.parent, v, u, ok, lane);
                            }
                        });
}

__global__ void __launch_bounds__(kBlock) k_count_roots(const uint32_t *__restrict__ labels,
                                                        uint32_t n, unsigned long long *out)
{
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    uint32_t c = 0;
    for (uint64_t v = (uint64_t)blockIdx.x * kBlock + threadIdx.x; v < n; v += stride)
        c += (__ldg(labels + v) == (uint32_t)v);
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c)
        atomicAdd(out, (unsigned long long)c);
}

__global__ void __launch_bounds__(kBlock) k_check_labels(const uint64_t *__restrict__ row_ptr,
                                                         const uint32_t *__restrict__ col,
                                                         uint32_t n, uint64_t m,
                                                         const uint32_t *__restrict__ L,
                                                         unsigned long long *bad)
{
    /* warp per vertex so that hub rows do not serialise one thread */
    const int lane = threadIdx.x & 31;
    const uint64_t wstride = (uint64_t)gridDim.x * kWarps;
    uint32_t local_bad = 0;
    for (uint64_t v = (uint64_t)blockIdx.x * kWarps + (threadIdx.x >> 5); v < n; v += wstride) {
        uint32_t lv = __ldg(L + v);
        if (lane == 0) {
            if (lv > v || lv >= n)
                local_bad++;
            else if (__ldg(L + lv) != lv)
                local_bad++;
        }
        Rows r = row_of(row_ptr, nullptr, (uint32_t)v, m);
        for (uint64_t j = r.beg + lane; j < r.end; j += 32) {
            uint32_t u = __ldg(col + j);
            if (u < n && __ldg(L + u) != lv)
                local_bad++;
        }
    }
    local_bad = __reduce_add_sync(0xffffffffu, local_bad);
    if (lane == 0 && local_bad)
        atomicAdd(bad, (unsigned long long)local_bad);
}

struct Geometry {
    unsigned stream_blocks; /* grid for the streaming kernels      */
    unsigned link_blocks;   /* resident grid for k_link_rows        */
};

int geometry(const ccgpu_ctx *ctx, Geometry *g)
{
    static thread_local int occ_rows = 0;
    if (!occ_rows) {
        CC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_rows, k_link_rows<false>,
                                                              kBlock, 0));
        if (occ_rows < 1)
            occ_rows = 1;
    }
    g->stream_blocks = (unsigned)ctx->sm_count * 8;
    g->link_blocks = (unsigned)ctx->sm_count * (unsigned)occ_rows;
    return CCGPU_OK;
}

template <bool LAZY>
int launch_sample(ccgpu_ctx *ctx, const LocalCCArgs &a, uint32_t vlo, uint32_t vhi, int r0,
                  int r1, cudaStream_t st, unsigned blocks)
{
    const int first_done = (a.o.hook_mode & CCGPU_HOOK_FIRST) != 0;
    const uint64_t *fseg = a.seg_filter ? a.seg : nullptr;
    CC_KLAUNCH(ctx, CCK_SAMPLE, k_sample<LAZY>, blocks, kBlock, 0, st, a.row_ptr, a.row_end, a.col, a.n,
               a.m, a.labels, vlo, vhi, r0, r1, first_done, fseg, a.nseg);
    return CCGPU_OK;
}

/* Step 1 over [vlo, vhi) for row entries [r0, r1), in the kernel the hook
 * mode asks for. */
int launch_sample_any(ccgpu_ctx *ctx, const LocalCCArgs &a, uint32_t vlo, uint32_t vhi, int r0,
                      int r1, cudaStream_t st, unsigned blocks)
{
    if (a.o.hook_mode & CCGPU_HOOK_MINHOOK) {
        const uint64_t *fseg = a.seg_filter ? a.seg : nullptr;
        CC_KLAUNCH(ctx, CCK_SAMPLE, k_sample_min, blocks, kBlock, 0, st, a.row_ptr, a.row_end, a.col, a.n,
                   a.m, a.labels, vlo, vhi, r0, r1, fseg, a.nseg);
        return CCGPU_OK;
    }
    if (a.o.hook_mode & CCGPU_HOOK_LAZY)
        return launch_sample<true>(ctx, a, vlo, vhi, r0, r1, st, blocks);
    return launch_sample<false>(ctx, a, vlo, vhi, r0, r1, st, blocks);
}

template <bool LAZY>
int launch_finish(ccgpu_ctx *ctx, const LinkParams &P, const Geometry &g, cudaStream_t st)
{
    CC_KLAUNCH(ctx, CCK_LINK_ROWS, k_link_rows<LAZY>, g.link_blocks, kBlock, 0, st, P);
    CC_KLAUNCH(ctx, CCK_LINK_HEAVY, k_link_heavy<LAZY>, g.link_blocks, kBlock, 0, st, P);
    return CCGPU_OK;
}

} // namespace

/* ------------------------------------------------------ internal entry */

int cc_local_resolve_opts(const ccgpu_cc_opts *in, ccgpu_cc_opts *o)
{
    ccgpu_cc_opts_default(o);
    if (in) {
        *o = *in;
        if (o->sample_rounds < 0)
            o->sample_rounds = 2;
        if (o->heavy_degree <= 0)
            o->heavy_degree = 8192;
        if (o->chunk_size <= 0)
            o->chunk_size = 4096;
        if (o->hook_mode < 0)
            o->hook_mode = CCGPU_HOOK_CADENCE | CCGPU_HOOK_MINHOOK;
    }
    if (o->sample_rounds > 8)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "sample_rounds %d above 8", o->sample_rounds);
    if (o->hook_mode > 15)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "hook_mode %d is not a mask of 1|2|4|8",
                               o->hook_mode);
    if (o->heavy_degree < 32)
        o->heavy_degree = 32;
    return CCGPU_OK;
}

void cc_local_carve(cc_carve *c, LocalCCScratch *s, const LocalCCArgs &a)
{
    uint64_t cap = a.m / (uint64_t)(a.o.heavy_degree > 0 ? a.o.heavy_degree : 1) + 1;
    if (cap > a.n)
        cap = a.n;
    if (cap == 0)
        cap = 1;
    s->counters = (LocalCCCounters *)cc_take(c, sizeof(LocalCCCounters));
    s->giants = (uint32_t *)cc_take(c, (size_t)(a.nseg ? a.nseg : 1) * sizeof(uint32_t));
    s->heavy_list = (uint32_t *)cc_take(c, cap * sizeof(uint32_t));
    s->heavy_cap = (uint32_t)cap;
    s->stash = a.stash ? (uint32_t *)cc_take(c, (size_t)a.n * sizeof(uint32_t)) : nullptr;
}

int cc_local_init(ccgpu_ctx *ctx, const LocalCCArgs &a, const LocalCCScratch &s, cudaStream_t st)
{
    Geometry g = {1, 1};
    CC_TRY(geometry(ctx, &g));
    const unsigned sb = cc_blocks(a.n, kBlock, g.stream_blocks);
    const int first = (a.o.hook_mode & CCGPU_HOOK_FIRST) && a.o.sample_rounds > 0;
    CC_KLAUNCH(ctx, CCK_INIT, k_init, sb, kBlock, 0, st, a.labels, a.n, s.counters,
               ((uintptr_t)a.labels & 15) == 0, a.row_ptr, a.row_end, a.col, a.m, first,
               a.seg_filter ? a.seg : (const uint64_t *)nullptr, a.nseg);
    return CCGPU_OK;
}

int cc_local_sample_range(ccgpu_ctx *ctx, const LocalCCArgs &a, uint32_t v_lo, uint32_t v_hi,
                          cudaStream_t st)
{
    if (a.o.sample_rounds <= 0 || v_hi <= v_lo)
        return CCGPU_OK;
    Geometry g = {1, 1};
    CC_TRY(geometry(ctx, &g));
    const unsigned sb = cc_blocks(v_hi - v_lo, kBlock, g.stream_blocks);
    return launch_sample_any(ctx, a, v_lo, v_hi, 0, a.o.sample_rounds, st, sb);
}

int cc_local_run(ccgpu_ctx *ctx, const LocalCCArgs &a, const LocalCCScratch &s, cudaStream_t st,
                 int init_done, int sampled)
{
    if (a.n == 0)
        return CCGPU_OK;
    Geometry g = {1, 1};
    CC_TRY(geometry(ctx, &g));
    const unsigned sb = cc_blocks(a.n, kBlock, g.stream_blocks);
    const bool lazy = (a.o.hook_mode & CCGPU_HOOK_LAZY) != 0;
    const int k = a.o.sample_rounds;
    if (!init_done)
        CC_TRY(cc_local_init(ctx, a, s, st));
    const bool skip = k > 0 && a.o.skip_giant;
    const bool minhook = (a.o.hook_mode & CCGPU_HOOK_MINHOOK) != 0;
    if (k > 0) {
        if (!sampled) {
            /* with MINHOOK the finish pass relinks entry 0, so the init
             * pass's first hook is all round 0 needs */
            const int r_start = (minhook && (a.o.hook_mode & CCGPU_HOOK_FIRST)) ? 1 : 0;
            /* rounds 0 and 1 through the stash when the scratch has one and
             * rows are long enough (>= 8 entries per vertex on average) for
             * the saved column gathers to outweigh the stash traffic */
            const bool use_stash = s.stash && minhook && !a.seg_filter && r_start == 0 &&
                                   k >= 2 && a.m >= 8ull * a.n;
            if (a.o.hook_mode & CCGPU_HOOK_CADENCE) {
                if (r_start > 0 && r_start < k)
                    CC_KLAUNCH(ctx, CCK_COMPRESS, k_compress, sb, kBlock, 0, st, a.labels, a.n);
                for (int r = r_start; r < k; ++r) {
                    if (use_stash && r < 2)
                        CC_KLAUNCH(ctx, CCK_SAMPLE, k_sample_stash, sb, kBlock, 0, st, a.row_ptr,
                                   a.row_end, a.col, a.n, a.m, a.labels, s.stash, r);
                    else
                        CC_TRY(launch_sample_any(ctx, a, 0, a.n, r, r + 1, st, sb));
                    if (r + 1 < k)
                        CC_KLAUNCH(ctx, CCK_COMPRESS, k_compress, sb, kBlock, 0, st, a.labels,
                                   a.n);
                }
            } else if (r_start < k) {
                CC_TRY(launch_sample_any(ctx, a, 0, a.n, r_start, k, st, sb));
            }
        }
        if (skip) {
            CC_KLAUNCH(ctx, CCK_COMPRESS, k_compress, sb, kBlock, 0, st, a.labels, a.n);
            CC_KLAUNCH(ctx, CCK_GIANT, k_giant, a.nseg, kGiantSamples, 0, st, a.labels, a.n,
                       a.seg, 0x5eed1234u, s.giants);
        }
    }
    LinkParams P;
    P.row_ptr = a.row_ptr;
    P.row_end = a.row_end;
    P.col = a.col;
    P.n = a.n;
    P.m = a.m;
    P.parent = a.labels;
    P.skip_from = minhook ? 0u : (uint32_t)k;
    P.giants = skip ? s.giants : nullptr;
    P.seg = a.seg;
    P.nseg = a.seg ? a.nseg : 1;
    P.chunk = a.o.chunk_size == 1 ? 0u : (uint32_t)a.o.chunk_size;
    P.cnt = s.counters;
    P.heavy_list = s.heavy_list;
    P.heavy_cap = s.heavy_cap;
    P.heavy_deg = (uint32_t)a.o.heavy_degree;
    P.vec = ((uintptr_t)a.col & 15) == 0;
    P.fseg = a.seg_filter ? a.seg : nullptr;
    if (lazy)
        CC_TRY(launch_finish<true>(ctx, P, g, st));
    else
        CC_TRY(launch_finish<false>(ctx, P, g, st));
    CC_KLAUNCH(ctx, CCK_FINAL_COMPRESS, k_compress, sb, kBlock, 0, st, a.labels, a.n);
    return CCGPU_OK;
}

/* ------------------------------------------------------------------ API */

extern "C" void ccgpu_cc_opts_default(ccgpu_cc_opts *o)
{
    if (!o)
        return;
    o->chunk_size = 4096;
    o->sample_rounds = 2;
    o->heavy_degree = 8192;
    o->skip_giant = 1;
    o->hook_mode = CCGPU_HOOK_CADENCE | CCGPU_HOOK_MINHOOK;
}

static int fill_stats(ccgpu_ctx *ctx, const LocalCCArgs &a, const LocalCCScratch &s,
                      uint32_t kernels, ccgpu_cc_stats *stats, cudaStream_t st)
{
    uint64_t roots = 0;
    CC_TRY(ccgpu_count_roots(ctx, a.labels, a.n, &roots, st));
    LocalCCCounters h;
    uint32_t giant = 0xffffffffu;
    CC_CUDA(cudaMemcpyAsync(&h, s.counters, sizeof(h), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaMemcpyAsync(&giant, s.giants, sizeof(giant), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
    stats->heavy_rows = h.heavy_count < s.heavy_cap ? h.heavy_count : s.heavy_cap;
    stats->giant_label = (a.o.sample_rounds > 0 && a.o.skip_giant) ? giant : 0xffffffffu;
    stats->components = (uint32_t)roots;
    stats->kernels = kernels + 1;
    stats->finish_rows = h.finish_rows;
    stats->finish_edges = h.finish_edges;
    return CCGPU_OK;
}

static int check_csr_args(const uint64_t *row_ptr, const uint32_t *col, uint32_t n, uint64_t m,
                          const uint32_t *labels, const char *who)
{
    if (n == 0)
        return CCGPU_OK;
    if (!row_ptr || !labels || (m > 0 && !col))
        return ccgpu_set_error(CCGPU_ERR_INVALID, "%s: NULL row_ptr/col_idx/labels", who);
    if (n == 0xffffffffu)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "%s: n must be below 2^32-1", who);
    return CCGPU_OK;
}

extern "C" int ccgpu_local_cc(ccgpu_ctx *ctx, const uint64_t *d_row_ptr, const uint32_t *d_col_idx,
                              uint32_t n, uint64_t m, uint32_t *d_labels,
                              const ccgpu_cc_opts *opts, ccgpu_cc_stats *stats, void *stream)
{
    CC_TRY(check_csr_args(d_row_ptr, d_col_idx, n, m, d_labels, "ccgpu_local_cc"));
    if (stats)
        memset(stats, 0, sizeof(*stats));
    if (n == 0)
        return CCGPU_OK;
    LocalCCArgs a = {d_row_ptr, d_col_idx, n, m, d_labels, nullptr, 1, {}, 0, 1};
    CC_TRY(cc_local_resolve_opts(opts, &a.o));
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = (cudaStream_t)stream;
    LocalCCScratch s;
    cc_carve c = {nullptr, 0};
    cc_local_carve(&c, &s, a);
    void *base = nullptr;
    CC_TRY(ccgpu_ctx_reserve(ctx, c.off, &base));
    c = {(char *)base, 0};
    cc_local_carve(&c, &s, a);
    const unsigned long long before = ctx->launches;
    CC_TRY(cc_local_run(ctx, a, s, st, 0, 0));
    if (stats)
        CC_TRY(fill_stats(ctx, a, s, (uint32_t)(ctx->launches - before), stats, st));
    return CCGPU_OK;
}

/* Host-buffer variant.  Device copies of the CSR and the labels live in
 * the context's scratch.  Column chunks are copied on a second stream and,
 * when the init pass needs no columns, each chunk's vertex range is sampled
 * as soon as its columns landed. */
extern "C" int ccgpu_local_cc_host(ccgpu_ctx *ctx, const uint64_t *h_row_ptr,
                                   const uint32_t *h_col_idx, uint32_t n, uint64_t m,
                                   uint32_t *h_labels, const ccgpu_cc_opts *opts,
                                   ccgpu_cc_stats *stats)
{
    CC_TRY(check_csr_args(h_row_ptr, h_col_idx, n, m, h_labels, "ccgpu_local_cc_host"));
    if (stats)
        memset(stats, 0, sizeof(*stats));
    if (n == 0)
        return CCGPU_OK;
    if (h_row_ptr[n] != m)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_local_cc_host: row_ptr[n]=%llu != m=%llu",
                               (unsigned long long)h_row_ptr[n], (unsigned long long)m);
    LocalCCArgs a = {nullptr, nullptr, n, m, nullptr, nullptr, 1, {}};
    CC_TRY(cc_local_resolve_opts(opts, &a.o));
    CC_TRY(ccgpu_ctx_resolve(&ctx));

    LocalCCScratch s;
    uint64_t *d_row = nullptr;
    uint32_t *d_col = nullptr, *d_lab = nullptr;
    void *base = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
        cc_carve c = {(char *)base, 0};
        cc_local_carve(&c, &s, a);
        d_row = (uint64_t *)cc_take(&c, ((size_t)n + 1) * sizeof(uint64_t));
        d_col = (uint32_t *)cc_take(&c, (size_t)(m ? m : 1) * sizeof(uint32_t));
        d_lab = (uint32_t *)cc_take(&c, (size_t)n * sizeof(uint32_t));
        if (pass == 0)
            CC_TRY(ccgpu_ctx_reserve(ctx, c.off, &base));
    }
    a.row_ptr = d_row;
    a.col = d_col;
    a.labels = d_lab;

    cudaStream_t st = nullptr, cp = nullptr;
    int rc = CCGPU_OK;
    const int kPieces = 8;
    cudaEvent_t ev[kPieces] = {};
    const unsigned long long before = ctx->launches;
    /* the init pass reads first neighbours when the first hook is on, so
     * it then waits for all columns; otherwise sampling overlaps the copy */
    const bool init_reads_cols = (a.o.hook_mode & CCGPU_HOOK_FIRST) && a.o.sample_rounds > 0;
#define HOST_TRY(call)                                                         \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            rc = ccgpu_cuda_fail(e_, #call, __FILE__, __LINE__);               \
            goto done;                                                         \
        }                                                                      \
    } while (0)
#define HOST_ST(call)                                                          \
    do {                                                                       \
        rc = (call);                                                           \
        if (rc != CCGPU_OK)                                                    \
            goto done;                                                         \
    } while (0)
    HOST_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    HOST_TRY(cudaStreamCreateWithFlags(&cp, cudaStreamNonBlocking));
    for (int i = 0; i < kPieces; ++i)
        HOST_TRY(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    HOST_TRY(cudaMemcpyAsync(d_row, h_row_ptr, ((size_t)n + 1) * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, st));
    if (!init_reads_cols)
        HOST_ST(cc_local_init(ctx, a, s, st));
    HOST_TRY(cudaEventRecord(ev[0], st));
    HOST_TRY(cudaStreamWaitEvent(cp, ev[0], 0));
    for (int i = 0; i < kPieces; ++i) {
        uint32_t vlo = (uint32_t)((uint64_t)n * i / kPieces);
        uint32_t vhi = (uint32_t)((uint64_t)n * (i + 1) / kPieces);
        uint64_t elo = h_row_ptr[vlo], ehi = h_row_ptr[vhi];
        if (ehi > elo)
            HOST_TRY(cudaMemcpyAsync(d_col + elo, h_col_idx + elo, (ehi - elo) * sizeof(uint32_t),
                                     cudaMemcpyHostToDevice, cp));
        HOST_TRY(cudaEventRecord(ev[i], cp));
        if (!init_reads_cols) {
            HOST_TRY(cudaStreamWaitEvent(st, ev[i], 0));
            HOST_ST(cc_local_sample_range(ctx, a, vlo, vhi, st));
        }
    }
    HOST_TRY(cudaStreamWaitEvent(st, ev[kPieces - 1], 0));
    if (init_reads_cols)
        HOST_ST(cc_local_run(ctx, a, s, st, 0, 0));
    else
        HOST_ST(cc_local_run(ctx, a, s, st, 1, 1));
    HOST_TRY(cudaMemcpyAsync(h_labels, d_lab, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             st));
    if (stats)
        HOST_ST(fill_stats(ctx, a, s, (uint32_t)(ctx->launches - before), stats, st));
    HOST_TRY(cudaStreamSynchronize(st));
done:
#undef HOST_TRY
#undef HOST_ST
    if (rc != CCGPU_OK && st)
        cudaStreamSynchronize(st);
    if (rc != CCGPU_OK && cp)
        cudaStreamSynchronize(cp);
    for (int i = 0; i < kPieces; ++i)
        if (ev[i])
            cudaEventDestroy(ev[i]);
    if (cp)
        cudaStreamDestroy(cp);
    if (st)
        cudaStreamDestroy(st);
    return rc;
}

extern "C" int ccgpu_count_roots(ccgpu_ctx *ctx, const uint32_t *d_labels, uint32_t n,
                                 uint64_t *count, void *stream)
{
    if (!count || (n && !d_labels))
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_count_roots: NULL argument");
    *count = 0;
    if (n == 0)
        return CCGPU_OK;
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = (cudaStream_t)stream;
    void *host = nullptr;
    CC_TRY(ccgpu_ctx_pinned(ctx, 64, &host));
    unsigned long long *cell = nullptr;
    CC_TRY(ccgpu_ctx_cell(ctx, &cell));
    CC_CUDA(cudaMemsetAsync(cell, 0, sizeof(unsigned long long), st));
    CC_KLAUNCH(ctx, CCK_COUNT_ROOTS, k_count_roots,
               cc_blocks(n, kBlock, (unsigned)ctx->sm_count * 8), kBlock, 0, st, d_labels, n,
               cell);
    CC_CUDA(cudaMemcpyAsync(host, cell, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
    *count = *(unsigned long long *)host;
    return CCGPU_OK;
}

extern "C" int ccgpu_check_labels(ccgpu_ctx *ctx, const uint64_t *d_row_ptr,
                                  const uint32_t *d_col_idx, uint32_t n, uint64_t m,
                                  const uint32_t *d_labels, uint64_t *violations, void *stream)
{
    if (!violations)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_check_labels: violations is NULL");
    CC_TRY(check_csr_args(d_row_ptr, d_col_idx, n, m, d_labels, "ccgpu_check_labels"));
    *violations = 0;
    if (n == 0)
        return CCGPU_OK;
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long *d_bad = nullptr;
    CC_TRY(ccgpu_ctx_cell(ctx, &d_bad));
    void *host = nullptr;
    CC_TRY(ccgpu_ctx_pinned(ctx, 64, &host));
    CC_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned long long), st));
    CC_KLAUNCH(ctx, CCK_CHECK, k_check_labels, (unsigned)ctx->sm_count * 8, kBlock, 0, st,
               d_row_ptr, d_col_idx, n, m, d_labels, d_bad);
    CC_CUDA(cudaMemcpyAsync(host, d_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
    *violations = *(unsigned long long *)host;
    return CCGPU_OK;
}
