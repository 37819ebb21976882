/*
 * Local connected components on one device-resident CSR (sm_100a).
 *
 * Replaces the reference's pthreads label propagation
 * (src/cc_pthreads.c:32-73 relax, :76-150 round loop, :152-229 driver),
 * whose result - each label is the minimum vertex id of its component - is
 * kept bit for bit.  The method here is union-find hooking (the larger root
 * is CAS-hooked under the smaller root, so every root is its tree's
 * minimum id) with Afforest-style neighbour sampling (Sutton, Ben-Nun and
 * Barak, IPDPS 2018): after linking each vertex with its first few
 * neighbours, the most frequent root is found and the remaining rows of its
 * tree are never read.  That skip is valid for symmetric graphs, which is
 * the reference's input contract.
 *
 * Kernels (all grid-stride, 256 threads):
 *   k_init       parent[v] = v (16-byte stores) and zeroes the counters
 *   k_sample     thread per vertex, links neighbours [r0, r1) of its row
 *   k_compress   parent[v] = root(v)
 *   k_giant      one CTA: most frequent root among 1024 seeded samples
 *   k_link_rows  degree-binned finish pass (CTA gather / warp / queue)
 *   k_link_heavy rows above the heavy threshold, split over every CTA
 *   k_count_roots, k_check_labels   reductions for stats and tests
 */
#include <cstdio>
#include <cstring>

#include "ccgpu_internal.h"

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr uint32_t kNoGiant = 0xffffffffu;
constexpr int kGiantSamples = 1024;
constexpr uint64_t kHeavySeg = 4096;

struct Rows {
    uint64_t beg, end;
};

__device__ __forceinline__ Rows row_of(const uint64_t *__restrict__ row_ptr, uint32_t v, uint64_t m)
{
    uint64_t b = __ldg(row_ptr + v), e = __ldg(row_ptr + v + 1);
    if (e > m)
        e = m;
    if (b > e)
        b = e;
    return {b, e};
}

/* MurmurHash3 fmix32 finaliser (Appleby, public domain) as a sample mixer. */
__device__ __forceinline__ uint32_t mix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

__global__ void __launch_bounds__(kBlock) k_init(uint32_t *__restrict__ parent, uint32_t n,
                                                 uint32_t *__restrict__ counters, int ncounters,
                                                 int vec)
{
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    const uint64_t tid = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (blockIdx.x == 0 && (int)threadIdx.x < ncounters)
        counters[threadIdx.x] = 0;
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

__global__ void __launch_bounds__(kBlock) k_sample(const uint64_t *__restrict__ row_ptr,
                                                   const uint32_t *__restrict__ col, uint32_t n,
                                                   uint64_t m, uint32_t *parent, uint32_t v_lo,
                                                   uint32_t v_hi, int r0, int r1)
{
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    for (uint64_t v = (uint64_t)v_lo + (uint64_t)blockIdx.x * kBlock + threadIdx.x; v < v_hi;
         v += stride) {
        Rows r = row_of(row_ptr, (uint32_t)v, m);
        for (int k = r0; k < r1; ++k) {
            uint64_t j = r.beg + (uint64_t)k;
            if (j >= r.end)
                break;
            uint32_t u = __ldg(col + j);
            if (u < n)
                cc_link(parent, (uint32_t)v, u);
        }
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

/* Most frequent root among kGiantSamples seeded samples.  Ties go to the
 * smaller root so the choice is deterministic for a given forest. */
__global__ void __launch_bounds__(kGiantSamples) k_giant(const uint32_t *parent, uint32_t n,
                                                         uint32_t seed, uint32_t *out)
{
    __shared__ uint32_t s[kGiantSamples];
    __shared__ unsigned long long s_best[kGiantSamples / 32];
    const uint32_t i = threadIdx.x;
    uint32_t v = (uint32_t)(((uint64_t)mix32(i * 0x9e3779b9u + seed) * n) >> 32);
    s[i] = cc_find_ro(parent, v);
    __syncthreads();
    for (uint32_t k = 2; k <= kGiantSamples; k <<= 1) {
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
    uint32_t cnt = 0, val = s[i];
    if (i == 0 || s[i - 1] != val) {
        uint32_t lo = i, hi = kGiantSamples;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (s[mid] <= val)
                lo = mid + 1;
            else
                hi = mid;
        }
        cnt = lo - i;
    }
    unsigned long long key = ((unsigned long long)cnt << 32) | (uint32_t)~val;
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if ((i & 31) == 0)
        s_best[i >> 5] = key;
    __syncthreads();
    if (i < 32) {
        key = s_best[i];
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
            key = other > key ? other : key;
        }
        if (i == 0)
            out[0] = ~(uint32_t)key;
    }
}

struct LinkParams {
    const uint64_t *row_ptr;
    const uint32_t *col;
    uint32_t n;
    uint64_t m;
    uint32_t *parent;
    uint32_t skip_from;        /* first row entry the finish pass links   */
    const uint32_t *giant;     /* device giant root, NULL = no skipping    */
    uint32_t chunk;            /* vertices per work grab, 0 = static       */
    unsigned long long *grab;  /* work counter                             */
    uint32_t *heavy_list;
    uint32_t *heavy_count;
    uint32_t heavy_cap;
    uint32_t heavy_deg;
    int vec;                   /* col is 16-byte aligned                    */
    unsigned long long *finish; /* [0] rows linked, [1] entries linked      */
};

/* One warp links v with row entries [beg, end): 16-byte column loads for
 * the aligned body, scalar head and tail. */
__device__ __forceinline__ void warp_link_row(const LinkParams &P, uint32_t v, uint64_t beg,
                                              uint64_t end, int lane)
{
    uint64_t a = beg, body_end = beg;
    if (P.vec) {
        a = (beg + 3) & ~3ull;
        if (a > end)
            a = end;
        body_end = end & ~3ull;
        if (body_end < a)
            body_end = a;
        if (beg + lane < a) {
            uint32_t u = __ldg(P.col + beg + lane);
            if (u < P.n)
                cc_link(P.parent, v, u);
        }
        const uint4 *c4 = reinterpret_cast<const uint4 *>(P.col);
        for (uint64_t q = a / 4 + lane; q < body_end / 4; q += 32) {
            uint4 x = __ldg(c4 + q);
            if (x.x < P.n)
                cc_link(P.parent, v, x.x);
            if (x.y < P.n)
                cc_link(P.parent, v, x.y);
            if (x.z < P.n)
                cc_link(P.parent, v, x.z);
            if (x.w < P.n)
                cc_link(P.parent, v, x.w);
        }
    }
    for (uint64_t j = body_end + lane; j < end; j += 32) {
        uint32_t u = __ldg(P.col + j);
        if (u < P.n)
            cc_link(P.parent, v, u);
    }
}

__global__ void __launch_bounds__(kBlock) k_link_rows(LinkParams P)
{
    __shared__ uint32_t s_off[kBlock + 1];
    __shared__ uint64_t s_beg[kBlock];
    __shared__ uint32_t s_wsum[kWarps];
    __shared__ unsigned long long s_base;

    const uint32_t giant = P.giant ? *P.giant : kNoGiant;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t my_rows = 0;
    unsigned long long my_edges = 0;

    uint64_t st_lo = 0, st_hi = 0;
    if (P.chunk == 0) {
        uint64_t per = ((uint64_t)P.n + gridDim.x - 1) / gridDim.x;
        per = (per + kBlock - 1) / kBlock * kBlock;
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
                s_base = atomicAdd(P.grab, (unsigned long long)P.chunk);
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
        for (uint64_t t0 = base; t0 < cend; t0 += kBlock) {
            const uint64_t v64 = t0 + threadIdx.x;
            const uint32_t v = (uint32_t)v64;
            uint64_t beg = 0, end = 0;
            if (v64 < cend && (giant == kNoGiant || cc_ldp(P.parent, v) != giant)) {
                Rows r = row_of(P.row_ptr, v, P.m);
                beg = r.beg + P.skip_from;
                end = r.end;
                if (beg > end)
                    beg = end;
                my_rows++;
                my_edges += end - beg;
            }
            uint64_t deg = end - beg;
            if (deg > P.heavy_deg) {
                uint32_t slot = atomicAdd(P.heavy_count, 1u);
                if (slot < P.heavy_cap) {
                    P.heavy_list[slot] = v;
                    deg = 0;
                }
            }
            /* warp-cooperative rows */
            unsigned big = __ballot_sync(0xffffffffu, deg >= 32);
            while (big) {
                int src = __ffs(big) - 1;
                big &= big - 1;
                uint32_t vv = __shfl_sync(0xffffffffu, v, src);
                uint64_t bb = __shfl_sync(0xffffffffu, beg, src);
                uint64_t ee = __shfl_sync(0xffffffffu, end, src);
                warp_link_row(P, vv, bb, ee, lane);
            }
            /* short rows: CTA-wide gather, walked edge-parallel */
            uint32_t small = deg < 32 ? (uint32_t)deg : 0u;
            uint32_t incl = small;
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o)
                    incl += y;
            }
            if (lane == 31)
                s_wsum[warp] = incl;
            s_beg[threadIdx.x] = beg;
            __syncthreads();
            uint32_t wpre = 0, total = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                uint32_t x = s_wsum[w];
                wpre += (w < warp) ? x : 0u;
                total += x;
            }
            s_off[threadIdx.x] = wpre + incl - small;
            if (threadIdx.x == 0)
                s_off[kBlock] = total;
            __syncthreads();
            for (uint32_t e = threadIdx.x; e < total; e += kBlock) {
                int lo = 0, hi = kBlock;
                while (hi - lo > 1) {
                    int mid = (lo + hi) >> 1;
                    if (s_off[mid] <= e)
                        lo = mid;
                    else
                        hi = mid;
                }
                uint64_t j = s_beg[lo] + (e - s_off[lo]);
                uint32_t u = __ldg(P.col + j);
                if (u < P.n)
                    cc_link(P.parent, (uint32_t)(t0 + lo), u);
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
        atomicAdd(P.finish, rows);
        atomicAdd(P.finish + 1, my_edges);
    }
}

__global__ void __launch_bounds__(kBlock) k_link_heavy(LinkParams P)
{
    uint32_t cnt = *P.heavy_count;
    if (cnt > P.heavy_cap)
        cnt = P.heavy_cap;
    for (uint32_t h = 0; h < cnt; ++h) {
        uint32_t v = P.heavy_list[h];
        Rows r = row_of(P.row_ptr, v, P.m);
        uint64_t beg = r.beg + P.skip_from;
        if (beg > r.end)
            beg = r.end;
        uint64_t nseg = (r.end - beg + kHeavySeg - 1) / kHeavySeg;
        for (uint64_t s = blockIdx.x; s < nseg; s += gridDim.x) {
            uint64_t sb = beg + s * kHeavySeg;
            uint64_t se = sb + kHeavySeg < r.end ? sb + kHeavySeg : r.end;
            for (uint64_t j = sb + threadIdx.x; j < se; j += kBlock) {
                uint32_t u = __ldg(P.col + j);
                if (u < P.n)
                    cc_link(P.parent, v, u);
            }
        }
    }
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
        Rows r = row_of(row_ptr, (uint32_t)v, m);
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

/* Device scratch of one local-CC call. */
struct Scratch {
    unsigned long long *grab;
    uint32_t *heavy_count;
    uint32_t *giant;
    unsigned long long *finish;
    uint32_t *heavy_list;
    uint32_t heavy_cap;
};

constexpr int kCounterWords = 8; /* grab (2 words), heavy_count, giant, finish (4) */

size_t carve_scratch(cc_carve *c, Scratch *s, uint32_t n, uint64_t m, uint32_t heavy_deg)
{
    uint64_t cap = m / (heavy_deg ? heavy_deg : 1) + 1;
    if (cap > n)
        cap = n;
    if (cap == 0)
        cap = 1;
    uint32_t *counters = (uint32_t *)cc_take(c, kCounterWords * sizeof(uint32_t));
    s->heavy_list = (uint32_t *)cc_take(c, cap * sizeof(uint32_t));
    s->heavy_cap = (uint32_t)cap;
    s->grab = (unsigned long long *)counters;
    s->heavy_count = counters + 2;
    s->giant = counters + 3;
    s->finish = (unsigned long long *)(counters + 4);
    return c->off;
}

int resolve_opts(const ccgpu_cc_opts *in, ccgpu_cc_opts *o)
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
    }
    if (o->sample_rounds > 8)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "sample_rounds %d above 8", o->sample_rounds);
    if (o->heavy_degree < 32)
        o->heavy_degree = 32;
    return CCGPU_OK;
}

struct Geometry {
    unsigned stream_blocks; /* grid for the streaming kernels      */
    unsigned link_blocks;   /* resident grid for k_link_rows        */
};

int geometry(const ccgpu_ctx *ctx, Geometry *g)
{
    static thread_local int occ_rows = 0;
    if (!occ_rows) {
        CC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_rows, k_link_rows, kBlock, 0));
        if (occ_rows < 1)
            occ_rows = 1;
    }
    g->stream_blocks = (unsigned)ctx->sm_count * 8;
    g->link_blocks = (unsigned)ctx->sm_count * (unsigned)occ_rows;
    return CCGPU_OK;
}

} // namespace

/* ------------------------------------------------------------------ API */

extern "C" void ccgpu_cc_opts_default(ccgpu_cc_opts *o)
{
    if (!o)
        return;
    o->chunk_size = 4096;
    o->sample_rounds = 2;
    o->heavy_degree = 8192;
    o->skip_giant = 1;
}

/* The solve itself, on scratch already carved.  `sample_hi` bounds the
 * vertices k_sample covers (the host pipeline samples ranges itself and
 * passes sampled = 1). */
static int local_cc_launch(ccgpu_ctx *ctx, const uint64_t *d_row_ptr, const uint32_t *d_col,
                           uint32_t n, uint64_t m, uint32_t *d_labels, const ccgpu_cc_opts *o,
                           const Scratch &s, cudaStream_t st, int init_done, int sampled,
                           uint32_t *kernels)
{
    Geometry g = {1, 1};
    CC_TRY(geometry(ctx, &g));
    const unsigned sb = cc_blocks(n, kBlock, g.stream_blocks);
    const unsigned long long before = ctx->launches;
    if (!init_done)
        CC_KLAUNCH(ctx, CCK_INIT, k_init, sb, kBlock, 0, st, d_labels, n, (uint32_t *)s.grab,
                   kCounterWords, ((uintptr_t)d_labels & 15) == 0);
    const int k = o->sample_rounds;
    const bool skip = k > 0 && o->skip_giant;
    if (k > 0) {
        if (!sampled)
            CC_KLAUNCH(ctx, CCK_SAMPLE, k_sample, sb, kBlock, 0, st, d_row_ptr, d_col, n, m,
                       d_labels, 0u, n, 0, k);
        if (skip) {
            CC_KLAUNCH(ctx, CCK_COMPRESS, k_compress, sb, kBlock, 0, st, d_labels, n);
            CC_KLAUNCH(ctx, CCK_GIANT, k_giant, 1, kGiantSamples, 0, st, d_labels, n,
                       0x5eed1234u, s.giant);
        }
    }
    LinkParams P;
    P.row_ptr = d_row_ptr;
    P.col = d_col;
    P.n = n;
    P.m = m;
    P.parent = d_labels;
    P.skip_from = (uint32_t)k;
    P.giant = skip ? s.giant : nullptr;
    P.chunk = o->chunk_size == 1 ? 0u : (uint32_t)o->chunk_size;
    P.grab = s.grab;
    P.heavy_list = s.heavy_list;
    P.heavy_count = s.heavy_count;
    P.heavy_cap = s.heavy_cap;
    P.heavy_deg = (uint32_t)o->heavy_degree;
    P.vec = ((uintptr_t)d_col & 15) == 0;
    P.finish = s.finish;
    CC_KLAUNCH(ctx, CCK_LINK_ROWS, k_link_rows, g.link_blocks, kBlock, 0, st, P);
    CC_KLAUNCH(ctx, CCK_LINK_HEAVY, k_link_heavy, g.link_blocks, kBlock, 0, st, P);
    CC_KLAUNCH(ctx, CCK_FINAL_COMPRESS, k_compress, sb, kBlock, 0, st, d_labels, n);
    const uint32_t launches = (uint32_t)(ctx->launches - before);
    if (kernels)
        *kernels = launches;
    return CCGPU_OK;
}

static int fill_stats(ccgpu_ctx *ctx, const Scratch &s, const uint32_t *d_labels, uint32_t n,
                      const ccgpu_cc_opts *o, uint32_t kernels, ccgpu_cc_stats *stats,
                      cudaStream_t st)
{
    uint64_t roots = 0;
    CC_TRY(ccgpu_count_roots(ctx, d_labels, n, &roots, st));
    uint32_t h[6] = {0, 0, 0, 0, 0, 0};
    CC_CUDA(cudaMemcpyAsync(h, s.heavy_count, 6 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
    memcpy(&stats->finish_rows, h + 2, sizeof(uint64_t));
    memcpy(&stats->finish_edges, h + 4, sizeof(uint64_t));
    stats->heavy_rows = h[0] < s.heavy_cap ? h[0] : s.heavy_cap;
    stats->giant_label = (o->sample_rounds > 0 && o->skip_giant) ? h[1] : 0xffffffffu;
    stats->components = (uint32_t)roots;
    stats->kernels = kernels + 1;
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
    ccgpu_cc_opts o;
    CC_TRY(resolve_opts(opts, &o));
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = (cudaStream_t)stream;
    Scratch s;
    cc_carve c = {nullptr, 0};
    size_t bytes = carve_scratch(&c, &s, n, m, (uint32_t)o.heavy_degree);
    void *base = nullptr;
    CC_TRY(ccgpu_ctx_reserve(ctx, bytes, &base));
    c = {(char *)base, 0};
    carve_scratch(&c, &s, n, m, (uint32_t)o.heavy_degree);
    uint32_t kernels = 0;
    CC_TRY(local_cc_launch(ctx, d_row_ptr, d_col_idx, n, m, d_labels, &o, s, st, 0, 0, &kernels));
    if (stats)
        CC_TRY(fill_stats(ctx, s, d_labels, n, &o, kernels, stats, st));
    return CCGPU_OK;
}

/* Host-buffer variant.  Device copies of the CSR and the labels live in
 * the context's scratch.  Column chunks are copied on a second stream and
 * each chunk's vertex range is sampled as soon as its columns landed. */
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
    ccgpu_cc_opts o;
    CC_TRY(resolve_opts(opts, &o));
    CC_TRY(ccgpu_ctx_resolve(&ctx));

    Scratch s;
    cc_carve c = {nullptr, 0};
    carve_scratch(&c, &s, n, m, (uint32_t)o.heavy_degree);
    uint64_t *d_row = (uint64_t *)cc_take(&c, ((size_t)n + 1) * sizeof(uint64_t));
    uint32_t *d_col = (uint32_t *)cc_take(&c, (size_t)(m ? m : 1) * sizeof(uint32_t));
    uint32_t *d_lab = (uint32_t *)cc_take(&c, (size_t)n * sizeof(uint32_t));
    void *base = nullptr;
    CC_TRY(ccgpu_ctx_reserve(ctx, c.off, &base));
    c = {(char *)base, 0};
    carve_scratch(&c, &s, n, m, (uint32_t)o.heavy_degree);
    d_row = (uint64_t *)cc_take(&c, ((size_t)n + 1) * sizeof(uint64_t));
    d_col = (uint32_t *)cc_take(&c, (size_t)(m ? m : 1) * sizeof(uint32_t));
    d_lab = (uint32_t *)cc_take(&c, (size_t)n * sizeof(uint32_t));

    cudaStream_t st = nullptr, cp = nullptr;
    int rc = CCGPU_OK;
    const int kPieces = 8;
    cudaEvent_t ev[kPieces] = {};
    Geometry g = {1, 1};
    CC_TRY(geometry(ctx, &g));
#define HOST_TRY(call)                                                         \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            rc = ccgpu_cuda_fail(e_, #call, __FILE__, __LINE__);               \
            goto done;                                                         \
        }                                                                      \
    } while (0)
    HOST_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    HOST_TRY(cudaStreamCreateWithFlags(&cp, cudaStreamNonBlocking));
    for (int i = 0; i < kPieces; ++i)
        HOST_TRY(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    HOST_TRY(cudaMemcpyAsync(d_row, h_row_ptr, ((size_t)n + 1) * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, st));
    if (ctx->prof)
        cc_prof_mark(ctx, CCK_INIT, 0, st);
    k_init<<<cc_blocks(n, kBlock, g.stream_blocks), kBlock, 0, st>>>(
        d_lab, n, (uint32_t *)s.grab, kCounterWords, 1);
    HOST_TRY(cudaGetLastError());
    ctx->launches++;
    if (ctx->prof)
        cc_prof_mark(ctx, CCK_INIT, 1, st);
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
        if (o.sample_rounds > 0) {
            HOST_TRY(cudaStreamWaitEvent(st, ev[i], 0));
            if (ctx->prof)
                cc_prof_mark(ctx, CCK_SAMPLE, 0, st);
            k_sample<<<cc_blocks(vhi - vlo, kBlock, g.stream_blocks), kBlock, 0, st>>>(
                d_row, d_col, n, m, d_lab, vlo, vhi, 0, o.sample_rounds);
            HOST_TRY(cudaGetLastError());
            ctx->launches++;
            if (ctx->prof)
                cc_prof_mark(ctx, CCK_SAMPLE, 1, st);
        }
    }
    HOST_TRY(cudaStreamWaitEvent(st, ev[kPieces - 1], 0));
    {
        uint32_t kernels = 0;
        rc = local_cc_launch(ctx, d_row, d_col, n, m, d_lab, &o, s, st, 1, 1, &kernels);
        if (rc != CCGPU_OK)
            goto done;
        HOST_TRY(cudaMemcpyAsync(h_labels, d_lab, (size_t)n * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st));
        if (stats) {
            rc = fill_stats(ctx, s, d_lab, n, &o, kernels + 1 + kPieces, stats, st);
            if (rc != CCGPU_OK)
                goto done;
        }
        HOST_TRY(cudaStreamSynchronize(st));
    }
done:
#undef HOST_TRY
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
    CC_KLAUNCH(ctx, CCK_COUNT_ROOTS, k_count_roots, cc_blocks(n, kBlock, (unsigned)ctx->sm_count * 8),
               kBlock, 0, st, d_labels, n, cell);
    CC_CUDA(cudaMemcpyAsync(host, cell, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st));
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
    unsigned long long h = *(unsigned long long *)host;
    *violations = h;
    return CCGPU_OK;
}
