/*
 * Scans and the LSD radix sort used by the partitioned solver.
 *
 * The radix sort replaces the reference's in-place MSD American-flag sort of
 * boundary edges (src/boundary_sort.c:34-98).  It is a stable
 * least-significant-digit sort with 8-bit digits; each pass is
 *   upsweep   per 4096-key tile digit histogram, stored digit-major
 *   scan      exclusive scan of the histograms = each tile's output offset
 *             for each digit
 *   downsweep each warp ranks its 512 keys digit by digit with
 *             __match_any_sync (stable: tile order = warp, batch, lane), the
 *             tile is reordered in shared memory and written out in runs
 */
#include <cstring>

#include "primitives.h"

/* ------------------------------------------------------------- buffers */

int cc_pool_tune(void)
{
    static thread_local int pool_tuned = -1;
    int dev = 0;
    CC_CUDA(cudaGetDevice(&dev));
    if (pool_tuned != dev) {
        cudaMemPool_t pool;
        CC_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
        uint64_t thresh = ~0ull;
        CC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh));
        pool_tuned = dev;
    }
    return CCGPU_OK;
}

int cc_bufs_init(DevBufs *b, cudaStream_t st)
{
    CC_TRY(cc_pool_tune());
    b->st = st;
    b->n = 0;
    return CCGPU_OK;
}

int cc_bufs_get(DevBufs *b, void **p, size_t bytes)
{
    if (b->n >= (int)(sizeof(b->ptrs) / sizeof(b->ptrs[0])))
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "internal: more than %d temporary buffers",
                               (int)(sizeof(b->ptrs) / sizeof(b->ptrs[0])));
    if (bytes == 0)
        bytes = 16;
    cudaError_t e = cudaMallocAsync(p, bytes, b->st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ccgpu_set_error(CCGPU_ERR_OOM, "cudaMallocAsync(%zu) failed: %s", bytes,
                               cudaGetErrorString(e));
    }
    b->ptrs[b->n++] = *p;
    return CCGPU_OK;
}

void cc_bufs_release(DevBufs *b)
{
    for (int i = b->n - 1; i >= 0; --i)
        cudaFreeAsync(b->ptrs[i], b->st);
    b->n = 0;
}

/* --------------------------------------------------------------- scans */

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint64_t kScanTile = kScanThreads * kScanItems;

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_reduce_tiles(const T *__restrict__ in,
                                                               uint64_t count,
                                                               uint64_t *__restrict__ sums)
{
    __shared__ uint64_t s_warp[8];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint64_t i = base + (uint64_t)k * kScanThreads + threadIdx.x;
        if (i < count)
            acc += (uint64_t)in[i];
    }
    for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0)
        s_warp[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t t = 0;
        for (int w = 0; w < 8; ++w)
            t += s_warp[w];
        sums[blockIdx.x] = t;
    }
}

/* out[i] = offsets[tile] + exclusive prefix within the tile; the block that
 * holds the last element also writes out[count]. */
template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const T *__restrict__ in,
                                                             uint64_t *out, uint64_t count,
                                                             const uint64_t *__restrict__ offsets)
{
    __shared__ uint64_t s_warp[8];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint64_t v[kScanItems];
    uint64_t tsum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint64_t i = base + k;
        v[k] = i < count ? (uint64_t)in[i] : 0;
        tsum += v[k];
    }
    uint64_t total = 0;
    uint64_t incl = cc_block_incl_scan256<uint64_t>(tsum, s_warp, &total);
    uint64_t run = (offsets ? offsets[blockIdx.x] : 0) + incl - tsum;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint64_t i = base + k;
        if (i < count)
            out[i] = run;
        run += v[k];
    }
    uint64_t last_block = (count == 0) ? 0 : (count - 1) / kScanTile;
    if (blockIdx.x == last_block && threadIdx.x == kScanThreads - 1)
        out[count] = (offsets ? offsets[blockIdx.x] : 0) + total;
}

template <typename T>
int scan_impl(ccgpu_ctx *ctx, const T *in, uint64_t *out, uint64_t count, DevBufs *b,
              cudaStream_t st)
{
    if (count == 0) {
        CC_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), st));
        return CCGPU_OK;
    }
    uint64_t nb = (count + kScanTile - 1) / kScanTile;
    if (nb > 0x7fffffffull)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "scan of %llu elements", (unsigned long long)count);
    if (nb == 1) {
        CC_KLAUNCH(ctx, CCK_SCAN, k_scan_tiles<T>, 1, kScanThreads, 0, st, in, out, count,
                   (const uint64_t *)nullptr);
        return CCGPU_OK;
    }
    uint64_t *sums = nullptr;
    CC_TRY(cc_bufs_get(b, (void **)&sums, (nb + 1) * sizeof(uint64_t)));
    CC_KLAUNCH(ctx, CCK_SCAN, k_reduce_tiles<T>, (unsigned)nb, kScanThreads, 0, st, in, count,
               sums);
    CC_TRY(scan_impl<uint64_t>(ctx, sums, sums, nb, b, st));
    CC_KLAUNCH(ctx, CCK_SCAN, k_scan_tiles<T>, (unsigned)nb, kScanThreads, 0, st, in, out, count,
               (const uint64_t *)sums);
    return CCGPU_OK;
}

} // namespace

int cc_scan_u32(ccgpu_ctx *ctx, const uint32_t *in, uint64_t *out, uint64_t count, DevBufs *b,
                cudaStream_t st)
{
    return scan_impl<uint32_t>(ctx, in, out, count, b, st);
}

int cc_scan_u64(ccgpu_ctx *ctx, const uint64_t *in, uint64_t *out, uint64_t count, DevBufs *b,
                cudaStream_t st)
{
    return scan_impl<uint64_t>(ctx, in, out, count, b, st);
}

/* ---------------------------------------------------------- radix sort */

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kKeysPerThread = 8;
constexpr int kSortTile = kSortThreads * kKeysPerThread; /* 2048 */
constexpr int kWarpKeys = kSortTile / kSortWarps;        /* 256  */
constexpr uint32_t kInvalidDigit = 256;

__global__ void __launch_bounds__(kSortThreads) k_sort_upsweep(const uint64_t *__restrict__ keys,
                                                               uint64_t count, int shift,
                                                               uint32_t *__restrict__ hist,
                                                               uint64_t ntiles)
{
    __shared__ uint32_t s_h[256];
    s_h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int j = 0; j < kKeysPerThread; ++j) {
        uint64_t i = base + (uint64_t)j * kSortThreads + threadIdx.x;
        uint32_t d = i < count ? (uint32_t)((keys[i] >> shift) & 0xff) : kInvalidDigit;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        if (d != kInvalidDigit && (__ffs(peers) - 1) == (int)(threadIdx.x & 31))
            atomicAdd(&s_h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = s_h[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) k_sort_downsweep(const uint64_t *__restrict__ keys,
                                                                 uint64_t *__restrict__ out,
                                                                 uint64_t count, int shift,
                                                                 const uint64_t *__restrict__ off,
                                                                 uint64_t ntiles)
{
    __shared__ uint32_t s_wh[kSortWarps][256];
    __shared__ uint32_t s_start[256];
    __shared__ uint64_t s_goff[256];
    __shared__ uint32_t s_warp[8];
    __shared__ uint64_t s_keys[kSortTile];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const uint64_t tile_base = (uint64_t)blockIdx.x * kSortTile;
    const uint64_t wbase = tile_base + (uint64_t)warp * kWarpKeys;

    for (int d = lane; d < 256; d += 32)
        s_wh[warp][d] = 0;
    s_goff[threadIdx.x] = off[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
    __syncwarp();

    uint64_t k[kKeysPerThread];
    uint32_t rank[kKeysPerThread];
#pragma unroll
    for (int j = 0; j < kKeysPerThread; ++j) { /* all loads first, then the ranks */
        const uint64_t i = wbase + (uint64_t)j * 32 + lane;
        k[j] = i < count ? keys[i] : 0;
    }
#pragma unroll
    for (int j = 0; j < kKeysPerThread; ++j) {
        uint64_t i = wbase + (uint64_t)j * 32 + lane;
        uint32_t d = i < count ? (uint32_t)((k[j] >> shift) & 0xff) : kInvalidDigit;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = 0;
        if (d != kInvalidDigit)
            before = s_wh[warp][d];
        __syncwarp();
        if (d != kInvalidDigit && (__ffs(peers) - 1) == lane)
            s_wh[warp][d] = before + (uint32_t)__popc(peers);
        __syncwarp();
        rank[j] = before + (uint32_t)__popc(peers & lt_mask);
    }
    __syncthreads();
    /* per digit: exclusive prefix over warps, and the tile total */
    {
        const int d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t c = s_wh[w][d];
            s_wh[w][d] = run;
            run += c;
        }
        uint32_t incl = cc_block_incl_scan256<uint32_t>(run, s_warp, nullptr);
        s_start[d] = incl - run;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kKeysPerThread; ++j) {
        uint64_t i = wbase + (uint64_t)j * 32 + lane;
        if (i < count) {
            uint32_t d = (uint32_t)((k[j] >> shift) & 0xff);
            s_keys[s_start[d] + s_wh[warp][d] + rank[j]] = k[j];
        }
    }
    __syncthreads();
    uint64_t tile_n = count - tile_base < (uint64_t)kSortTile ? count - tile_base : kSortTile;
    for (uint32_t i = threadIdx.x; i < tile_n; i += kSortThreads) {
        uint64_t key = s_keys[i];
        uint32_t d = (uint32_t)((key >> shift) & 0xff);
        out[s_goff[d] + (i - s_start[d])] = key;
    }
}

} // namespace

int cc_radix_sort_u64(ccgpu_ctx *ctx, uint64_t *keys, uint64_t *alt, uint64_t count, int bits,
                      uint64_t **sorted, int *passes, DevBufs *b, cudaStream_t st)
{
    *sorted = keys;
    if (passes)
        *passes = 0;
    if (count <= 1 || bits <= 0)
        return CCGPU_OK;
    if (bits > 64)
        bits = 64;
    const int ndigits = (bits + 7) / 8;
    const uint64_t ntiles = (count + kSortTile - 1) / kSortTile;
    if (ntiles > 0x7fffffffull)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "sort of %llu keys", (unsigned long long)count);
    uint32_t *hist = nullptr;
    uint64_t *off = nullptr;
    CC_TRY(cc_bufs_get(b, (void **)&hist, ntiles * 256 * sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(b, (void **)&off, (ntiles * 256 + 1) * sizeof(uint64_t)));
    uint64_t *src = keys, *dst = alt;
    int np = 0;
    for (int d = 0; d < ndigits; ++d) {
        const int shift = 8 * d;
        CC_KLAUNCH(ctx, CCK_SORT_HIST, k_sort_upsweep, (unsigned)ntiles, kSortThreads, 0, st, src,
                   count, shift, hist, ntiles);
        CC_TRY(cc_scan_u32(ctx, hist, off, ntiles * 256, b, st));
        CC_KLAUNCH(ctx, CCK_SORT_SCATTER, k_sort_downsweep, (unsigned)ntiles, kSortThreads, 0, st,
                   src, dst, count, shift, (const uint64_t *)off, ntiles);
        uint64_t *t = src;
        src = dst;
        dst = t;
        np++;
    }
    *sorted = src;
    if (passes)
        *passes = np;
    return CCGPU_OK;
}
