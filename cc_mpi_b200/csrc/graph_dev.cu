/*
 * Device memory helpers and device-resident CSR graphs for the host C layer,
 * including the CSC -> CSR transposition of a .mat sparse matrix on the
 * device.
 */
#include <cstdlib>
#include <mutex>

#include "ccgpu_internal.h"
#include "primitives.h"

struct ccgpu_graph {
    uint64_t *row_ptr;
    uint32_t *col;
    uint32_t n;
    uint64_t m;
    int device;
    size_t rp_cap, col_cap; /* bytes allocated for row_ptr / col */
    uint32_t *labels;       /* ccgpu_graph_label_array, lab_cap bytes */
    size_t lab_cap;
};

namespace {

/* The arrays of the last freed graph of each device, kept for the next
 * upload: a caller that uploads, solves and frees a graph of the same size
 * over and over (the reference's load / solve / free cycle) maps its
 * gigabytes once instead of on every call. */
constexpr int kGraphCacheDevices = 64;
struct GraphCache {
    uint64_t *row_ptr = nullptr;
    uint32_t *col = nullptr;
    size_t rp_cap = 0, col_cap = 0;
    uint32_t *labels = nullptr;
    size_t lab_cap = 0;
};
GraphCache g_gcache[kGraphCacheDevices];
std::mutex g_gcache_mu;

/* Arrays for a graph on the current device: the cached ones when they are
 * large enough, else new ones (the cache is released first if cudaMalloc
 * fails). */
cudaError_t graph_arrays(ccgpu_graph *g, size_t rp_bytes, size_t col_bytes)
{
    {
        std::lock_guard<std::mutex> lk(g_gcache_mu);
        if (g->device >= 0 && g->device < kGraphCacheDevices) {
            GraphCache &c = g_gcache[g->device];
            if (c.row_ptr && c.rp_cap >= rp_bytes && c.col_cap >= col_bytes) {
                g->row_ptr = c.row_ptr;
                g->col = c.col;
                g->rp_cap = c.rp_cap;
                g->col_cap = c.col_cap;
                g->labels = c.labels;
                g->lab_cap = c.lab_cap;
                c = GraphCache();
                return cudaSuccess;
            }
        }
    }
    for (int attempt = 0; attempt < 2; ++attempt) {
        cudaError_t e = cudaMalloc((void **)&g->row_ptr, rp_bytes);
        if (e == cudaSuccess) {
            e = cudaMalloc((void **)&g->col, col_bytes);
            if (e != cudaSuccess) {
                cudaFree(g->row_ptr);
                g->row_ptr = nullptr;
            }
        }
        if (e == cudaSuccess) {
            g->rp_cap = rp_bytes;
            g->col_cap = col_bytes;
            return cudaSuccess;
        }
        cudaGetLastError();
        if (attempt == 0) { /* give the cached arrays back and try again */
            std::lock_guard<std::mutex> lk(g_gcache_mu);
            if (g->device >= 0 && g->device < kGraphCacheDevices) {
                GraphCache &c = g_gcache[g->device];
                cudaFree(c.row_ptr);
                cudaFree(c.col);
                cudaFree(c.labels);
                c = GraphCache();
            }
        } else {
            return e;
        }
    }
    return cudaErrorMemoryAllocation;
}

} // namespace

extern "C" int ccgpu_alloc(void **d_ptr, size_t bytes)
{
    if (!d_ptr)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_alloc: NULL out pointer");
    *d_ptr = nullptr;
    CC_TRY(ccgpu_device_check());
    CC_CUDA(cudaMalloc(d_ptr, bytes ? bytes : 16));
    return CCGPU_OK;
}

extern "C" void ccgpu_free(void *d_ptr)
{
    if (d_ptr)
        cudaFree(d_ptr);
}

extern "C" int ccgpu_memcpy_h2d(void *d_dst, const void *h_src, size_t bytes)
{
    if (bytes == 0)
        return CCGPU_OK;
    CC_CUDA(cudaMemcpy(d_dst, h_src, bytes, cudaMemcpyHostToDevice));
    return CCGPU_OK;
}

extern "C" int ccgpu_memcpy_d2h(void *h_dst, const void *d_src, size_t bytes)
{
    if (bytes == 0)
        return CCGPU_OK;
    CC_CUDA(cudaMemcpy(h_dst, d_src, bytes, cudaMemcpyDeviceToHost));
    return CCGPU_OK;
}

extern "C" int ccgpu_graph_upload(const uint64_t *h_row_ptr, const uint32_t *h_col_idx,
                                  uint32_t n, uint64_t m, ccgpu_graph **out)
{
    if (!out || !h_row_ptr || (m && !h_col_idx))
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_graph_upload: NULL argument");
    *out = nullptr;
    CC_TRY(ccgpu_device_check());
    ccgpu_graph *g = (ccgpu_graph *)calloc(1, sizeof(ccgpu_graph));
    if (!g)
        return ccgpu_set_error(CCGPU_ERR_OOM, "ccgpu_graph_upload: host OOM");
    cudaGetDevice(&g->device);
    g->n = n;
    g->m = m;
    cudaError_t e = graph_arrays(g, ((size_t)n + 1) * sizeof(uint64_t),
                                 (size_t)(m ? m : 1) * sizeof(uint32_t));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->row_ptr, h_row_ptr, ((size_t)n + 1) * sizeof(uint64_t),
                            cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess && m)
        e = cudaMemcpyAsync(g->col, h_col_idx, (size_t)m * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        int rc = ccgpu_cuda_fail(e, "ccgpu_graph_upload", __FILE__, __LINE__);
        ccgpu_graph_free(g);
        return rc;
    }
    *out = g;
    return CCGPU_OK;
}

extern "C" void ccgpu_graph_free(ccgpu_graph *g)
{
    if (!g)
        return;
    /* like cudaFree, wait for work that may still read the arrays; then
     * keep them for the next upload on this device, or free them when the
     * cache already holds a graph's arrays */
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != g->device)
        cudaSetDevice(g->device);
    cudaDeviceSynchronize();
    bool kept = false;
    if (g->row_ptr && g->col && g->device >= 0 && g->device < kGraphCacheDevices) {
        std::lock_guard<std::mutex> lk(g_gcache_mu);
        GraphCache &c = g_gcache[g->device];
        if (!c.row_ptr) {
            c.row_ptr = g->row_ptr;
            c.col = g->col;
            c.rp_cap = g->rp_cap;
            c.col_cap = g->col_cap;
            c.labels = g->labels;
            c.lab_cap = g->lab_cap;
            kept = true;
        }
    }
    if (!kept) {
        cudaFree(g->row_ptr);
        cudaFree(g->col);
        cudaFree(g->labels);
    }
    if (cur >= 0 && cur != g->device)
        cudaSetDevice(cur);
    free(g);
}

extern "C" const uint64_t *ccgpu_graph_row_ptr(const ccgpu_graph *g) { return g ? g->row_ptr : nullptr; }
extern "C" const uint32_t *ccgpu_graph_col_idx(const ccgpu_graph *g) { return g ? g->col : nullptr; }
extern "C" uint32_t ccgpu_graph_n(const ccgpu_graph *g) { return g ? g->n : 0; }
extern "C" uint64_t ccgpu_graph_m(const ccgpu_graph *g) { return g ? g->m : 0; }

extern "C" int ccgpu_graph_label_array(ccgpu_graph *g, uint32_t **d_labels)
{
    if (!g || !d_labels)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_graph_label_array: NULL argument");
    const size_t bytes = (size_t)(g->n ? g->n : 1) * sizeof(uint32_t);
    if (!g->labels || g->lab_cap < bytes) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != g->device)
            cudaSetDevice(g->device);
        cudaFree(g->labels);
        g->labels = nullptr;
        g->lab_cap = 0;
        cudaError_t e = cudaMalloc((void **)&g->labels, bytes);
        if (cur >= 0 && cur != g->device)
            cudaSetDevice(cur);
        if (e != cudaSuccess) {
            g->labels = nullptr;
            return ccgpu_cuda_fail(e, "ccgpu_graph_label_array", __FILE__, __LINE__);
        }
        g->lab_cap = bytes;
    }
    *d_labels = g->labels;
    return CCGPU_OK;
}

/* ------------------------------------------------- CSC -> CSR on device */

namespace {

constexpr int kCsc = 256;

/* Key of entry j of the CSC: (row << cb) | column; rows outside [0, nrows)
 * get row nrows, which sorts after every kept key.  The column of j is the
 * last c with jc[c] <= j (empty columns repeat their start).  Row lengths
 * are counted with one atomic per run of equal rows in a warp. */
__global__ void __launch_bounds__(kCsc) k_csc_keys(const uint64_t *__restrict__ jc, uint32_t ncols,
                                                   const uint32_t *__restrict__ ir, uint64_t nnz,
                                                   uint32_t nrows, int cb, uint64_t *keys,
                                                   uint32_t *rowcnt)
{
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * kCsc;
    for (uint64_t base = (uint64_t)blockIdx.x * kCsc; base < nnz; base += stride) {
        const uint64_t j = base + threadIdx.x;
        uint32_t r = 0xffffffffu;
        if (j < nnz) {
            uint32_t lo = 0, hi = ncols;
            while (hi - lo > 1) {
                const uint32_t mid = lo + (hi - lo) / 2;
                if (__ldg(jc + mid) <= j)
                    lo = mid;
                else
                    hi = mid;
            }
            r = __ldg(ir + j);
            const uint64_t row = r < nrows ? r : nrows;
            keys[j] = (row << cb) | lo;
        }
        const bool ok = r < nrows;
        const unsigned peers = __match_any_sync(0xffffffffu, ok ? r : 0xffffffffu);
        if (ok && (__ffs(peers) - 1) == lane)
            atomicAdd(rowcnt + r, (uint32_t)__popc(peers));
    }
}

__global__ void __launch_bounds__(kCsc) k_csc_cols(const uint64_t *__restrict__ sorted, uint64_t m,
                                                   uint64_t cmask, uint32_t *col)
{
    const uint64_t stride = (uint64_t)gridDim.x * kCsc;
    for (uint64_t i = (uint64_t)blockIdx.x * kCsc + threadIdx.x; i < m; i += stride)
        col[i] = (uint32_t)(__ldg(sorted + i) & cmask);
}

int bits_of(uint64_t max_value)
{
    int b = 0;
    while (b < 64 && (max_value >> b) != 0)
        ++b;
    return b < 1 ? 1 : b;
}

} // namespace

extern "C" int ccgpu_graph_from_csc(const uint64_t *h_jc, const uint32_t *h_ir, uint32_t nrows,
                                    uint32_t ncols, uint64_t nnz, ccgpu_graph **out)
{
    if (!out || !h_jc || (nnz && !h_ir))
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_graph_from_csc: NULL argument");
    *out = nullptr;
    if (nrows == 0xffffffffu)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "ccgpu_graph_from_csc: nrows must be below 2^32-1");
    if (nnz > h_jc[ncols])
        nnz = h_jc[ncols];
    const int cb = bits_of(ncols ? ncols - 1 : 0);
    const int bits = cb + bits_of(nrows);
    if (bits > 64)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "ccgpu_graph_from_csc: key needs %d bits", bits);
    ccgpu_ctx *ctx = nullptr;
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = nullptr;
    CC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    DevBufs B;
    int rc = cc_bufs_init(&B, st);
    ccgpu_graph *g = nullptr;
    uint64_t *d_jc = nullptr, *keys = nullptr, *alt = nullptr, *sorted = nullptr;
    uint32_t *d_ir = nullptr, *rowcnt = nullptr;
    uint64_t m = 0;
    int passes = 0;
    const unsigned grid = (unsigned)ctx->sm_count * 8;
    auto cuda = [&](cudaError_t e, int line) {
        if (rc == CCGPU_OK && e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "ccgpu_graph_from_csc", __FILE__, line);
    };
    if (rc == CCGPU_OK) {
        g = (ccgpu_graph *)calloc(1, sizeof(ccgpu_graph));
        if (!g)
            rc = ccgpu_set_error(CCGPU_ERR_OOM, "ccgpu_graph_from_csc: host OOM");
    }
    if (rc == CCGPU_OK) {
        cudaGetDevice(&g->device);
        g->n = nrows;
        cuda(cudaMalloc((void **)&g->row_ptr, ((size_t)nrows + 1) * sizeof(uint64_t)), __LINE__);
        g->rp_cap = ((size_t)nrows + 1) * sizeof(uint64_t);
    }
    if (rc == CCGPU_OK)
        rc = cc_bufs_get(&B, (void **)&d_jc, ((size_t)ncols + 1) * sizeof(uint64_t));
    if (rc == CCGPU_OK)
        rc = cc_bufs_get(&B, (void **)&d_ir, (size_t)(nnz ? nnz : 1) * sizeof(uint32_t));
    if (rc == CCGPU_OK)
        rc = cc_bufs_get(&B, (void **)&keys, (size_t)(nnz ? nnz : 1) * sizeof(uint64_t));
    if (rc == CCGPU_OK)
        rc = cc_bufs_get(&B, (void **)&alt, (size_t)(nnz ? nnz : 1) * sizeof(uint64_t));
    if (rc == CCGPU_OK)
        rc = cc_bufs_get(&B, (void **)&rowcnt, ((size_t)nrows + 1) * sizeof(uint32_t));
    if (rc == CCGPU_OK) {
        cuda(cudaMemcpyAsync(d_jc, h_jc, ((size_t)ncols + 1) * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, st), __LINE__);
        if (nnz)
            cuda(cudaMemcpyAsync(d_ir, h_ir, (size_t)nnz * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, st), __LINE__);
        cuda(cudaMemsetAsync(rowcnt, 0, ((size_t)nrows + 1) * sizeof(uint32_t), st), __LINE__);
    }
    if (rc == CCGPU_OK && nnz) {
        CC_KLAUNCH(ctx, CCK_MISC, k_csc_keys, cc_blocks(nnz, kCsc, grid), kCsc, 0, st, d_jc,
                   ncols, d_ir, nnz, nrows, cb, keys, rowcnt);
        rc = cc_radix_sort_u64(ctx, keys, alt, nnz, bits, &sorted, &passes, &B, st);
    }
    if (rc == CCGPU_OK)
        rc = cc_scan_u32(ctx, rowcnt, g->row_ptr, nrows, &B, st);
    if (rc == CCGPU_OK) {
        cuda(cudaMemcpyAsync(&m, g->row_ptr + nrows, sizeof(m), cudaMemcpyDeviceToHost, st),
             __LINE__);
        cuda(cudaStreamSynchronize(st), __LINE__);
    }
    if (rc == CCGPU_OK) {
        g->m = m;
        cuda(cudaMalloc((void **)&g->col, (size_t)(m ? m : 1) * sizeof(uint32_t)), __LINE__);
        g->col_cap = (size_t)(m ? m : 1) * sizeof(uint32_t);
    }
    if (rc == CCGPU_OK && m) {
        CC_KLAUNCH(ctx, CCK_MISC, k_csc_cols, cc_blocks(m, kCsc, grid), kCsc, 0, st, sorted, m,
                   (cb >= 64 ? ~0ull : ((1ull << cb) - 1)), g->col);
    }
    if (rc == CCGPU_OK)
        cuda(cudaStreamSynchronize(st), __LINE__);
    cc_bufs_release(&B);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (rc != CCGPU_OK) {
        ccgpu_graph_free(g);
        return rc;
    }
    *out = g;
    return CCGPU_OK;
}
