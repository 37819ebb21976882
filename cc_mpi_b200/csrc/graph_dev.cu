/*
 * Device memory helpers and device-resident CSR graphs for the host C layer.
 */
#include <cstdlib>

#include "ccgpu_internal.h"

struct ccgpu_graph {
    uint64_t *row_ptr;
    uint32_t *col;
    uint32_t n;
    uint64_t m;
    int device;
};

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
    cudaError_t e = cudaMalloc(&g->row_ptr, ((size_t)n + 1) * sizeof(uint64_t));
    if (e == cudaSuccess)
        e = cudaMalloc(&g->col, (size_t)(m ? m : 1) * sizeof(uint32_t));
    if (e == cudaSuccess)
        e = cudaMemcpy(g->row_ptr, h_row_ptr, ((size_t)n + 1) * sizeof(uint64_t),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess && m)
        e = cudaMemcpy(g->col, h_col_idx, (size_t)m * sizeof(uint32_t), cudaMemcpyHostToDevice);
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
    cudaFree(g->row_ptr);
    cudaFree(g->col);
    free(g);
}

extern "C" const uint64_t *ccgpu_graph_row_ptr(const ccgpu_graph *g) { return g ? g->row_ptr : nullptr; }
extern "C" const uint32_t *ccgpu_graph_col_idx(const ccgpu_graph *g) { return g ? g->col : nullptr; }
extern "C" uint32_t ccgpu_graph_n(const ccgpu_graph *g) { return g ? g->n : 0; }
extern "C" uint64_t ccgpu_graph_m(const ccgpu_graph *g) { return g ? g->m : 0; }
