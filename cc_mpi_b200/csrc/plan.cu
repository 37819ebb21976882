/*
 * CUDA-graph plans of the local-CC solve: the launch sequence for fixed
 * arguments is captured once on a private stream and replayed with a single
 * cudaGraphLaunch, which removes the per-kernel host launch cost (about ten
 * launches per solve).
 */
#include <cstdlib>
#include <cstring>

#include "local_cc.h"

struct ccgpu_plan {
    ccgpu_ctx *ctx;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    int kernels;
};

extern "C" void ccgpu_plan_destroy(ccgpu_plan *p)
{
    if (!p)
        return;
    if (p->exec)
        cudaGraphExecDestroy(p->exec);
    if (p->graph)
        cudaGraphDestroy(p->graph);
    ccgpu_ctx_destroy(p->ctx);
    free(p);
}

extern "C" int ccgpu_local_cc_plan(const uint64_t *d_row_ptr, const uint32_t *d_col_idx,
                                   uint32_t n, uint64_t m, uint32_t *d_labels,
                                   const ccgpu_cc_opts *opts, ccgpu_plan **out)
{
    if (!out)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_local_cc_plan: out is NULL");
    *out = nullptr;
    if (n == 0 || !d_row_ptr || !d_labels || (m > 0 && !d_col_idx))
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_local_cc_plan: empty graph or NULL");
    LocalCCArgs a = {d_row_ptr, d_col_idx, n, m, d_labels, nullptr, 1, {}, 0, 1};
    CC_TRY(cc_local_resolve_opts(opts, &a.o));
    ccgpu_plan *p = (ccgpu_plan *)calloc(1, sizeof(ccgpu_plan));
    if (!p)
        return ccgpu_set_error(CCGPU_ERR_OOM, "ccgpu_local_cc_plan: host OOM");
    int rc = ccgpu_ctx_create(&p->ctx);
    cudaStream_t st = nullptr;
    LocalCCScratch s;
    if (rc == CCGPU_OK) {
        cc_carve c = {nullptr, 0};
        cc_local_carve(&c, &s, a);
        void *base = nullptr;
        rc = ccgpu_ctx_reserve(p->ctx, c.off, &base);
        c = {(char *)base, 0};
        cc_local_carve(&c, &s, a);
    }
    if (rc == CCGPU_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "plan capture", __FILE__, __LINE__);
    }
    if (rc == CCGPU_OK) {
        const unsigned long long before = p->ctx->launches;
        int run = cc_local_run(p->ctx, a, s, st, 0, 0);
        cudaError_t e = cudaStreamEndCapture(st, &p->graph);
        if (run != CCGPU_OK)
            rc = run;
        else if (e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        p->kernels = (int)(p->ctx->launches - before);
    }
    if (rc == CCGPU_OK) {
        cudaError_t e = cudaGraphInstantiate(&p->exec, p->graph, 0);
        if (e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    }
    if (st)
        cudaStreamDestroy(st);
    if (rc != CCGPU_OK) {
        ccgpu_plan_destroy(p);
        return rc;
    }
    *out = p;
    return CCGPU_OK;
}

extern "C" int ccgpu_plan_launch(ccgpu_plan *p, void *stream)
{
    if (!p || !p->exec)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_plan_launch: no plan");
    CC_CUDA(cudaGraphLaunch(p->exec, (cudaStream_t)stream));
    p->ctx->launches += (unsigned long long)p->kernels;
    return CCGPU_OK;
}

extern "C" int ccgpu_plan_kernels(const ccgpu_plan *p)
{
    return p ? p->kernels : 0;
}
