/*
 * Runtime plumbing of libccb200: per-thread error messages, device checks
 * and the scratch contexts the solvers carve their temporaries from.
 */
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "ccgpu_internal.h"

#define CCGPU_VERSION_NUM 10000

static thread_local char g_err[512];

extern "C" const char *ccgpu_last_error(void) { return g_err; }

extern "C" void ccgpu_clear_error(void) { g_err[0] = 0; }

extern "C" int ccgpu_version(void) { return CCGPU_VERSION_NUM; }

int ccgpu_set_error(int status, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return status;
}

/* The same, with C linkage, for the host C sources. */
extern "C" int ccb200_set_error(int status, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return status;
}

int ccgpu_cuda_fail(cudaError_t e, const char *what, const char *file, int line)
{
    const char *base = strrchr(file, '/');
    int st = (e == cudaErrorMemoryAllocation) ? CCGPU_ERR_OOM : CCGPU_ERR_CUDA;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        st = CCGPU_ERR_NODEVICE;
    return ccgpu_set_error(st, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e),
                           base ? base + 1 : file, line);
}

extern "C" int ccgpu_device_check(void)
{
    int dev = 0, count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return ccgpu_set_error(CCGPU_ERR_NODEVICE, "no CUDA device visible (%s)",
                               e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
    }
    CC_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    CC_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10)
        return ccgpu_set_error(CCGPU_ERR_NODEVICE,
                               "device %d is sm_%d%d; this library is built for sm_100a",
                               dev, prop.major, prop.minor);
    return CCGPU_OK;
}

/* ------------------------------------------------------------- contexts */

extern "C" int ccgpu_ctx_create(ccgpu_ctx **out)
{
    if (!out)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_ctx_create: out is NULL");
    *out = NULL;
    CC_TRY(ccgpu_device_check());
    ccgpu_ctx *c = (ccgpu_ctx *)calloc(1, sizeof(ccgpu_ctx));
    if (!c)
        return ccgpu_set_error(CCGPU_ERR_OOM, "ccgpu_ctx_create: host OOM");
    CC_CUDA(cudaGetDevice(&c->device));
    CC_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device));
    *out = c;
    return CCGPU_OK;
}

extern "C" void ccgpu_ctx_destroy(ccgpu_ctx *ctx)
{
    if (!ctx || ctx->owned_by_default)
        return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(ctx->device);
    cc_batch_cache_free(ctx);
    if (ctx->base)
        cudaFree(ctx->base);
    if (ctx->host_pinned)
        cudaFreeHost(ctx->host_pinned);
    if (ctx->cell)
        cudaFree(ctx->cell);
    if (prev >= 0)
        cudaSetDevice(prev);
    free(ctx);
}

extern "C" size_t ccgpu_ctx_scratch_bytes(const ccgpu_ctx *ctx) { return ctx ? ctx->cap : 0; }

/* One default context per (host thread, device). */
#define CC_MAX_DEVICES 64
static thread_local ccgpu_ctx *g_default_ctx[CC_MAX_DEVICES];

int ccgpu_ctx_resolve(ccgpu_ctx **ctx)
{
    if (*ctx)
        return CCGPU_OK;
    int dev = 0;
    CC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= CC_MAX_DEVICES)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "device ordinal %d above %d", dev, CC_MAX_DEVICES);
    if (!g_default_ctx[dev]) {
        ccgpu_ctx *c = NULL;
        CC_TRY(ccgpu_ctx_create(&c));
        c->owned_by_default = 1;
        g_default_ctx[dev] = c;
    }
    *ctx = g_default_ctx[dev];
    return CCGPU_OK;
}

int ccgpu_ctx_reserve(ccgpu_ctx *ctx, size_t bytes, void **base)
{
    if (bytes == 0)
        bytes = 256;
    if (bytes > ctx->cap) {
        if (ctx->base) {
            CC_CUDA(cudaFree(ctx->base)); /* implicit device sync */
            ctx->base = NULL;
            ctx->cap = 0;
        }
        size_t want = bytes + bytes / 8; /* headroom for nearby sizes */
        void *p = NULL;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            e = cudaMalloc(&p, bytes);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return ccgpu_set_error(CCGPU_ERR_OOM, "scratch: cudaMalloc(%zu) failed: %s", bytes,
                                       cudaGetErrorString(e));
            }
            want = bytes;
        }
        ctx->base = p;
        ctx->cap = want;
    }
    *base = ctx->base;
    return CCGPU_OK;
}

int ccgpu_ctx_pinned(ccgpu_ctx *ctx, size_t bytes, void **host)
{
    if (bytes > ctx->host_cap) {
        if (ctx->host_pinned)
            CC_CUDA(cudaFreeHost(ctx->host_pinned));
        ctx->host_pinned = NULL;
        ctx->host_cap = 0;
        CC_CUDA(cudaMallocHost(&ctx->host_pinned, bytes < 4096 ? 4096 : bytes));
        ctx->host_cap = bytes < 4096 ? 4096 : bytes;
    }
    *host = ctx->host_pinned;
    return CCGPU_OK;
}

int ccgpu_ctx_cell(ccgpu_ctx *ctx, unsigned long long **cell)
{
    if (!ctx->cell)
        CC_CUDA(cudaMalloc((void **)&ctx->cell, 256));
    *cell = ctx->cell;
    return CCGPU_OK;
}

/* ------------------------------------------------------------- profiler */

#include <vector>

static const char *const kKernelNames[CCK_NUM] = {
    "init", "sample", "compress", "giant", "link_rows", "link_heavy", "final_compress",
    "count_roots", "check_labels", "dist_split", "dist_fill", "dist_reps", "dist_pairs",
    "sort_hist", "sort_scan", "sort_scatter", "dist_dedup", "dist_ghosts", "dist_plan",
    "merge_init", "merge_hook", "merge_upd", "merge_exchange", "merge_exch_push",
    "dist_labels", "dist_bounds", "scan", "batch", "misc", "dist_pairs_heavy",
    "dist_pairs_bitmap", "batch_init", "batch_sample", "batch_compress", "batch_giant",
    "batch_link", "batch_heavy", "batch_final", "dist_local_count", "dist_local_fill",
    "dist_tiles", "dist_gflag", "dist_merge_keys", "merge_exch_pull",
    "dist_pairs_local"};

struct cc_prof {
    std::vector<cudaEvent_t> pool;
    size_t next = 0;
    struct Rec {
        int kid;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    cudaEvent_t open[CCK_NUM] = {};
};

static cudaEvent_t prof_event(cc_prof *p)
{
    if (p->next == p->pool.size()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess)
            return nullptr;
        p->pool.push_back(e);
    }
    return p->pool[p->next++];
}

void cc_prof_mark(ccgpu_ctx *ctx, int kid, int end, cudaStream_t st)
{
    cc_prof *p = ctx->prof;
    if (!p || kid < 0 || kid >= CCK_NUM)
        return;
    cudaEvent_t e = prof_event(p);
    if (!e)
        return;
    cudaEventRecord(e, st);
    if (!end) {
        p->open[kid] = e;
    } else if (p->open[kid]) {
        p->recs.push_back({kid, p->open[kid], e});
        p->open[kid] = nullptr;
    }
}

static void prof_free(cc_prof *p)
{
    for (cudaEvent_t e : p->pool)
        cudaEventDestroy(e);
    delete p;
}

extern "C" int ccgpu_prof_enable(ccgpu_ctx *ctx, int on)
{
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    if (on && !ctx->prof)
        ctx->prof = new cc_prof();
    if (!on && ctx->prof) {
        prof_free(ctx->prof);
        ctx->prof = nullptr;
    }
    return CCGPU_OK;
}

extern "C" int ccgpu_prof_collect(ccgpu_ctx *ctx, double *ms, uint64_t *launches)
{
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    for (int k = 0; k < CCK_NUM; ++k) {
        if (ms)
            ms[k] = 0.0;
        if (launches)
            launches[k] = 0;
    }
    cc_prof *p = ctx->prof;
    if (!p)
        return CCGPU_OK;
    for (const cc_prof::Rec &r : p->recs) {
        CC_CUDA(cudaEventSynchronize(r.b));
        float t = 0.f;
        CC_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
        if (ms)
            ms[r.kid] += t;
        if (launches)
            launches[r.kid]++;
    }
    p->recs.clear();
    p->next = 0;
    for (int k = 0; k < CCK_NUM; ++k)
        p->open[k] = nullptr;
    return CCGPU_OK;
}

extern "C" int ccgpu_prof_kernels(void) { return CCK_NUM; }

extern "C" const char *ccgpu_prof_name(int kid)
{
    return (kid >= 0 && kid < CCK_NUM) ? kKernelNames[kid] : "";
}

extern "C" uint64_t ccgpu_ctx_launches(const ccgpu_ctx *ctx)
{
    if (!ctx) {
        ccgpu_ctx *d = nullptr;
        if (ccgpu_ctx_resolve(&d) != CCGPU_OK)
            return 0;
        return d->launches;
    }
    return ctx->launches;
}
