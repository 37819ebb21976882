/*
 * ccgpu_local_cc_noalloc: the local CC solve for callers that cannot
 * allocate device memory.
 *
 * Some callers cannot call cudaMalloc: serving processes whose memory
 * manager reserved the whole HBM budget up front, plug-ins that must not own
 * device memory of their own, and latency-critical loops that must not take
 * the device-wide synchronisation cudaMalloc/cudaFree imply.  This variant keeps the solve's
 * scratch - the work counters, the giant root and the heavy-row queue - in a
 * file-scope device array of fixed size, so the caller only passes the graph
 * and the label buffer.
 *
 * Set-up: the first call on a device looks up the array's device address
 * with cudaGetSymbolAddress (with that device current) and caches it; make
 * that first call before any stream capture.  Every later call on the device
 * reuses the same array, which keeps the previous call's contents; the init
 * kernel clears the counters each call, everything else is written before it
 * is read.  Calls whose kernels overlap on the GPU (two streams, or two host
 * threads) share the array and race: serialise them.  The cached address
 * belongs to the device's current context: after cudaDeviceReset the module
 * may be loaded elsewhere, so the call must not be used after a reset in
 * the same process.
 */
#include <cstdint>
#include <cstring>
#include <mutex>

#include "local_cc.h"

#define CCGPU_NOALLOC_SCRATCH_BYTES (1u << 20)

/* Every GPU that loads the library holds this array until the process exits. */
static __device__ __align__(256) unsigned char g_cc_noalloc_scratch[CCGPU_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;

struct DeviceState {
    bool ready;
    void *scratch; /* device address of g_cc_noalloc_scratch */
    ccgpu_ctx ctx; /* launch bookkeeping only: no arena, never freed */
};

DeviceState g_state[kMaxDevices];
std::mutex g_mu;

int setup(int dev, DeviceState **out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceState &s = g_state[dev];
    if (!s.ready) {
        void *p = nullptr;
        CC_CUDA(cudaGetSymbolAddress(&p, g_cc_noalloc_scratch));
        int sms = 0;
        CC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        memset(&s.ctx, 0, sizeof(s.ctx));
        s.ctx.device = dev;
        s.ctx.sm_count = sms;
        s.ctx.owned_by_default = 1;
        s.scratch = p;
        s.ready = true;
    }
    *out = &s;
    return CCGPU_OK;
}

size_t required_bytes(const LocalCCArgs &a)
{
    LocalCCScratch s;
    cc_carve c = {nullptr, 0};
    cc_local_carve(&c, &s, a);
    return c.off;
}

} // namespace

extern "C" size_t ccgpu_local_cc_noalloc_capacity(void)
{
    return CCGPU_NOALLOC_SCRATCH_BYTES;
}

extern "C" size_t ccgpu_local_cc_noalloc_required(uint32_t n, uint64_t m,
                                                  const ccgpu_cc_opts *opts)
{
    LocalCCArgs a = {nullptr, nullptr, n, m, nullptr, nullptr, 1, {}, 0};
    if (cc_local_resolve_opts(opts, &a.o) != CCGPU_OK)
        return SIZE_MAX; /* invalid options: never fits (the error is set) */
    return required_bytes(a);
}

extern "C" int ccgpu_local_cc_noalloc(const uint64_t *d_row_ptr, const uint32_t *d_col_idx,
                                      uint32_t n, uint64_t m, uint32_t *d_labels,
                                      const ccgpu_cc_opts *opts, void *stream)
{
    if (n == 0)
        return CCGPU_OK;
    if (!d_row_ptr || !d_labels || (m > 0 && !d_col_idx))
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_local_cc_noalloc: NULL argument");
    if (n == 0xffffffffu)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "ccgpu_local_cc_noalloc: n must be below 2^32-1");
    LocalCCArgs a = {d_row_ptr, d_col_idx, n, m, d_labels, nullptr, 1, {}, 0};
    CC_TRY(cc_local_resolve_opts(opts, &a.o));
    const size_t need = required_bytes(a);
    if (need > CCGPU_NOALLOC_SCRATCH_BYTES)
        return ccgpu_set_error(CCGPU_ERR_LIMIT,
                               "ccgpu_local_cc_noalloc: this graph needs %zu bytes of scratch "
                               "(heavy-row queue of m/heavy_degree+1 entries), above the fixed "
                               "%u bytes; raise heavy_degree or use ccgpu_local_cc",
                               need, CCGPU_NOALLOC_SCRATCH_BYTES);
    int dev = 0;
    CC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "ccgpu_local_cc_noalloc: device %d above %d", dev,
                               kMaxDevices);
    DeviceState *s = nullptr;
    CC_TRY(setup(dev, &s));
    LocalCCScratch ls;
    cc_carve c = {(char *)s->scratch, 0};
    cc_local_carve(&c, &ls, a);
    return cc_local_run(&s->ctx, a, ls, (cudaStream_t)stream, 0, 0);
}
