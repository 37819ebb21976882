/*
 * Device primitives shared by the partitioned and batched solvers: a
 * stream-ordered buffer helper, exclusive scans and the LSD radix sort of
 * 64-bit keys.
 */
#ifndef CCB200_PRIMITIVES_H
#define CCB200_PRIMITIVES_H

#include "ccgpu_internal.h"

/* Stream-ordered device buffers (cudaMallocAsync on the device's default
 * pool, whose release threshold is raised once so repeated solves reuse
 * memory instead of returning it to the driver). */
struct DevBufs {
    cudaStream_t st;
    void *ptrs[128];
    int n;
};
int cc_bufs_init(DevBufs *b, cudaStream_t st);
/* Raises the release threshold of the current device's default pool (once
 * per thread and device). */
int cc_pool_tune(void);
int cc_bufs_get(DevBufs *b, void **p, size_t bytes);
void cc_bufs_release(DevBufs *b);

/* out[i] = sum(in[0..i)) for i in [0, count]; out has count + 1 entries,
 * out[count] is the total.  in may alias out only for the u64 variant. */
int cc_scan_u32(ccgpu_ctx *ctx, const uint32_t *in, uint64_t *out, uint64_t count, DevBufs *b,
                cudaStream_t st);
int cc_scan_u64(ccgpu_ctx *ctx, const uint64_t *in, uint64_t *out, uint64_t count, DevBufs *b,
                cudaStream_t st);

/* Sorts keys[0..count) ascending on bits [0, bits) (higher bits must be
 * zero).  alt is a buffer of the same size.  *sorted receives keys or alt,
 * whichever holds the result; *passes (may be NULL) the passes run.
 * Asynchronous on st. */
int cc_radix_sort_u64(ccgpu_ctx *ctx, uint64_t *keys, uint64_t *alt, uint64_t count, int bits,
                      uint64_t **sorted, int *passes, DevBufs *b, cudaStream_t st);

/* Block-wide inclusive scan helper for 256-thread blocks. */
#ifdef __CUDACC__
template <typename T>
__device__ __forceinline__ T cc_block_incl_scan256(T v, T *s_warp /* [8] */, T *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o)
            v += y;
    }
    if (lane == 31)
        s_warp[warp] = v;
    __syncthreads();
    T pre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        T x = s_warp[w];
        pre += (w < warp) ? x : (T)0;
        tot += x;
    }
    __syncthreads();
    if (total)
        *total = tot;
    return v + pre;
}
#endif

#endif
