/*
 * compat.h -- force-included (nvcc -include) when the reference's own CUDA
 * sources are compiled for sm_100a to serve as the parity oracle.  Part of
 * the test harness, not of the product.
 *
 * The reference was written for Fermi..Pascal with CUB 1.2/1.3 and
 * ModernGPU 1.1 (reference README.md:24-39).  Nothing here changes its
 * algorithm; it only supplies names that CUDA 12.9 / CUB 2.x no longer have:
 *   - __ballot / __any (pre-Volta warp votes, rt/include/cutil_subset.h:44,52,
 *     apps/bfs/kernel.cu:209, apps/sssp/kernel.cu:221) as their _sync forms
 *     over the currently active lanes;
 *   - cub::ShuffleBroadcast (rt/include/worklist.h:364) as __shfl_sync over
 *     the active lanes;
 *   - device-side cudaDeviceSynchronize, used only by the dead
 *     dynamic-parallelism drivers gg_main_pipe_1_gpu (apps/bfs/kernel.cu:335,
 *     apps/sssp/kernel.cu:392) whose launch is commented out; CUDA 12 removed
 *     it from device code, so on the device it becomes a no-op and on the
 *     host it is the normal call.
 * CUB must be included before the macros are defined (they would otherwise
 * rewrite libcu++ internals).
 */
#pragma once
#include <cuda_runtime.h>
#include <cub/cub.cuh>

namespace cub {
template <typename T>
__device__ __forceinline__ T ShuffleBroadcast(T input, int src_lane)
{
    return __shfl_sync(__activemask(), input, src_lane);
}
}  // namespace cub

#define __ballot(p) __ballot_sync(__activemask(), (p))
#define __any(p) __any_sync(__activemask(), (p))

static __host__ __device__ inline cudaError_t ref_compat_device_sync()
{
#ifdef __CUDA_ARCH__
    return cudaSuccess;
#else
    return (cudaDeviceSynchronize)();
#endif
}
#define cudaDeviceSynchronize() ref_compat_device_sync()
