/*
 * Stub of ModernGPU 1.1's util/mgpucontext.h (not vendored by the
 * reference, README.md:29).  The BFS/SSSP path only constructs a context
 * (skelapp/skel.cu:147-148); the sort entry points that use it
 * (rt/include/worklist.h:141-147) are never called on this path.
 */
#pragma once
#include <memory>
#include <string>
#include <cstdio>
#include <cuda_runtime.h>

namespace mgpu {
struct CudaContext {
    int device = 0;
    std::string DeviceString() const
    {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return "unknown";
        char buf[256];
        snprintf(buf, sizeof buf, "%s (sm_%d%d, %d SMs)", p.name, p.major, p.minor, p.multiProcessorCount);
        return buf;
    }
};
typedef std::shared_ptr<CudaContext> ContextPtr;
inline ContextPtr CreateCudaDevice(int dev)
{
    ContextPtr c = std::make_shared<CudaContext>();
    c->device = dev;
    return c;
}
template <typename T> struct less {
    __host__ __device__ bool operator()(T a, T b) const { return a < b; }
};
}  // namespace mgpu
