/*
 * Stub of ModernGPU 1.1's kernels/mergesort.cuh.  Declared so that
 * rt/include/worklist.h:141-147 and rt/include/aolist.h:48 compile; the
 * BFS/SSSP path never sorts a worklist, and calling these aborts.
 */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <util/mgpucontext.h>

namespace mgpu {
template <typename K, typename C>
void MergesortKeys(K *, int, C, CudaContext &)
{
    fprintf(stderr, "mgpu::MergesortKeys is not available in this build\n");
    abort();
}
template <typename K, typename V, typename C>
void MergesortPairs(K *, V *, int, C, CudaContext &)
{
    fprintf(stderr, "mgpu::MergesortPairs is not available in this build\n");
    abort();
}
}  // namespace mgpu
using mgpu::MergesortKeys;
using mgpu::MergesortPairs;
