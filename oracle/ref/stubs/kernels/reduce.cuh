// Stub of ModernGPU 1.1's kernels/reduce.cuh (the library is not vendored
// with the reference).  apps/pr/kernel.cu:13 includes it but calls nothing
// from it, so no declarations are needed.  Test harness only.
#pragma once
#include "../util/mgpucontext.h"
