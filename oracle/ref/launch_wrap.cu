/*
 * launch_wrap.cu -- linked into the reference oracle build with
 * -Xlinker --wrap=cudaLaunchKernel,--wrap=cudaMalloc,--wrap=cudaFree.  Test
 * harness only.
 *
 * 1. Cooperative launch of the persistent drivers.
 * The reference's persistent drivers gg_main_pipe_N_gpu_gb
 * (apps/bfs/kernel.cu:375, apps/sssp/kernel.cu:448, apps/cc/kernel.cu:481,569,
 * apps/pr/kernel.cu:271)
 * synchronise their CTAs
 * with a software grid barrier that spins without a limit
 * (rt/include/gbar.cuh:84-120), sized by a hand-written occupancy table
 * (rt/include/cuda_launch_config.hpp:205-265).  A grid that is not fully
 * co-resident would hang.  This wrapper launches exactly those kernels with
 * cudaLaunchCooperativeKernel instead: same grid, same block, same
 * arguments, so the same results, but the driver refuses a grid that cannot
 * be co-resident (cudaErrorCooperativeLaunchTooLarge) instead of letting it
 * spin.  Every other launch passes through unchanged.
 *
 * 2. Padded device allocations.
 * The reference's BFS visit is a racy check-then-write
 * (apps/bfs/kernel.cu:194-199) and its SSSP relaxation pushes whenever the
 * unsynchronised check passes (apps/sssp/kernel.cu:246-258), so a vertex can
 * be pushed several times in one iteration, while the BFS queue holds only
 * nnodes entries (apps/bfs/kernel.cu:389) and is guarded by a device assert
 * (rt/include/worklist.h:349-368).  Every cudaMalloc is padded (4x the
 * request plus 16 MiB) and the logical capacity each worklist records at
 * construction (init_wl, rt/include/worklist.h:35-40, launched from the
 * Worklist constructor :93) is raised to the padded size, so a burst of
 * duplicates lands in memory the queue owns instead of tripping the device
 * assert or overwriting a neighbouring allocation; the assert still guards
 * the padded bound.  Duplicate entries do not change results: they carry
 * the same BFS level, or a distance that is simply relaxed again.
 *
 * 3. Optional instruments for the many-query driver (multi_driver.cu); both
 * are off unless that driver switches them on, so the plain bfs/sssp/cc/pr
 * builds behave as before.
 *   - Launch timing: CUDA events around every launch on its own stream, the
 *     device time summed until gft_ref_take_kernel_ms() reads it.  The host
 *     waits for each timed launch to end; the reference waits for each of
 *     its launches anyway (a cudaDeviceSynchronize or a blocking cudaMemcpy
 *     follows every one on this path).
 *   - Allocation tracking: device allocations made while tracking is on are
 *     remembered so that gft_ref_free_tracked() can release them.  The
 *     reference's gg_main never frees its worklists; without this, a process
 *     answering many queries would run out of device memory.
 */
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <vector>

static bool g_time_launches = false;
static double g_kernel_ms = 0.0;
static cudaEvent_t g_ev0, g_ev1;
static bool g_track_allocs = false;
static std::vector<void *> g_tracked;

extern "C" void gft_ref_time_launches(int on)
{
    if (on && !g_ev0) {
        cudaEventCreate(&g_ev0);
        cudaEventCreate(&g_ev1);
    }
    g_time_launches = on != 0;
}

extern "C" double gft_ref_take_kernel_ms()
{
    double ms = g_kernel_ms;
    g_kernel_ms = 0.0;
    return ms;
}

extern "C" void gft_ref_track_allocs(int on) { g_track_allocs = on != 0; }

extern "C" size_t gft_ref_free_tracked()
{
    std::vector<void *> mine;
    mine.swap(g_tracked);
    for (void *p : mine) cudaFree(p);
    return mine.size();
}

static cudaError_t timed(cudaError_t (*launch)(const void *, dim3, dim3, void **, size_t, cudaStream_t),
                         const void *func, dim3 grid, dim3 block, void **args, size_t smem, cudaStream_t stream)
{
    if (!g_time_launches) return launch(func, grid, block, args, smem, stream);
    cudaEventRecord(g_ev0, stream);
    cudaError_t e = launch(func, grid, block, args, smem, stream);
    if (e != cudaSuccess) return e;
    cudaEventRecord(g_ev1, stream);
    if (cudaEventSynchronize(g_ev1) == cudaSuccess) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, g_ev0, g_ev1) == cudaSuccess) g_kernel_ms += ms;
    }
    return e;
}

static cudaError_t coop_launch(const void *func, dim3 grid, dim3 block, void **args, size_t smem,
                               cudaStream_t stream)
{
    return cudaLaunchCooperativeKernel(func, grid, block, args, smem, stream);
}

extern "C" cudaError_t __real_cudaLaunchKernel(const void *func, dim3 grid, dim3 block, void **args,
                                               size_t smem, cudaStream_t stream);

extern "C" cudaError_t __wrap_cudaLaunchKernel(const void *func, dim3 grid, dim3 block, void **args,
                                               size_t smem, cudaStream_t stream)
{
    const char *name = nullptr;
    if (cudaFuncGetName(&name, func) == cudaSuccess && name && strstr(name, "init_wl") && args && args[0]) {
        int *size = static_cast<int *>(args[0]);
        long long padded = (long long)*size * 4 + (4ll << 20);  // ints in the padded dwl allocation
        *size = (int)(padded > 0x7FFFFFFFll ? 0x7FFFFFFFll : padded);
    }
    if (name && strstr(name, "_gpu_gb")) {  // gg_main_pipe_N_gpu_gb: bfs, sssp, cc, pr
        cudaError_t e = timed(coop_launch, func, grid, block, args, smem, stream);
        if (e != cudaSuccess)
            fprintf(stderr, "oracle-ref: cooperative launch of %s (%u x %u) refused: %s\n", name, grid.x,
                    block.x, cudaGetErrorString(e));
        return e;
    }
    return timed(__real_cudaLaunchKernel, func, grid, block, args, smem, stream);
}

extern "C" cudaError_t __real_cudaMalloc(void **ptr, size_t size);

extern "C" cudaError_t __wrap_cudaMalloc(void **ptr, size_t size)
{
    const size_t pad = size * 3 + ((size_t)16 << 20);
    cudaError_t e = __real_cudaMalloc(ptr, size + pad);
    if (e == cudaSuccess && g_track_allocs) g_tracked.push_back(*ptr);
    return e;
}

// Pass-through, except that a tracked allocation the reference frees itself
// (the drivers' one-int cl_* cells) is forgotten, so it is not freed twice.
extern "C" cudaError_t __real_cudaFree(void *ptr);

extern "C" cudaError_t __wrap_cudaFree(void *ptr)
{
    for (size_t i = 0; i < g_tracked.size(); i++)
        if (g_tracked[i] == ptr) {
            g_tracked[i] = g_tracked.back();
            g_tracked.pop_back();
            break;
        }
    return __real_cudaFree(ptr);
}
