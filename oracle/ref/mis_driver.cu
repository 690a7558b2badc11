/*
 * mis_driver.cu -- test harness: the gg_main of the reference MIS build
 * (oracle/_ref/mis).  Not part of the product.
 *
 * The reference's own gg_main (apps/mis/kernel.cu:215-231) runs its rounds
 * from a one-thread parent kernel, gg_main_pipe_1_gpu (:170-197), that
 * launches the round kernels and waits for each with a device-side
 * cudaDeviceSynchronize.  CUDA 12 no longer provides that call on the
 * device, and without it the parent would read the worklist length before
 * the round that sets it has run.  The same file also has the host-driven
 * loop gg_main_pipe_1 (:151-169), the same kernels in the same order.  This
 * driver does what the reference gg_main does (priorities from gen_prio_gpu
 * on kernel_sizing's grid with SEED1..SEED4, a worklist of nnodes entries,
 * "Total steps: N") and runs the rounds through that host loop.  The
 * reference's gg_main is compiled under another name (-Dgg_main=...) and
 * never called; every kernel that runs is the reference's own.
 */
#include "gg.h"
#include "ggcuda.h"

void kernel_sizing(CSRGraphTy &, dim3 &, dim3 &);
__global__ void gen_prio_gpu(CSRGraphTex graph, unsigned int *prio, unsigned int x, unsigned int y, unsigned int z,
                             unsigned int w);
void gg_main_pipe_1(CSRGraphTy &gg, int &STEPS, Shared<unsigned int> &prio, PipeContextT<WorklistT> &pipe,
                    dim3 &blocks, dim3 &threads);

void gg_main(CSRGraphTy &hg, CSRGraphTy &gg)
{
    dim3 blocks, threads;
    kernel_sizing(gg, blocks, threads);
    PipeContextT<WorklistT> pipe;
    Shared<unsigned int> prio(hg.nnodes);
    int steps = 0;
    // SEED1..SEED4 of apps/mis/kernel.cu:13-16.
    gen_prio_gpu<<<blocks, threads>>>(gg, prio.gpu_wr_ptr(), 0x12345678u, 0xabbdef12u, 0xcafe1234u, 0x09832516u);
    check_cuda(cudaDeviceSynchronize());
    pipe = PipeContextT<WorklistT>(gg.nnodes);
    gg_main_pipe_1(gg, steps, prio, pipe, blocks, threads);
    check_cuda(cudaDeviceSynchronize());
    printf("Total steps: %d\n", steps);
}
