/*
 * ingest_driver.cu -- test harness: the reference's graph ingest timed on
 * one .gr file (oracle/_ref/ingest).  Not part of the product.
 *
 * The reference reads a graph with CSRGraph::read (readFromGR,
 * rt/src/csr_graph.cu:152-241: mmap, then a serial per-edge copy loop) and
 * uploads it with copy_to_gpu (:250-261: allocOnDevice and four synchronous
 * cudaMemcpy, edge_data included even for an unweighted graph), both
 * outside the timer skel.cu prints (skelapp/skel.cu:44-78).  This driver
 * runs exactly those two calls, each under a ggc::Timer, and prints
 *   oracle-ref-ingest read_ns R upload_ns U
 * on stderr.  The CUDA context is created first, so neither time includes it.
 */
#include <cstdio>

#include "gg.h"
#include "Timer.h"

int main(int argc, char *argv[])
{
    if (argc != 2) {
        fprintf(stderr, "usage: %s graph.gr\n", argv[0]);
        return 2;
    }
    check_cuda(cudaFree(0));
    CSRGraphTy g, gg;
    ggc::Timer tr("read"), tu("upload");
    tr.start();
    if (g.read(argv[1]) != 0) return 1;
    tr.stop();
    tu.start();
    g.copy_to_gpu(gg);
    check_cuda(cudaDeviceSynchronize());
    tu.stop();
    fprintf(stderr, "oracle-ref-ingest read_ns %llu upload_ns %llu\n", (unsigned long long)tr.duration(),
            (unsigned long long)tu.duration());
    return 0;
}
