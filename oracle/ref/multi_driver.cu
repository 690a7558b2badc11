/*
 * multi_driver.cu -- test harness: many BFS or SSSP queries in one process
 * of the reference build (oracle/_ref/bfs_multi, oracle/_ref/sssp_multi).
 * Not part of the product.
 *
 * skel.cu reads the graph, uploads it and times one call of gg_main
 * (skelapp/skel.cu:44-78), so a process answers one query and a 2 GB graph
 * costs seconds of parsing per query.  This file is the gg_main that
 * skel.cu calls.  It runs the reference's own gg_main
 * (apps/bfs/kernel.cu:380-393, apps/sssp/kernel.cu:455-480, compiled here
 * under the name gft_ref_gg_main) once per query:
 *   - sources: GFT_REF_SOURCES="s1,s2,..." (default: the -s source), each
 *     run GFT_REF_REPEAT times (default 1);
 *   - every call is timed the way skel.cu times its one call: a ggc::Timer
 *     around gg_main and a cudaDeviceSynchronize;
 *   - the kernels the call launched are timed with CUDA events
 *     (launch_wrap.cu), summed into the call's kernel-only time;
 *   - GFT_REF_DUMP=<dir> writes each query's node_data, raw int32, to
 *     <dir>/<source>.i32 for the parity check.
 * One line per query goes to stderr:
 *   oracle-ref-query source S total_ns N kernel_ms K
 * The reference's gg_main never frees its worklists.  Its first call also
 * sets up the drivers' static barriers, so that call's allocations are
 * kept; what every later call allocates is released after it
 * (launch_wrap.cu), so many queries fit in device memory.  The last query's
 * node_data stays in the device graph, which skel.cu copies back and writes
 * with -o as usual.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gg.h"
#include "Timer.h"

extern int start_node;
void gft_ref_gg_main(CSRGraphTy &hg, CSRGraphTy &gg);
extern "C" void gft_ref_time_launches(int on);
extern "C" double gft_ref_take_kernel_ms();
extern "C" void gft_ref_track_allocs(int on);
extern "C" size_t gft_ref_free_tracked();

static std::vector<int> sources_from_env()
{
    std::vector<int> out;
    const char *s = getenv("GFT_REF_SOURCES");
    if (!s || !*s) {
        out.push_back(start_node);
        return out;
    }
    std::string list(s);
    size_t pos = 0;
    while (pos < list.size()) {
        size_t comma = list.find(',', pos);
        if (comma == std::string::npos) comma = list.size();
        if (comma > pos) out.push_back(atoi(list.substr(pos, comma - pos).c_str()));
        pos = comma + 1;
    }
    return out;
}

void gg_main(CSRGraphTy &hg, CSRGraphTy &gg)
{
    std::vector<int> sources = sources_from_env();
    const char *rep = getenv("GFT_REF_REPEAT");
    int repeat = rep ? atoi(rep) : 1;
    if (repeat < 1) repeat = 1;
    const char *dump = getenv("GFT_REF_DUMP");
    std::vector<int> host;
    gft_ref_time_launches(1);
    bool first = true;
    for (int r = 0; r < repeat; r++) {
        for (int s : sources) {
            if (s < 0 || (unsigned)s >= gg.nnodes) {
                fprintf(stderr, "oracle-ref-query: source %d out of range\n", s);
                exit(1);
            }
            start_node = s;
            gft_ref_track_allocs(first ? 0 : 1);
            gft_ref_take_kernel_ms();
            ggc::Timer t("gg_main");
            t.start();
            gft_ref_gg_main(hg, gg);
            check_cuda(cudaDeviceSynchronize());
            t.stop();
            double kms = gft_ref_take_kernel_ms();
            gft_ref_track_allocs(0);
            fprintf(stderr, "oracle-ref-query source %d total_ns %llu kernel_ms %.6f\n", s,
                    (unsigned long long)t.duration(), kms);
            if (dump && r == 0) {
                host.resize(gg.nnodes);
                check_cuda(cudaMemcpy(host.data(), gg.node_data, sizeof(int) * gg.nnodes, cudaMemcpyDeviceToHost));
                std::string path = std::string(dump) + "/" + std::to_string(s) + ".i32";
                FILE *f = fopen(path.c_str(), "wb");
                if (!f || fwrite(host.data(), sizeof(int), gg.nnodes, f) != gg.nnodes) {
                    fprintf(stderr, "oracle-ref-query: cannot write %s\n", path.c_str());
                    exit(1);
                }
                fclose(f);
            }
            if (!first) gft_ref_free_tracked();
            first = false;
        }
    }
    gft_ref_time_launches(0);
}
