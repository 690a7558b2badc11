// bfs_kernel.cu -- drop-in replacement for the reference's apps/bfs/kernel.cu.
//
// Link it with the reference's own skelapp/skel.cu and apps/bfs/support.cu
// (and -lgft): skel reads the .gr file, uploads it (CSRGraph::copy_to_gpu),
// times gg_main, copies node_data back and calls output(), exactly as with
// the reference kernel; gg_main runs this engine's BFS through the C ABI on
// the device arrays skel uploaded.  Provides the link contract of
// apps/bfs/kernel.cu:10-16 (GGC_OPTIONS, INF, enable_lb) and gg_main
// (:380-393).
#include <climits>
#include <cstdio>
#include <cstdlib>

#include "gg.h"
#include "gft.h"

const char *GGC_OPTIONS = "gft: sm_100a persistent BFS (libgft)";
extern int start_node;           // apps/bfs/support.cu:10
bool enable_lb = false;          // -l is accepted; load balancing is always on
extern const int INF = INT_MAX;  // read by output()

static void gft_die(const char *what)
{
    fprintf(stderr, "gft: %s: %s\n", what, gft_last_error());
    exit(1);
}

void gg_main(CSRGraph &hg, CSRGraph &gg)
{
    int dev = 0;
    cudaGetDevice(&dev);  // the device skel selected with -g
    static gft_engine *eng = nullptr;
    if (!eng && gft_engine_create(dev, &eng) != GFT_OK) gft_die("engine");
    gft_graph *g = nullptr;  // adopts skel's device arrays, no copy
    if (gft_graph_wrap(dev, gg.nnodes, gg.nedges, gg.row_start, gg.edge_dst, gg.edge_data, &g) != GFT_OK)
        gft_die("wrap");
    const gft_status s = gft_bfs(eng, g, (uint32_t)start_node, gg.node_data, nullptr, nullptr, nullptr, nullptr);
    gft_graph_free(g);  // the wrapper only
    if (s != GFT_OK) gft_die("bfs");
}
