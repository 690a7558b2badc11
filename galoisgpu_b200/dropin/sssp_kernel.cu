// sssp_kernel.cu -- drop-in replacement for the reference's
// apps/sssp/kernel.cu, linked with the reference's own skelapp/skel.cu and
// apps/sssp/support.cu (and -lgft).  Provides the link contract of
// apps/sssp/kernel.cu:10-18 (GGC_OPTIONS, INF, enable_lb) and gg_main
// (:455-480), which runs this engine's SSSP with the -d delta that
// support.cu parsed, on the device arrays skel uploaded.  Like the
// reference it prints "delta: D" and "iterations: N" (phases run).
#include <climits>
#include <cstdio>
#include <cstdlib>

#include "gg.h"
#include "gft.h"

const char *GGC_OPTIONS = "gft: sm_100a persistent near-far SSSP (libgft)";
extern int DELTA;                // apps/sssp/support.cu:10
extern int start_node;           // apps/sssp/support.cu:12
bool enable_lb = false;
extern const int INF = INT_MAX;

static void gft_die(const char *what)
{
    fprintf(stderr, "gft: %s: %s\n", what, gft_last_error());
    exit(1);
}

void gg_main(CSRGraph &hg, CSRGraph &gg)
{
    int dev = 0;
    cudaGetDevice(&dev);
    static gft_engine *eng = nullptr;
    if (!eng && gft_engine_create(dev, &eng) != GFT_OK) gft_die("engine");
    gft_graph *g = nullptr;
    if (gft_graph_wrap(dev, gg.nnodes, gg.nedges, gg.row_start, gg.edge_dst, gg.edge_data, &g) != GFT_OK)
        gft_die("wrap");
    printf("delta: %d\n", DELTA);
    gft_stats st;
    const gft_status s =
        gft_sssp(eng, g, (uint32_t)start_node, DELTA, gg.node_data, nullptr, nullptr, nullptr, &st);
    gft_graph_free(g);
    if (s != GFT_OK) gft_die("sssp");
    printf("iterations: %u\n", st.levels);
}
