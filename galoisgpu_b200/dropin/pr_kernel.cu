// pr_kernel.cu -- drop-in replacement for the reference's apps/pr/kernel.cu,
// linked with the reference's own skelapp/skel.cu and apps/pr/support.cu
// (and -lgft).  Provides the link contract of apps/pr/kernel.cu:10-20
// (GGC_OPTIONS, the ALPHA and EPSILON constants, P_CURR / P_NEXT, which
// support.cu's output() reads) and gg_main (:362-389): gg_main runs this
// engine's residual-push PageRank on the device graph skel uploaded, honours
// support.cu's -x limit (MAX_ITERATIONS), copies the ranks to host memory
// for output() and prints the reference's "PR took N iterations" line.
#include <climits>
#include <cstdio>
#include <cstdlib>

#include "gg.h"
#include "gft.h"

const char *GGC_OPTIONS = "gft: persistent residual-push PageRank (libgft)";
float *P_CURR;
float *P_NEXT;
extern const float ALPHA = 0.85;     // apps/pr/kernel.cu:19; the engine uses the same value
extern const float EPSILON = 0.000001;
extern int MAX_ITERATIONS;           // apps/pr/support.cu:26
bool enable_lb = false;

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
    float *ranks = (float *)malloc((size_t)(gg.nnodes ? gg.nnodes : 1) * sizeof(float));
    if (!ranks) gft_die("host allocation");
    gft_stats st;
    const uint32_t limit = MAX_ITERATIONS < 0 ? 0u : (uint32_t)MAX_ITERATIONS;
    const gft_status s = gft_pr_host(eng, g, ranks, limit, nullptr, nullptr, &st);
    gft_graph_free(g);
    if (s != GFT_OK) gft_die("pr");
    printf("PR took %u iterations\n", st.levels);
    P_CURR = ranks;
    P_NEXT = ranks;
}
