// cc_kernel.cu -- drop-in replacement for the reference's apps/cc/kernel.cu,
// linked with the reference's own skelapp/skel.cu and apps/cc/support.cu
// (and -lgft).  Provides the link contract of apps/cc/kernel.cu:10-13
// (GGC_OPTIONS, enable_lb) and gg_main (:630-723): gg_main labels the
// device graph skel uploaded through the C ABI, writing gg.node_data, and
// prints the reference's "components: N" line.  Each vertex is labelled with
// the smallest vertex id of its component; the reference's labels are
// whichever roots its racy hooks leave, so output() prints the same
// partition with canonical labels.
#include <cstdio>
#include <cstdlib>

#include "gg.h"
#include "gft.h"

const char *GGC_OPTIONS = "gft: union-find connected components (libgft)";
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
    gft_graph *g = nullptr;  // adopts skel's device arrays, no copy; not marked symmetric
    if (gft_graph_wrap(dev, gg.nnodes, gg.nedges, gg.row_start, gg.edge_dst, gg.edge_data, &g) != GFT_OK)
        gft_die("wrap");
    uint64_t comps = 0;
    const gft_status s = gft_cc(eng, g, gg.node_data, nullptr, nullptr, nullptr, &comps);
    gft_graph_free(g);
    if (s != GFT_OK) gft_die("cc");
    printf("components: %llu\n", (unsigned long long)comps);
}
