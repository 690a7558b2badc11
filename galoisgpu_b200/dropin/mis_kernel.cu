// mis_kernel.cu -- drop-in replacement for the reference's apps/mis/kernel.cu,
// linked with the reference's own skelapp/skel.cu and apps/mis/support.cu
// (all built with -DCSRG_TEX, as apps/mis/Makefile:7 builds them) and
// -lgft.  Provides the link contract (GGC_OPTIONS, gg_main of
// apps/mis/kernel.cu:215-231): gg_main runs this engine's MIS on the device
// graph skel uploaded and writes the reference's node_data states (1 = in
// the set, 2 = excluded) into gg.node_data, which skel copies back for
// support.cu's output(); it prints the reference's "Total steps: N" line.
// The priorities are the reference's on this device, so the set is too.
#include <cstdio>
#include <cstdlib>

#include "gg.h"
#include "gft.h"

const char *GGC_OPTIONS = "gft: persistent round-based MIS (libgft)";

static void gft_die(const char *what)
{
    fprintf(stderr, "gft: %s: %s\n", what, gft_last_error());
    exit(1);
}

void gg_main(CSRGraphTy &hg, CSRGraphTy &gg)
{
    int dev = 0;
    cudaGetDevice(&dev);
    static gft_engine *eng = nullptr;
    if (!eng && gft_engine_create(dev, &eng) != GFT_OK) gft_die("engine");
    gft_graph *g = nullptr;
    if (gft_graph_wrap(dev, gg.nnodes, gg.nedges, gg.row_start, gg.edge_dst, gg.edge_data, &g) != GFT_OK)
        gft_die("wrap");
    gft_stats st;
    const gft_status s = gft_mis(eng, g, gg.node_data, 0, nullptr, nullptr, &st);
    gft_graph_free(g);
    if (s != GFT_OK) gft_die("mis");
    if (cudaDeviceSynchronize() != cudaSuccess) gft_die("sync");
    printf("Total steps: %u\n", st.levels);
}
