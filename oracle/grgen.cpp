// grgen.cpp -- the seeded synthetic input graphs as a library of their own
// (oracle/libgrgen.so).  TEST AND MEASUREMENT INFRASTRUCTURE ONLY.
//
// bench.py's reference arm times the reference's own CUDA build on the same
// seeded graphs as the engine's arm, and it must not load the engine library
// to do so.  This file links the engine's host generators
// (galoisgpu_b200/csrc/gen_host.cpp, compiled in unchanged, so the graphs
// are the same by construction) with the two functions that file expects
// from the engine (error reporting and gft_csr_free), plus a .gr v1 writer
// with the layout CSRGraph::readFromGR parses (rt/src/csr_graph.cu:187-228):
// four little-endian u64 (version 1, sizeEdgeTy, numNodes, numEdges), u64
// end offsets per node, u32 destinations, a u32 pad when numEdges is odd,
// then u32 weights when sizeEdgeTy is 4.
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "gft.h"

namespace gft {

static thread_local char g_err[512];

gft_status fail(gft_status s, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return s;
}

}  // namespace gft

extern "C" {

void gft_csr_free(gft_csr *g)
{
    if (!g) return;
    free(g->row_start);
    free(g->edge_dst);
    free(g->edge_data);
    memset(g, 0, sizeof *g);
}

const char *grgen_last_error(void) { return gft::g_err; }

// Writes g as a .gr v1 file; 0 on success.
int grgen_write_gr(const char *path, const gft_csr *g)
{
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    uint64_t hdr[4] = {1, g->edge_data ? 4ull : 0ull, g->nnodes, g->nedges};
    bool ok = fwrite(hdr, sizeof hdr, 1, f) == 1;
    std::vector<uint64_t> end(g->nnodes);
    for (uint32_t i = 0; i < g->nnodes; i++) end[i] = g->row_start[i + 1];
    ok = ok && fwrite(end.data(), 8, g->nnodes, f) == g->nnodes;
    ok = ok && fwrite(g->edge_dst, 4, g->nedges, f) == g->nedges;
    if (ok && (g->nedges & 1)) {
        uint32_t pad = 0;
        ok = fwrite(&pad, 4, 1, f) == 1;
    }
    if (ok && g->edge_data) ok = fwrite(g->edge_data, 4, g->nedges, f) == g->nedges;
    if (fclose(f) != 0) ok = false;
    return ok ? 0 : -1;
}

}  // extern "C"
