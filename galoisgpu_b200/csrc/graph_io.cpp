// graph_io.cpp -- .gr binary CSR reader/writer, output text writer and the
// library's error reporting.
//
// The .gr v1 layout is the one CSRGraph::readFromGR parses
// (rt/src/csr_graph.cu:187-228): header of four little-endian u64 (version,
// sizeEdgeTy, numNodes, numEdges), u64 outIdx[numNodes] holding the END
// offset of each node's edges, u32 outs[numEdges], a u32 pad when numEdges
// is odd, then u32 edge data when sizeEdgeTy != 0.  The reference copies it
// edge by edge in a serial loop (:210-228); here the sections are read in
// bulk and validated by all host threads.
#include <errno.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>

#include "gft_internal.h"

namespace gft {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

gft_status fail(gft_status s, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

// Runs f(begin, end) over [0, n) on up to hardware_concurrency threads.
template <typename F>
static void parallel_for(uint64_t n, F f)
{
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    if (n < (1u << 16) || nt == 1) {
        f(0, n);
        return;
    }
    nt = std::min<unsigned>(nt, 64);
    std::vector<std::thread> th;
    uint64_t chunk = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        uint64_t b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([=] { f(b, e); });
    }
    for (auto &x : th) x.join();
}

static bool read_all(FILE *f, void *dst, size_t bytes)
{
    char *p = (char *)dst;
    while (bytes) {
        size_t chunk = std::min<size_t>(bytes, (size_t)1 << 28);
        size_t got = fread(p, 1, chunk, f);
        if (got != chunk) return false;
        p += got;
        bytes -= got;
    }
    return true;
}

static bool write_all(FILE *f, const void *src, size_t bytes)
{
    const char *p = (const char *)src;
    while (bytes) {
        size_t chunk = std::min<size_t>(bytes, (size_t)1 << 28);
        if (fwrite(p, 1, chunk, f) != chunk) return false;
        p += chunk;
        bytes -= chunk;
    }
    return true;
}

}  // namespace gft

using namespace gft;

extern "C" {

int gft_version(void) { return GFT_VERSION; }

const char *gft_last_error(void) { return g_last_error.c_str(); }

const char *gft_status_string(gft_status s)
{
    switch (s) {
    case GFT_OK: return "ok";
    case GFT_ERR_INVALID_ARG: return "invalid argument";
    case GFT_ERR_IO: return "i/o error";
    case GFT_ERR_FORMAT: return "malformed .gr file";
    case GFT_ERR_CUDA: return "CUDA error";
    case GFT_ERR_OOM: return "out of memory";
    case GFT_ERR_TIMEOUT: return "device wait timed out";
    case GFT_ERR_OVERFLOW: return "capacity or range exceeded";
    case GFT_ERR_NOT_SUPPORTED: return "not supported";
    case GFT_ERR_BUSY: return "busy";
    }
    return "unknown status";
}

void gft_csr_free(gft_csr *g)
{
    if (!g) return;
    free(g->row_start);
    free(g->edge_dst);
    free(g->edge_data);
    memset(g, 0, sizeof *g);
}

gft_status gft_gr_read(const char *path, gft_csr *out)
{
    if (!path || !out) return fail(GFT_ERR_INVALID_ARG, "gft_gr_read: null argument");
    memset(out, 0, sizeof *out);
    FILE *f = fopen(path, "rb");
    if (!f) return fail(GFT_ERR_IO, "gft_gr_read: cannot open %s: %s", path, strerror(errno));
    uint64_t hdr[4];
    if (!read_all(f, hdr, sizeof hdr)) {
        fclose(f);
        return fail(GFT_ERR_FORMAT, "gft_gr_read: %s: truncated header", path);
    }
    if (hdr[0] != 1) {
        fclose(f);
        return fail(GFT_ERR_FORMAT, "gft_gr_read: %s: version %llu, expected 1", path, (unsigned long long)hdr[0]);
    }
    uint64_t size_edge_ty = hdr[1], nn = hdr[2], ne = hdr[3];
    if (size_edge_ty != 0 && size_edge_ty != 4) {
        fclose(f);
        return fail(GFT_ERR_FORMAT, "gft_gr_read: %s: sizeEdgeTy %llu unsupported (0 or 4)", path,
                    (unsigned long long)size_edge_ty);
    }
    if (nn >= 0xFFFFFFFFull || ne >= 0xFFFFFFFFull) {
        fclose(f);
        return fail(GFT_ERR_FORMAT, "gft_gr_read: %s: %llu nodes / %llu edges exceed 32-bit ids", path,
                    (unsigned long long)nn, (unsigned long long)ne);
    }
    uint64_t *out_idx = (uint64_t *)malloc(std::max<uint64_t>(nn, 1) * 8);
    out->row_start = (uint32_t *)malloc((nn + 1) * 4);
    out->edge_dst = (uint32_t *)malloc(std::max<uint64_t>(ne, 1) * 4);
    if (size_edge_ty) out->edge_data = (int32_t *)malloc(std::max<uint64_t>(ne, 1) * 4);
    if (!out_idx || !out->row_start || !out->edge_dst || (size_edge_ty && !out->edge_data)) {
        free(out_idx);
        fclose(f);
        gft_csr_free(out);
        return fail(GFT_ERR_OOM, "gft_gr_read: host allocation failed");
    }
    bool ok = read_all(f, out_idx, nn * 8) && read_all(f, out->edge_dst, ne * 4);
    if (ok && size_edge_ty) {
        uint32_t pad;
        if (ne % 2) ok = read_all(f, &pad, 4);
        // Weights are u32 on disk and int in memory (csr_graph.cu:199,223-224).
        ok = ok && read_all(f, out->edge_data, ne * 4);
    }
    fclose(f);
    if (!ok) {
        free(out_idx);
        gft_csr_free(out);
        return fail(GFT_ERR_FORMAT, "gft_gr_read: %s: truncated file", path);
    }
    out->nnodes = (uint32_t)nn;
    out->nedges = (uint32_t)ne;
    std::atomic<int> bad_idx{0};
    out->row_start[0] = 0;
    parallel_for(nn, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            uint64_t prev = i ? out_idx[i - 1] : 0;
            if (out_idx[i] < prev || out_idx[i] > ne) bad_idx.store(1, std::memory_order_relaxed);
            out->row_start[i + 1] = (uint32_t)out_idx[i];
        }
    });
    if (nn && out_idx[nn - 1] != ne) bad_idx = 1;
    if (!nn && ne) bad_idx = 1;
    free(out_idx);
    if (bad_idx) {
        gft_csr_free(out);
        return fail(GFT_ERR_FORMAT, "gft_gr_read: %s: outIdx is not a monotone end-offset array ending at numEdges",
                    path);
    }
    std::atomic<uint64_t> bad_edge{~0ull};
    const uint32_t *dst = out->edge_dst;
    parallel_for(ne, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++)
            if (dst[i] >= nn) {
                uint64_t cur = bad_edge.load();
                while (i < cur && !bad_edge.compare_exchange_weak(cur, i)) {
                }
                break;
            }
    });
    if (bad_edge.load() != ~0ull) {
        uint64_t i = bad_edge.load();
        gft_status s = fail(GFT_ERR_FORMAT, "gft_gr_read: %s: edge %llu has destination %u >= numNodes %llu", path,
                            (unsigned long long)i, out->edge_dst[i], (unsigned long long)nn);
        gft_csr_free(out);
        return s;
    }
    clear_error();
    return GFT_OK;
}

gft_status gft_gr_write(const char *path, const gft_csr *g)
{
    if (!path || !g || !g->row_start || (g->nedges && !g->edge_dst))
        return fail(GFT_ERR_INVALID_ARG, "gft_gr_write: null argument");
    if (g->row_start[0] != 0 || g->row_start[g->nnodes] != g->nedges)
        return fail(GFT_ERR_INVALID_ARG, "gft_gr_write: row_start must run from 0 to nedges");
    FILE *f = fopen(path, "wb");
    if (!f) return fail(GFT_ERR_IO, "gft_gr_write: cannot open %s: %s", path, strerror(errno));
    uint64_t hdr[4] = {1, g->edge_data ? 4ull : 0ull, g->nnodes, g->nedges};
    bool ok = write_all(f, hdr, sizeof hdr);
    std::vector<uint64_t> out_idx(g->nnodes);
    for (uint32_t i = 0; i < g->nnodes; i++) out_idx[i] = g->row_start[i + 1];
    ok = ok && write_all(f, out_idx.data(), (size_t)g->nnodes * 8);
    ok = ok && write_all(f, g->edge_dst, (size_t)g->nedges * 4);
    if (ok && (g->nedges % 2)) {
        uint32_t pad = 0;
        ok = write_all(f, &pad, 4);
    }
    if (ok && g->edge_data) ok = write_all(f, g->edge_data, (size_t)g->nedges * 4);
    if (fclose(f) != 0) ok = false;
    if (!ok) return fail(GFT_ERR_IO, "gft_gr_write: write to %s failed", path);
    return GFT_OK;
}

gft_status gft_write_output(const char *path, uint32_t nnodes, const int32_t *h_val)
{
    if (!path || (nnodes && !h_val)) return fail(GFT_ERR_INVALID_ARG, "gft_write_output: null argument");
    bool to_stdout = strcmp(path, "-") == 0;
    FILE *f = to_stdout ? stdout : fopen(path, "w");
    if (!f) return fail(GFT_ERR_IO, "gft_write_output: cannot open %s: %s", path, strerror(errno));
    // Formatted in parallel blocks, written in order.  Lines are
    // "%d %d\n" or "%d INF\n" (apps/bfs/support.cu:39-45).
    const uint32_t block = 1u << 20;
    uint32_t nblocks = (nnodes + block - 1) / block;
    bool ok = true;
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (uint32_t b0 = 0; b0 < nblocks && ok; b0 += nt) {
        uint32_t nb = std::min<uint32_t>(nt, nblocks - b0);
        std::vector<std::string> text(nb);
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < nb; t++)
            th.emplace_back([&, t] {
                uint32_t lo = (b0 + t) * block, hi = std::min<uint32_t>(nnodes, lo + block);
                std::string &s = text[t];
                s.reserve((size_t)(hi - lo) * 16);
                char line[48];
                for (uint32_t i = lo; i < hi; i++) {
                    int n = h_val[i] == GFT_INF ? snprintf(line, sizeof line, "%d INF\n", (int)i)
                                                : snprintf(line, sizeof line, "%d %d\n", (int)i, h_val[i]);
                    s.append(line, n);
                }
            });
        for (auto &x : th) x.join();
        for (auto &s : text) ok = ok && write_all(f, s.data(), s.size());
    }
    if (to_stdout) fflush(f);
    else if (fclose(f) != 0) ok = false;
    if (!ok) return fail(GFT_ERR_IO, "gft_write_output: write to %s failed", path);
    return GFT_OK;
}

gft_status gft_write_cc_output(const char *path, const gft_csr *g, const int32_t *h_label)
{
    if (!path || !g || !g->row_start || (g->nnodes && !h_label) || (g->nedges && !g->edge_dst))
        return fail(GFT_ERR_INVALID_ARG, "gft_write_cc_output: null argument");
    bool to_stdout = strcmp(path, "-") == 0;
    FILE *f = to_stdout ? stdout : fopen(path, "w");
    if (!f) return fail(GFT_ERR_IO, "gft_write_cc_output: cannot open %s: %s", path, strerror(errno));
    // apps/cc/support.cu:16-36: per node "%d %d\n" (id, label), then per
    // out-edge j "\te %d: %d %d %d\n" (j, dst, edge_data[j], label[dst]);
    // edge_data is 0 for an unweighted graph.  Formatted in parallel blocks of
    // nodes, written in order.
    const uint32_t n = g->nnodes, block = 1u << 18;
    uint32_t nblocks = (n + block - 1) / block;
    bool ok = true;
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (uint32_t b0 = 0; b0 < nblocks && ok; b0 += nt) {
        uint32_t nb = std::min<uint32_t>(nt, nblocks - b0);
        std::vector<std::string> text(nb);
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < nb; t++)
            th.emplace_back([&, t] {
                uint32_t lo = (b0 + t) * block, hi = std::min<uint32_t>(n, lo + block);
                std::string &s = text[t];
                s.reserve((size_t)(hi - lo) * 16 + (size_t)(g->row_start[hi] - g->row_start[lo]) * 32);
                char line[96];
                for (uint32_t i = lo; i < hi; i++) {
                    s.append(line, snprintf(line, sizeof line, "%d %d\n", (int)i, h_label[i]));
                    for (uint32_t j = g->row_start[i]; j < g->row_start[i + 1]; j++) {
                        const uint32_t d = g->edge_dst[j];
                        s.append(line, snprintf(line, sizeof line, "\te %d: %d %d %d\n", (int)j, (int)d,
                                                g->edge_data ? g->edge_data[j] : 0, h_label[d]));
                    }
                }
            });
        for (auto &x : th) x.join();
        for (auto &s : text) ok = ok && write_all(f, s.data(), s.size());
    }
    if (to_stdout) fflush(f);
    else if (fclose(f) != 0) ok = false;
    if (!ok) return fail(GFT_ERR_IO, "gft_write_cc_output: write to %s failed", path);
    return GFT_OK;
}

gft_status gft_write_pr_output(const char *path, uint32_t nnodes, const float *h_rank)
{
    if (!path || (nnodes && !h_rank)) return fail(GFT_ERR_INVALID_ARG, "gft_write_pr_output: null argument");
    bool to_stdout = strcmp(path, "-") == 0;
    FILE *f = to_stdout ? stdout : fopen(path, "w");
    if (!f) return fail(GFT_ERR_IO, "gft_write_pr_output: cannot open %s: %s", path, strerror(errno));
    // "%d %f\n" per node, node order (apps/pr/support.cu:95-101); formatted in
    // parallel blocks, written in order.
    const uint32_t block = 1u << 20;
    uint32_t nblocks = (nnodes + block - 1) / block;
    bool ok = true;
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (uint32_t b0 = 0; b0 < nblocks && ok; b0 += nt) {
        uint32_t nb = std::min<uint32_t>(nt, nblocks - b0);
        std::vector<std::string> text(nb);
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < nb; t++)
            th.emplace_back([&, t] {
                uint32_t lo = (b0 + t) * block, hi = std::min<uint32_t>(nnodes, lo + block);
                std::string &s = text[t];
                s.reserve((size_t)(hi - lo) * 20);
                char line[64];
                for (uint32_t i = lo; i < hi; i++) s.append(line, snprintf(line, sizeof line, "%d %f\n", (int)i, (double)h_rank[i]));
            });
        for (auto &x : th) x.join();
        for (auto &s : text) ok = ok && write_all(f, s.data(), s.size());
    }
    if (to_stdout) fflush(f);
    else if (fclose(f) != 0) ok = false;
    if (!ok) return fail(GFT_ERR_IO, "gft_write_pr_output: write to %s failed", path);
    return GFT_OK;
}

gft_status gft_write_mis_output(const char *path, uint32_t nnodes, const int32_t *h_state)
{
    if (!path || (nnodes && !h_state)) return fail(GFT_ERR_INVALID_ARG, "gft_write_mis_output: null argument");
    bool to_stdout = strcmp(path, "-") == 0;
    FILE *f = to_stdout ? stdout : fopen(path, "w");
    if (!f) return fail(GFT_ERR_IO, "gft_write_mis_output: cannot open %s: %s", path, strerror(errno));
    // The set's size, then its member ids in order (apps/mis/support.cu:
    // 29-37); members are state 1.
    unsigned count = 0;
    for (uint32_t i = 0; i < nnodes; i++) count += h_state[i] == 1;
    std::string s;
    s.reserve((size_t)count * 9 + 16);
    char line[32];
    s.append(line, snprintf(line, sizeof line, "%u\n", count));
    bool ok = true;
    for (uint32_t i = 0; i < nnodes && ok; i++) {
        if (h_state[i] == 1) s.append(line, snprintf(line, sizeof line, "%d\n", (int)i));
        if (s.size() >= (1u << 24)) {
            ok = write_all(f, s.data(), s.size());
            s.clear();
        }
    }
    ok = ok && write_all(f, s.data(), s.size());
    if (to_stdout) fflush(f);
    else if (fclose(f) != 0) ok = false;
    if (!ok) return fail(GFT_ERR_IO, "gft_write_mis_output: write to %s failed", path);
    return GFT_OK;
}

}  // extern "C"
