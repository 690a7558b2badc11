// output.cpp -- compressed text and binary dumps of result arrays
// (gft_write_output_gz, gft_write_node_data, gft_read_node_data).
//
// The reference writes a result as text, one fprintf per vertex
// (apps/bfs/support.cu:27-45, apps/sssp/support.cu:34-53): ~250 MB for a
// 16.8 M-vertex graph.  gft_write_output_gz produces the same text,
// compressed: every block of kLines lines is formatted and deflated by its
// own thread into a complete gzip member, and the members are written in
// block order.  A gzip file may hold several members (RFC 1952 2.2), which
// every reader decompresses as one stream, so the result is the text file.
// The binary dump is the array itself behind a 24-byte header.
#include <errno.h>
#include <stdio.h>
#include <string.h>
#include <zlib.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "gft_internal.h"

namespace gft {
namespace {

constexpr uint32_t kLines = 1u << 20;  // lines per gzip member
const char kMagic[8] = {'G', 'F', 'T', 'N', 'O', 'D', 'E', '1'};

// Text of lines [lo, hi): "%d %d\n" or "%d INF\n" (apps/bfs/support.cu:39-45).
void format_lines(const int32_t *v, uint32_t lo, uint32_t hi, std::string &s)
{
    s.clear();
    s.reserve((size_t)(hi - lo) * 16);
    char line[48];
    for (uint32_t i = lo; i < hi; i++) {
        int n = v[i] == GFT_INF ? snprintf(line, sizeof line, "%d INF\n", (int)i)
                                : snprintf(line, sizeof line, "%d %d\n", (int)i, v[i]);
        s.append(line, n);
    }
}

// One complete gzip member holding `text`; false on a zlib failure.
bool gzip_member(const std::string &text, int level, std::string &out)
{
    z_stream z;
    memset(&z, 0, sizeof z);
    if (deflateInit2(&z, level, Z_DEFLATED, 15 + 16, 8, Z_DEFAULT_STRATEGY) != Z_OK) return false;
    out.resize(deflateBound(&z, text.size()) + 64);
    z.next_in = (Bytef *)text.data();
    z.avail_in = (uInt)text.size();
    z.next_out = (Bytef *)&out[0];
    z.avail_out = (uInt)out.size();
    const int r = deflate(&z, Z_FINISH);
    out.resize(z.total_out);
    deflateEnd(&z);
    return r == Z_STREAM_END;
}

bool write_bytes(FILE *f, const void *p, size_t n) { return fwrite(p, 1, n, f) == n; }

}  // namespace
}  // namespace gft

using namespace gft;

extern "C" {

gft_status gft_write_output_gz(const char *path, uint32_t nnodes, const int32_t *h_val, int level)
{
    if (!path || (nnodes && !h_val)) return fail(GFT_ERR_INVALID_ARG, "gft_write_output_gz: null argument");
    if (level < 0 || level > 9) return fail(GFT_ERR_INVALID_ARG, "gft_write_output_gz: level %d not in 0..9", level);
    if (level == 0) level = 1;
    FILE *f = fopen(path, "wb");
    if (!f) return fail(GFT_ERR_IO, "gft_write_output_gz: cannot open %s: %s", path, strerror(errno));
    const uint32_t nblocks = std::max<uint32_t>(1, (nnodes + kLines - 1) / kLines);
    const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    bool ok = true;
    for (uint32_t b0 = 0; b0 < nblocks && ok; b0 += nt) {
        const uint32_t nb = std::min<uint32_t>(nt, nblocks - b0);
        std::vector<std::string> gz(nb);
        std::vector<char> good(nb, 0);
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < nb; t++)
            th.emplace_back([&, t] {
                const uint32_t lo = (b0 + t) * kLines, hi = std::min<uint32_t>(nnodes, lo + kLines);
                std::string text;
                if (lo < hi) format_lines(h_val, lo, hi, text);
                good[t] = gzip_member(text, level, gz[t]);
            });
        for (auto &x : th) x.join();
        for (uint32_t t = 0; t < nb && ok; t++) ok = good[t] && write_bytes(f, gz[t].data(), gz[t].size());
    }
    if (fclose(f) != 0) ok = false;
    if (!ok) return fail(GFT_ERR_IO, "gft_write_output_gz: write to %s failed", path);
    return GFT_OK;
}

gft_status gft_write_node_data(const char *path, uint32_t nnodes, const void *h_val, uint32_t elem_type)
{
    if (!path || (nnodes && !h_val)) return fail(GFT_ERR_INVALID_ARG, "gft_write_node_data: null argument");
    if (elem_type != GFT_ELEM_I32 && elem_type != GFT_ELEM_F32)
        return fail(GFT_ERR_INVALID_ARG, "gft_write_node_data: unknown element type %u", elem_type);
    FILE *f = fopen(path, "wb");
    if (!f) return fail(GFT_ERR_IO, "gft_write_node_data: cannot open %s: %s", path, strerror(errno));
    const uint32_t meta[2] = {elem_type, 0};
    const uint64_t n = nnodes;
    bool ok = write_bytes(f, kMagic, 8) && write_bytes(f, meta, 8) && write_bytes(f, &n, 8) &&
              write_bytes(f, h_val, (size_t)nnodes * 4);
    if (fclose(f) != 0) ok = false;
    if (!ok) return fail(GFT_ERR_IO, "gft_write_node_data: write to %s failed", path);
    return GFT_OK;
}

gft_status gft_read_node_data(const char *path, uint32_t *nnodes, uint32_t *elem_type, void *h_val)
{
    if (!path || !nnodes) return fail(GFT_ERR_INVALID_ARG, "gft_read_node_data: null argument");
    FILE *f = fopen(path, "rb");
    if (!f) return fail(GFT_ERR_IO, "gft_read_node_data: cannot open %s: %s", path, strerror(errno));
    char magic[8];
    uint32_t meta[2];
    uint64_t n = 0;
    bool ok = fread(magic, 1, 8, f) == 8 && fread(meta, 1, 8, f) == 8 && fread(&n, 1, 8, f) == 8;
    if (!ok || memcmp(magic, kMagic, 8) != 0 || meta[0] > GFT_ELEM_F32 || n >= 0xFFFFFFFFull) {
        fclose(f);
        return fail(GFT_ERR_FORMAT, "gft_read_node_data: %s is not a node-data dump", path);
    }
    if (h_val) {
        if (*nnodes < n) {
            fclose(f);
            return fail(GFT_ERR_INVALID_ARG, "gft_read_node_data: buffer of %u values for %llu", *nnodes,
                        (unsigned long long)n);
        }
        ok = fread(h_val, 4, (size_t)n, f) == n;
    }
    fclose(f);
    if (!ok) return fail(GFT_ERR_FORMAT, "gft_read_node_data: %s: truncated", path);
    *nnodes = (uint32_t)n;
    if (elem_type) *elem_type = meta[0];
    return GFT_OK;
}

}  // extern "C"
