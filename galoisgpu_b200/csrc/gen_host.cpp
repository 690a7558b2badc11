// gen_host.cpp -- host builders of the seeded synthetic graphs (definitions
// in gen_common.h) and of query sources.  The device builders in
// gen_device.cu produce identical CSR arrays.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <thread>
#include <unordered_set>

#include "gen_common.h"
#include "gft_internal.h"

namespace gft {

template <typename F>
static void par_for(uint64_t n, F f)
{
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (n < (1u << 15) || nt == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    uint64_t chunk = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        uint64_t b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([=] { f(b, e); });
    }
    for (auto &x : th) x.join();
}

// Builds the symmetric CSR of the undirected pairs produced by
// get(i, &u, &v) for i in [0, npairs) (get returns false to skip a pair).
// Self loops and duplicates are dropped and every row is sorted; weights
// come from pair_weight when max_weight > 0.
template <typename Get>
static gft_status build_symmetric(uint32_t nnodes, uint64_t npairs, Get get, uint32_t max_weight, uint64_t wkey,
                                  gft_csr *out)
{
    memset(out, 0, sizeof *out);
    std::unique_ptr<std::atomic<uint32_t>[]> cnt(new (std::nothrow) std::atomic<uint32_t>[nnodes + 1]);
    if (!cnt) return fail(GFT_ERR_OOM, "generator: host allocation failed");
    par_for(nnodes + 1ull, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) cnt[i].store(0, std::memory_order_relaxed);
    });
    par_for(npairs, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            uint32_t u, v;
            if (!get(i, &u, &v) || u == v) continue;
            cnt[u].fetch_add(1, std::memory_order_relaxed);
            cnt[v].fetch_add(1, std::memory_order_relaxed);
        }
    });
    std::vector<uint64_t> off(nnodes + 1);
    uint64_t total = 0;
    for (uint32_t i = 0; i < nnodes; i++) {
        off[i] = total;
        total += cnt[i].load(std::memory_order_relaxed);
    }
    off[nnodes] = total;
    if (total >= 0xFFFFFFFFull) return fail(GFT_ERR_OVERFLOW, "generator: %llu directed edges exceed 32-bit ids",
                                            (unsigned long long)total);
    uint32_t *tmp = (uint32_t *)malloc(std::max<uint64_t>(total, 1) * 4);
    if (!tmp) return fail(GFT_ERR_OOM, "generator: host allocation failed");
    par_for(nnodes, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) cnt[i].store(0, std::memory_order_relaxed);
    });
    par_for(npairs, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            uint32_t u, v;
            if (!get(i, &u, &v) || u == v) continue;
            tmp[off[u] + cnt[u].fetch_add(1, std::memory_order_relaxed)] = v;
            tmp[off[v] + cnt[v].fetch_add(1, std::memory_order_relaxed)] = u;
        }
    });
    // Sort and deduplicate every row in place; cnt[] becomes the final degree.
    par_for(nnodes, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            uint32_t *r = tmp + off[i];
            uint64_t d = off[i + 1] - off[i];
            std::sort(r, r + d);
            uint64_t k = std::unique(r, r + d) - r;
            cnt[i].store((uint32_t)k, std::memory_order_relaxed);
        }
    });
    out->nnodes = nnodes;
    out->row_start = (uint32_t *)malloc((nnodes + 1ull) * 4);
    if (!out->row_start) {
        free(tmp);
        return fail(GFT_ERR_OOM, "generator: host allocation failed");
    }
    uint64_t ne = 0;
    for (uint32_t i = 0; i < nnodes; i++) {
        out->row_start[i] = (uint32_t)ne;
        ne += cnt[i].load(std::memory_order_relaxed);
    }
    out->row_start[nnodes] = (uint32_t)ne;
    out->nedges = (uint32_t)ne;
    out->edge_dst = (uint32_t *)malloc(std::max<uint64_t>(ne, 1) * 4);
    if (max_weight) out->edge_data = (int32_t *)malloc(std::max<uint64_t>(ne, 1) * 4);
    if (!out->edge_dst || (max_weight && !out->edge_data)) {
        free(tmp);
        gft_csr_free(out);
        return fail(GFT_ERR_OOM, "generator: host allocation failed");
    }
    par_for(nnodes, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            uint32_t d = out->row_start[i + 1] - out->row_start[i];
            memcpy(out->edge_dst + out->row_start[i], tmp + off[i], (size_t)d * 4);
            if (max_weight)
                for (uint32_t j = 0; j < d; j++)
                    out->edge_data[out->row_start[i] + j] =
                        (int32_t)pair_weight(wkey, (uint32_t)i, out->edge_dst[out->row_start[i] + j], max_weight);
        }
    });
    free(tmp);
    return GFT_OK;
}

// Draws k distinct vertices of out-degree > 0: draw i of the source stream,
// modulo nnodes, skipping repeats and isolated vertices.
gft_status pick_sources_rs(uint32_t nnodes, const uint32_t *row_start, uint64_t seed, uint32_t k, uint32_t *out)
{
    if (nnodes == 0 && k) return fail(GFT_ERR_INVALID_ARG, "pick_sources: empty graph");
    uint64_t key = stream_key(seed, kStreamSource);
    std::unordered_set<uint32_t> seen;
    uint32_t got = 0;
    uint64_t limit = 64ull * nnodes + (1u << 20);
    for (uint64_t i = 0; got < k && i < limit; i++) {
        uint32_t v = (uint32_t)(draw(key, i) % nnodes);
        if (row_start[v + 1] == row_start[v] || seen.count(v)) continue;
        seen.insert(v);
        out[got++] = v;
    }
    if (got < k) return fail(GFT_ERR_INVALID_ARG, "pick_sources: only %u of %u sources found", got, k);
    return GFT_OK;
}

}  // namespace gft

using namespace gft;

extern "C" {

gft_status gft_gen_grid(uint32_t rows, uint32_t cols, uint64_t seed, uint32_t max_weight, gft_csr *out)
{
    if (!out || rows == 0 || cols == 0 || (uint64_t)rows * cols >= 0xFFFFFFFFull)
        return fail(GFT_ERR_INVALID_ARG, "gft_gen_grid: bad size %u x %u", rows, cols);
    uint64_t wkey = stream_key(seed, kStreamWeight);
    uint64_t n_und = grid_undirected_edges(rows, cols);
    if (rows == 1 || cols == 1) n_und = (uint64_t)rows * cols - 1;  // a path
    auto get = [=](uint64_t i, uint32_t *u, uint32_t *v) {
        if (rows == 1 || cols == 1) {
            *u = (uint32_t)i;
            *v = (uint32_t)i + 1;
            return true;
        }
        grid_edge_endpoints(rows, cols, i, u, v);
        return true;
    };
    gft_status s = build_symmetric(rows * cols, n_und, get, max_weight, wkey, out);
    // max_weight == 1 means unit weights, which pair_weight yields as 1 + x % 1.
    return s;
}

gft_status gft_gen_road(uint32_t side, uint64_t seed, uint32_t delete_ppm, uint32_t shortcut_ppm,
                        uint32_t max_weight, gft_csr *out)
{
    if (!out || side < 2 || (uint64_t)side * side >= 0xFFFFFFFFull || delete_ppm > 1000000)
        return fail(GFT_ERR_INVALID_ARG, "gft_gen_road: bad arguments");
    uint32_t nn = side * side;
    uint64_t n_grid = grid_undirected_edges(side, side);
    uint64_t n_short = road_shortcuts(side, shortcut_ppm);
    uint64_t dkey = stream_key(seed, kStreamDelete), skey = stream_key(seed, kStreamShortcut),
             wkey = stream_key(seed, kStreamWeight);
    auto get = [=](uint64_t i, uint32_t *u, uint32_t *v) {
        if (i < n_grid) {
            if (!road_keep(dkey, i, delete_ppm)) return false;
            grid_edge_endpoints(side, side, i, u, v);
            return true;
        }
        road_shortcut(skey, i - n_grid, nn, u, v);
        return true;
    };
    return build_symmetric(nn, n_grid + n_short, get, max_weight, wkey, out);
}

gft_status gft_gen_rmat(uint32_t scale, uint32_t edge_factor, uint32_t a_q32, uint32_t b_q32, uint32_t c_q32,
                        uint64_t seed, uint32_t max_weight, gft_csr *out)
{
    if (!out || scale == 0 || scale > 31 || edge_factor == 0 || (uint64_t)a_q32 + b_q32 + c_q32 > 0xFFFFFFFFull)
        return fail(GFT_ERR_INVALID_ARG, "gft_gen_rmat: bad arguments");
    uint32_t nn = 1u << scale;
    uint64_t ns = (uint64_t)edge_factor << scale;
    uint64_t rkey = stream_key(seed, kStreamRmat), wkey = stream_key(seed, kStreamWeight);
    Perm perm = make_perm(seed, scale);
    RmatThresholds t = rmat_thresholds(a_q32, b_q32, c_q32);
    auto get = [=](uint64_t i, uint32_t *u, uint32_t *v) {
        uint32_t a, b;
        rmat_sample(rkey, i, scale, t.ta, t.tab, t.tabc, &a, &b);
        *u = perm_apply(perm, a);
        *v = perm_apply(perm, b);
        return true;
    };
    return build_symmetric(nn, ns, get, max_weight, wkey, out);
}

gft_status gft_pick_sources(const gft_csr *g, uint64_t seed, uint32_t k, uint32_t *out_sources)
{
    if (!g || !g->row_start || (k && !out_sources)) return fail(GFT_ERR_INVALID_ARG, "gft_pick_sources: null argument");
    return gft::pick_sources_rs(g->nnodes, g->row_start, seed, k, out_sources);
}

}  // extern "C"
