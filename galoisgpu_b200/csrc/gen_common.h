// gen_common.h -- seeded synthetic-graph definitions shared by the host
// generators (gen_host.cpp) and the device generators (gen_device.cu).
//
// Every random choice is a pure function of (seed, stream, index), drawn from
// the SplitMix64 sequence (Steele, Lea, Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014): output i of a generator with key k is
// mix64(k + (i + 1) * GAMMA).  Being counter based, a draw can be computed by
// any thread in any order, so the host and device produce the same graph bit
// for bit.
//
// The graphs stand in for the reference's downloaded inputs (road-NY/USA,
// rmat22, r4-2e23, named in apps/sssp/bmktest2.py:23), which are not
// available; they are built symmetric, without self loops or duplicate
// edges, with each row sorted by destination.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GFT_HD __host__ __device__ __forceinline__
#else
#define GFT_HD inline
#endif

namespace gft {

constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;

GFT_HD uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Key of an independent stream derived from a user seed.
GFT_HD uint64_t stream_key(uint64_t seed, uint64_t stream)
{
    return mix64(seed ^ mix64(stream * kGamma + kGamma));
}

// Output `i` of the SplitMix64 sequence with key `key`.
GFT_HD uint64_t draw(uint64_t key, uint64_t i) { return mix64(key + (i + 1) * kGamma); }

enum Stream : uint64_t {
    kStreamDelete = 1,    // road: per undirected grid edge, keep / delete
    kStreamWeight = 2,    // per undirected pair (min, max): weight
    kStreamShortcut = 3,  // road: shortcut endpoints
    kStreamRmat = 4,      // rmat: quadrant choices
    kStreamPermute = 5,   // rmat: vertex permutation constants
    kStreamSource = 6,    // query sources
};

// Weight of the undirected pair {u, v}: uniform in [1, max_weight].  Being a
// function of the pair alone, both directions and any duplicate carry the
// same weight.
GFT_HD uint32_t pair_weight(uint64_t wkey, uint32_t u, uint32_t v, uint32_t max_weight)
{
    uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
    uint64_t pair = ((uint64_t)lo << 32) | hi;
    return 1u + (uint32_t)(draw(wkey, pair) % max_weight);
}

// ---- grids -----------------------------------------------------------------
// rows x cols grid, vertex id r*cols + c.  Undirected edges are numbered:
// horizontal (r,c)-(r,c+1) -> r*(cols-1) + c, then vertical (r,c)-(r+1,c) ->
// rows*(cols-1) + r*cols + c.
GFT_HD uint64_t grid_undirected_edges(uint32_t rows, uint32_t cols)
{
    return (uint64_t)rows * (cols - 1) + (uint64_t)(rows - 1) * cols;
}

GFT_HD void grid_edge_endpoints(uint32_t rows, uint32_t cols, uint64_t id, uint32_t *u, uint32_t *v)
{
    uint64_t nh = (uint64_t)rows * (cols - 1);
    if (id < nh) {
        uint32_t r = (uint32_t)(id / (cols - 1)), c = (uint32_t)(id % (cols - 1));
        *u = r * cols + c;
        *v = *u + 1;
    } else {
        id -= nh;
        uint32_t r = (uint32_t)(id / cols), c = (uint32_t)(id % cols);
        *u = r * cols + c;
        *v = *u + cols;
    }
}

// Road: grid edge `id` survives unless its draw falls under delete_ppm per
// million.
GFT_HD bool road_keep(uint64_t dkey, uint64_t id, uint32_t delete_ppm)
{
    return (draw(dkey, id) % 1000000ull) >= delete_ppm;
}

GFT_HD uint64_t road_shortcuts(uint32_t side, uint32_t shortcut_ppm)
{
    return grid_undirected_edges(side, side) * shortcut_ppm / 1000000ull;
}

// Shortcut k joins two uniform vertices (a self loop is dropped later).
GFT_HD void road_shortcut(uint64_t skey, uint64_t k, uint32_t nnodes, uint32_t *u, uint32_t *v)
{
    *u = (uint32_t)(draw(skey, 2 * k) % nnodes);
    *v = (uint32_t)(draw(skey, 2 * k + 1) % nnodes);
}

// ---- R-MAT -----------------------------------------------------------------
// Chakrabarti, Zhan, Faloutsos, "R-MAT: A Recursive Model for Graph Mining",
// SDM 2004, with the Graph500 parameters a=.57 b=.19 c=.19 d=.05.  Sample k
// descends `scale` levels; level l uses 32 bits of draw(rkey, k*ceil(scale/2)
// + l/2) and picks quadrant a/b/c/d by comparing against the cumulative
// thresholds (parts per 2^32).
GFT_HD void rmat_sample(uint64_t rkey, uint64_t k, uint32_t scale, uint64_t ta, uint64_t tab, uint64_t tabc,
                        uint32_t *u, uint32_t *v)
{
    uint32_t su = 0, sv = 0;
    uint32_t per = (scale + 1) / 2;
    uint64_t r = 0;
    for (uint32_t l = 0; l < scale; l++) {
        if ((l & 1) == 0) r = draw(rkey, k * per + l / 2);
        uint64_t x = (l & 1) ? (r >> 32) : (r & 0xFFFFFFFFull);
        uint32_t bu, bv;
        if (x < ta) { bu = 0; bv = 0; }
        else if (x < tab) { bu = 0; bv = 1; }
        else if (x < tabc) { bu = 1; bv = 0; }
        else { bu = 1; bv = 1; }
        su = (su << 1) | bu;
        sv = (sv << 1) | bv;
    }
    *u = su;
    *v = sv;
}

// Seeded bijection of [0, 2^scale): three rounds of (odd multiply, xorshift,
// add), each invertible modulo 2^scale.  Scatters the R-MAT hubs over the id
// space as the Graph500 generator's vertex permutation does.
struct Perm {
    uint64_t mul[3], add[3];
    uint32_t scale;
};

inline Perm make_perm(uint64_t seed, uint32_t scale)
{
    Perm p;
    uint64_t key = stream_key(seed, kStreamPermute);
    for (int i = 0; i < 3; i++) {
        p.mul[i] = draw(key, 2 * i) | 1ull;
        p.add[i] = draw(key, 2 * i + 1);
    }
    p.scale = scale;
    return p;
}

GFT_HD uint32_t perm_apply(const Perm &p, uint32_t x0)
{
    uint64_t mask = (p.scale >= 64) ? ~0ull : ((1ull << p.scale) - 1);
    uint64_t x = x0;
    uint32_t sh = p.scale / 2 + 1;
    for (int i = 0; i < 3; i++) {
        x = (x * p.mul[i]) & mask;
        x ^= x >> sh;
        x = (x + p.add[i]) & mask;
    }
    return (uint32_t)x;
}

// Cumulative quadrant thresholds from per-2^32 probabilities.
struct RmatThresholds {
    uint64_t ta, tab, tabc;
};
GFT_HD RmatThresholds rmat_thresholds(uint32_t a, uint32_t b, uint32_t c)
{
    RmatThresholds t;
    t.ta = a;
    t.tab = (uint64_t)a + b;
    t.tabc = (uint64_t)a + b + c;
    return t;
}

}  // namespace gft
