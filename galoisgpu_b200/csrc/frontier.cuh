// frontier.cuh -- the traversal engine's device code, shared by the
// single-query kernels (traversal.cu) and the batched / served kernels
// (batch.cu): kernel parameters, the per-edge visitors (BFS visit, SSSP
// relaxation), the per-vertex expansion tiers and the BFS / SSSP bodies,
// written once against an execution mode (whole cooperative grid or one
// CTA).
#pragma once
#include <stdint.h>

#include "gft_internal.h"
#include "traverse.cuh"

namespace gft {
namespace dev {

constexpr uint32_t kHubChunk = 2048;  // edges of a hub handled per warp claim
constexpr unsigned kInf = 0x7FFFFFFFu;

__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p) { return __ldcs(p); }

// a[i & 1] without dynamic indexing (keeps a local parameter copy out of
// local memory).
__device__ __forceinline__ uint32_t *sel2(uint32_t *const (&a)[2], unsigned i) { return (i & 1) ? a[1] : a[0]; }
__device__ __forceinline__ uint4 ld_stream4(const uint32_t *p) { return __ldcs(reinterpret_cast<const uint4 *>(p)); }

// ---------------------------------------------------------------------------
// Parameters
// ---------------------------------------------------------------------------
// Frontier vertices of at least this many edges are expanded by a whole
// warp, smaller ones flattened across the warp (gft_tuning.warp_degree).
constexpr uint32_t kDefaultWarpDegree = 32;

struct TravParams {
    const uint32_t *__restrict__ row_start;
    const uint32_t *__restrict__ edge_dst;
    const int32_t *__restrict__ edge_data;  // SSSP; NULL = every weight 0
    const uint2 *__restrict__ edge_dw;      // SSSP: (edge_dst, edge_data) interleaved, or NULL
    const uint4 *__restrict__ bfs_slots;    // one-CTA thread-per-vertex BFS: 16-byte slot per vertex, or NULL
    uint32_t nnodes;
    uint32_t src;
    int32_t *out;       // level / dist
    uint32_t *parent;   // BFS parent or NULL
    uint32_t *visited;  // BFS bitmap
    uint32_t *q[2];     // frontier / near pile
    uint32_t *far[2];   // SSSP far pile
    uint32_t *qstamp;   // SSSP: the last pile stamp per vertex (see SsspVisitorT); distances live in `out`
    uint2 *hubs;
    uint32_t hub_cap;
    uint32_t hub_degree;
    uint32_t qcap;
    uint32_t delta;
    TraversalCtl *ctl;
    unsigned long long timeout_ns;
    int skip_block;
    int vec_ok;
    uint32_t nedges;
    int dir_opt;  // BFS: direction-optimising (graph marked symmetric)
    int uniform;  // every out-degree <= kUniformDegree: static chunks
    uint32_t cta_small;  // SSSP on the grid: iterations of at most this many vertices run on one CTA (0 = never)
    uint32_t fuse;       // SSSP: near vertices a warp may expand itself in the iteration that found them (0 = none)
    uint32_t warp_degree = kDefaultWarpDegree;  // a vertex of at least this many edges is expanded by a whole warp
};

// ---------------------------------------------------------------------------
// Visitors: what happens to one edge.
// ---------------------------------------------------------------------------
struct BfsOwn {
    uint32_t u;
};

#ifndef GFT_BFS_BATCH
#define GFT_BFS_BATCH 2
#endif
#ifndef GFT_SSSP_BATCH
#define GFT_SSSP_BATCH 2
#endif

#ifdef GFT_TRACE
// Diagnostic builds only: per-iteration (time, work) records of the last
// single-query traversal, read back by gft_debug_trace.
__device__ unsigned long long g_trace[2 * 8192];
__device__ __forceinline__ void trace_iter(unsigned i, unsigned long long info)
{
    if (i < 8192) {
        g_trace[2 * i] = globaltimer_ns();
        g_trace[2 * i + 1] = info;
    }
}
#else
__device__ __forceinline__ void trace_iter(unsigned, unsigned long long) {}
#endif

// A probe of the BFS visited bitmap.  The grid's bitmap is in global memory
// and read around L1 (other SMs set its bits); a single-CTA traversal of a
// small graph keeps it in shared memory, where a probe and a claim cost tens
// of cycles instead of an L2 round trip each.
template <bool kLocalBits>
__device__ __forceinline__ uint32_t ld_bits(const uint32_t *p)
{
    if constexpr (kLocalBits)
        return *(const volatile uint32_t *)p;
    else
        return __ldcg(p);
}

template <bool kLocalBits = false, unsigned kQB = kQueueBuf>
struct BfsVisitorT {
    static constexpr int kBatch = GFT_BFS_BATCH;  // edges per lane in one flattened step
    static constexpr bool kEarlyRow = false;      // owner() loads nothing
    const uint32_t *__restrict__ edge_dst;
    const uint32_t *__restrict__ row_start;  // non-NULL: sum the out-degrees of claimed vertices
    unsigned long long mf;                    // that sum, per lane
    uint32_t *visited;
    int32_t *level;
    uint32_t *parent;
    int newlevel;
    WarpQueueT<kQB> q;  // pushes of the next frontier, a kQB-entry buffer per warp
    unsigned long long edges;  // per lane
    unsigned long long claimed;
    bool vec;

    __device__ __forceinline__ BfsOwn owner(bool has, uint32_t u) const { return BfsOwn{u}; }
    __device__ __forceinline__ bool active(const BfsOwn &) const { return true; }
    __device__ __forceinline__ BfsOwn shfl(const BfsOwn &o, int lane) const
    {
        return BfsOwn{__shfl_sync(kFull, o.u, lane)};
    }

    // K visits per lane, staged so that the lane's K bitmap probes, then its
    // K claims, are each in flight together: one memory latency per stage
    // instead of one per edge.  Two of a lane's K edges may name the same
    // vertex; the second claim then sees the first one's bit.
    template <int K>
    __device__ __forceinline__ void visitK(const bool (&valid)[K], const uint32_t (&dst)[K], const BfsOwn (&o)[K],
                                           unsigned lane)
    {
        uint32_t word[K];
#pragma unroll
        for (int k = 0; k < K; k++) word[k] = valid[k] ? ld_bits<kLocalBits>(visited + (dst[k] >> 5)) : 0xFFFFFFFFu;
        bool mine[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const uint32_t b = 1u << (dst[k] & 31);
            mine[k] = false;
            if (valid[k]) edges++;
            if (!(word[k] & b)) word[k] = atomicOr(visited + (dst[k] >> 5), b), mine[k] = !(word[k] & b);
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (mine[k]) {
                level[dst[k]] = newlevel;
                if (parent) parent[dst[k]] = o[k].u;
                claimed++;
                if (row_start) mf += __ldg(row_start + dst[k] + 1) - __ldg(row_start + dst[k]);
            }
            q.push(mine[k], dst[k], lane);
        }
    }
    template <int K>
    __device__ __forceinline__ void edgeK(const bool (&valid)[K], const uint32_t (&e)[K], const BfsOwn (&o)[K],
                                          unsigned lane)
    {
        uint32_t d[K];
#pragma unroll
        for (int k = 0; k < K; k++) d[k] = valid[k] ? ld_stream(edge_dst + e[k]) : 0u;
        visitK<K>(valid, d, o, lane);
    }
    __device__ __forceinline__ void edge1(bool valid, uint32_t e, const BfsOwn &o, unsigned lane)
    {
        const bool v[1] = {valid};
        const uint32_t ee[1] = {e};
        const BfsOwn oo[1] = {o};
        edgeK<1>(v, ee, oo, lane);
    }
    __device__ __forceinline__ void edge4(bool valid, uint32_t e, const BfsOwn &o, unsigned lane)
    {
        const uint4 d = valid ? ld_stream4(edge_dst + e) : make_uint4(0, 0, 0, 0);
        const bool v[4] = {valid, valid, valid, valid};
        const uint32_t dd[4] = {d.x, d.y, d.z, d.w};
        const BfsOwn oo[4] = {o, o, o, o};
        visitK<4>(v, dd, oo, lane);
    }
};
using BfsVisitor = BfsVisitorT<false>;

struct SsspOwn {
    uint32_t u;
    uint32_t du;
};

// SSSP relaxation (apps/sssp/kernel.cu:244-259): nd = dist[u] + w; if nd
// beats dist[v], atomicMin.  Distances are the 4-byte int32 output array
// itself (a probe fetches a sector of eight of them, and the whole array
// stays L2-resident on graphs of up to ~2^24 vertices).  An improvement then
// raises v's stamp in one 4-byte array with atomicMax.  Stamps increase with
// the iteration I: far 4(I+1), fused 4(I+1)+1, near (bucket threshold met)
// 4(I+1)+2.
//   - near: v joins the near pile unless the stamp it replaced is this
//     iteration's near stamp (so the pile holds v at most once per
//     iteration);
//   - far: v joins the far pile unless the stamp it replaced is from the
//     current phase (at least phase_stamp, the far stamp of the iteration
//     that started it, which the far split writes for the vertices it
//     carries over).
// With atomicMax a far stamp never replaces a near (or fused) stamp of the
// same iteration: a far improvement that loses the race to a near one is
// dropped, rightly (v's distance is already below the threshold).  Once v is
// near in a phase it cannot go far again in that phase (distances only
// fall), so a near stamp hides no far-pile entry.
//
// kSolo: the single-query kernel's visitor, which also reads interleaved
// (dst, weight) pairs when the graph has them, loads a vertex's row
// alongside its distance, and runs bucket fusion; the batched kernel's jobs
// use the leaner visitor, which keeps that kernel's register budget.
template <bool kSolo, unsigned kQB = kQueueBuf>
struct SsspVisitorT {
    static constexpr int kBatch = GFT_SSSP_BATCH;  // edges per lane in one flattened step
    static constexpr bool kEarlyRow = kSolo;       // owner() loads the distance
    static constexpr bool kFuse = kSolo;           // warps may expand the near vertices they found
    const uint32_t *__restrict__ edge_dst;
    const int32_t *__restrict__ edge_data;
    const uint2 *__restrict__ edge_dw;  // interleaved (dst, weight), or NULL
    uint32_t *dist;
    uint32_t *qstamp;
    uint32_t near_stamp, phase_stamp;  // this iteration's far stamp is near_stamp - 2
    uint32_t threshold;  // inclusive; a bucket bound above 2^32 - 1 is clamped (every distance is below it)
    WarpQueueT<kQB> nq, fq;  // near and far pushes, kQB-entry buffers per warp
    unsigned far_min;
    unsigned long long edges;
    unsigned *err, *err_where;
    bool vec;

    __device__ __forceinline__ SsspOwn owner(bool has, uint32_t u) const
    {
        return SsspOwn{u, has ? __ldcg(dist + u) : kInf};
    }
    __device__ __forceinline__ bool active(const SsspOwn &o) const { return o.du != kInf; }
    __device__ __forceinline__ SsspOwn shfl(const SsspOwn &o, int lane) const
    {
        return SsspOwn{__shfl_sync(kFull, o.u, lane), __shfl_sync(kFull, o.du, lane)};
    }

    // K relaxations per lane, staged so that the lane's K distance probes,
    // then its K atomicMins, then its K stamps, are each in flight together:
    // one memory latency per stage instead of one per edge.  Two of a lane's
    // K edges may name the same vertex; its atomics then apply in program
    // order, so the second sees the first and the vertex is queued once, as
    // with one edge at a time.
    template <int K>
    __device__ __forceinline__ void relaxK(const bool (&valid)[K], const uint32_t (&v)[K], const uint32_t (&w)[K],
                                           const SsspOwn (&o)[K], unsigned lane)
    {
        uint32_t cur[K];
#pragma unroll
        for (int k = 0; k < K; k++) cur[k] = valid[k] ? __ldcg(dist + v[k]) : 0u;
        uint32_t nd[K];
        bool imp[K], near[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            imp[k] = near[k] = false;
            nd[k] = o[k].du + w[k];  // du < 2^31 and w < 2^32: a wrap is caught below
            if (!valid[k]) continue;
            edges++;
            if (nd[k] >= kInf || nd[k] < o[k].du) {
                raise_error(err, err_where, GFT_ERR_OVERFLOW, o[k].u);
            } else if (nd[k] < cur[k]) {
                imp[k] = nd[k] < atomicMin(dist + v[k], nd[k]);
                near[k] = nd[k] <= threshold;
            }
        }
        uint32_t old[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            old[k] = 0;
            if (imp[k]) {
                if (!near[k]) far_min = min(far_min, nd[k]);
                old[k] = atomicMax(qstamp + v[k], near[k] ? near_stamp : near_stamp - 2u);
            }
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            nq.push(imp[k] && near[k] && old[k] != near_stamp, v[k], lane);
            fq.push(imp[k] && !near[k] && old[k] < phase_stamp, v[k], lane);
        }
    }
    template <int K>
    __device__ __forceinline__ void edgeK(const bool (&valid)[K], const uint32_t (&e)[K], const SsspOwn (&o)[K],
                                          unsigned lane)
    {
        uint32_t d[K], w[K];
        if (kSolo && edge_dw) {  // one 8-byte load per edge
#pragma unroll
            for (int k = 0; k < K; k++) {
                const uint2 x = valid[k] ? __ldcs(edge_dw + e[k]) : make_uint2(0, 0);
                d[k] = x.x;
                w[k] = x.y;
            }
        } else {
#pragma unroll
            for (int k = 0; k < K; k++) {
                d[k] = valid[k] ? ld_stream(edge_dst + e[k]) : 0u;
                w[k] = (valid[k] && edge_data) ? (uint32_t)__ldcs(edge_data + e[k]) : 0u;
            }
        }
        relaxK<K>(valid, d, w, o, lane);
    }
    __device__ __forceinline__ void edge1(bool valid, uint32_t e, const SsspOwn &o, unsigned lane)
    {
        const bool vv[1] = {valid};
        const uint32_t ee[1] = {e};
        const SsspOwn oo[1] = {o};
        edgeK<1>(vv, ee, oo, lane);
    }
    __device__ __forceinline__ void edge4(bool valid, uint32_t e, const SsspOwn &o, unsigned lane)
    {
        uint4 d = make_uint4(0, 0, 0, 0), w = make_uint4(0, 0, 0, 0);
        if (valid) {
            if (kSolo && edge_dw) {  // e % 4 == 0: two 16-byte loads of 32-byte-aligned pairs
                const uint4 a = __ldcs(reinterpret_cast<const uint4 *>(edge_dw + e));
                const uint4 b = __ldcs(reinterpret_cast<const uint4 *>(edge_dw + e + 2));
                d = make_uint4(a.x, a.z, b.x, b.z);
                w = make_uint4(a.y, a.w, b.y, b.w);
            } else {
                d = ld_stream4(edge_dst + e);
                if (edge_data) w = __ldcs(reinterpret_cast<const uint4 *>(edge_data + e));
            }
        }
        const bool vv[4] = {valid, valid, valid, valid};
        const uint32_t dd[4] = {d.x, d.y, d.z, d.w}, ww[4] = {w.x, w.y, w.z, w.w};
        const SsspOwn oo[4] = {o, o, o, o};
        relaxK<4>(vv, dd, ww, oo, lane);
    }
};

// ---------------------------------------------------------------------------
// Expansion tiers
// ---------------------------------------------------------------------------

// The whole warp streams the edge range [start, start+len) of one vertex;
// 16-byte loads for the aligned body, scalar head and tail.
template <class Vis, class Own>
__device__ __forceinline__ void warp_range(Vis &vis, uint32_t start, uint32_t len, const Own &o, unsigned lane)
{
    const uint32_t end = start + len;
    if (vis.vec) {
        uint32_t a = min(end, (start + 3u) & ~3u);
        if (a > start) vis.edge1(start + lane < a, start + lane, o, lane);
        uint32_t bend = a + ((end - a) & ~3u);
        for (uint32_t base = a; base < bend; base += 128) {
            uint32_t e = base + lane * 4;
            vis.edge4(e < bend, e, o, lane);
        }
        if (end > bend) vis.edge1(bend + lane < end, bend + lane, o, lane);
    } else {
        for (uint32_t base = start; base < end; base += 32) vis.edge1(base + lane < end, base + lane, o, lane);
    }
}

// Chunk schedule shared by every grid-wide loop: chunk c covers items
// [c * grain, (c + 1) * grain).  Warp w first takes chunk w with no atomic;
// only when there are more chunks than warps do warps claim further chunks
// from the iteration's cursor (one atomic per chunk).  A small frontier
// therefore costs no atomics at all.
struct ChunkSched {
    unsigned nchunks, nwarps, gwarp, lane;
    unsigned *cursor;
    __device__ __forceinline__ unsigned first() const { return gwarp; }
    __device__ __forceinline__ unsigned next() const
    {
        if (nchunks <= nwarps) return nchunks;
        unsigned c = 0;
        if (lane == 0) c = nwarps + atomicAdd(cursor, 1u);
        return __shfl_sync(kFull, c, 0);
    }
};

// Flattened expansion of the edge ranges [start, start+deg) held one per
// lane (thread granularity): the warp takes the ranges' edges 32 * K at a
// time, K per lane, finds each edge's owner lane with a shuffle binary
// search over the exclusive prefix of the degrees, and hands the lane's K
// edges to the visitor together, so their memory operations overlap.
template <int K, class Vis, class Own>
__device__ __forceinline__ void flatten_edges(Vis &vis, uint32_t start, uint32_t deg, const Own &o, unsigned lane)
{
    const uint32_t incl = warp_incl_sum(deg, lane);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t excl = incl - deg;
    for (uint32_t base = 0; base < total; base += 32u * K) {
        bool valid[K];
        uint32_t e[K];
        Own ow[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const uint32_t g = base + 32u * k + lane;
            int j = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1)
                if (__shfl_sync(kFull, excl, j + step) <= g) j += step;
            const uint32_t ostart = __shfl_sync(kFull, start, j), oexcl = __shfl_sync(kFull, excl, j);
            valid[k] = g < total;
            e[k] = ostart + (g - oexcl);
            ow[k] = vis.shfl(o, j);
        }
        vis.template edgeK<K>(valid, e, ow, lane);
    }
}

// Expands one vertex per lane (`has` false on idle lanes): degree >=
// p.warp_degree by the whole warp, smaller lists flattened across it;
// vertices of degree >= hub_degree go to the hub list for the grid-wide hub
// phase.
template <class Vis, class Own>
__device__ __forceinline__ void expand_lanes(Vis &vis, const TravParams &p, bool has, uint32_t u,
                                             unsigned long long *hub_ctr, unsigned lane)
{
    // A visitor whose owner() loads per-vertex state (the SSSP distance, the
    // PageRank residual) has the row loaded alongside it, not after it: both
    // depend only on u, so the loads share one memory round trip.
    const uint32_t v = u;
    uint32_t start = 0, deg = 0;
    if (Vis::kEarlyRow && has) {
        start = __ldg(p.row_start + v);
        deg = __ldg(p.row_start + v + 1) - start;
    }
    Own o = vis.owner(has, u);
    if (!Vis::kEarlyRow && has && vis.active(o)) {
        start = __ldg(p.row_start + v);
        deg = __ldg(p.row_start + v + 1) - start;
    }
    if (!(has && vis.active(o))) deg = 0;
    if (deg >= p.hub_degree) {
        unsigned nch = (deg + kHubChunk - 1) / kHubChunk;
        unsigned long long old = atomicAdd(hub_ctr, (1ull << 32) | nch);
        unsigned h = (unsigned)(old >> 32);
        if (h < p.hub_cap) p.hubs[h] = make_uint2(v, (unsigned)old);
        else raise_error(&p.ctl->error, &p.ctl->error_where, GFT_ERR_OVERFLOW, h);
        deg = 0;
    }
    unsigned m = __ballot_sync(kFull, deg >= p.warp_degree);
    while (m) {
        const int l = __ffs(m) - 1;
        m &= m - 1;
        const uint32_t s = __shfl_sync(kFull, start, l), d = __shfl_sync(kFull, deg, l);
        warp_range(vis, s, d, vis.shfl(o, l), lane);
    }
    if (deg >= p.warp_degree) deg = 0;
    flatten_edges<Vis::kBatch>(vis, start, deg, o, lane);
}

// Expands the frontier `in[0, n)` in chunks of `grain` vertices.
template <class Vis, class Own>
__device__ __forceinline__ void expand_frontier(Vis &vis, const TravParams &p, const uint32_t *in, uint32_t n,
                                                unsigned *claim, unsigned long long *hub_ctr, unsigned grain,
                                                unsigned gwarp, unsigned nwarps, unsigned lane)
{
    const ChunkSched cs{(n + grain - 1) / grain, nwarps, gwarp, lane, claim};
    for (unsigned c = cs.first(); c < cs.nchunks; c = cs.next()) {
        const unsigned base = c * grain;
        const unsigned end = min(n, base + grain);
        for (unsigned i0 = base; i0 < end; i0 += 32) {
            const unsigned idx = i0 + lane;
            const bool has = idx < end;
            const uint32_t u = has ? __ldcg(in + idx) : 0u;
            expand_lanes<Vis, Own>(vis, p, has, u, hub_ctr, lane);
        }
    }
}

// Grid-wide processing of the hub list of one iteration: warps claim
// kHubChunk-edge chunks; hub h owns chunks [hubs[h].y, hubs[h+1].y).
template <class Vis, class Own>
__device__ __forceinline__ void expand_hubs(Vis &vis, const TravParams &p, unsigned nh, unsigned nc,
                                            unsigned *hub_claim, unsigned gwarp, unsigned nwarps, unsigned lane)
{
    const ChunkSched cs{nc, nwarps, gwarp, lane, hub_claim};
    for (unsigned c = cs.first(); c < nc; c = cs.next()) {
        unsigned lo = 0, hi = nh;
        while (hi - lo > 1) {
            unsigned mid = (lo + hi) >> 1;
            if (__ldcg(&p.hubs[mid].y) <= c) lo = mid;
            else hi = mid;
        }
        const uint2 hb = __ldcg(p.hubs + lo);
        const uint32_t u = hb.x;
        Own o = vis.owner(true, u);
        if (!vis.active(o)) continue;  // warp uniform: every lane read the same hub
        const uint32_t start = __ldg(p.row_start + u);
        const uint32_t deg = __ldg(p.row_start + u + 1) - start;
        const uint32_t off = (c - hb.y) * kHubChunk;
        const uint32_t len = min(kHubChunk, deg - off);
        warp_range(vis, start + off, len, o, lane);
    }
}

// Chunk size (vertices) for a frontier of n vertices over nwarps warps.  A
// frontier smaller than one 32-vertex chunk per warp is spread over all
// warps.  On a graph of uniform degree (road networks, grids) a larger
// frontier is cut into one chunk per warp, so no warp claims work through
// the shared cursor, whose atomics serialise in one L2 slice; on skewed
// graphs (R-MAT) about four chunks per warp are claimed dynamically, which
// keeps the warps balanced.
__device__ __forceinline__ unsigned pick_grain(unsigned n, unsigned nwarps, bool uniform)
{
    if (n < nwarps * 32u) return max(1u, (n + nwarps - 1) / nwarps);
    if (uniform) return 32u * ((n + nwarps * 32u - 1) / (nwarps * 32u));
    unsigned per = n / (nwarps * 32u * 4u);
    return 32u * max(1u, min(8u, per));
}

// One bottom-up BFS level (Beamer, Asanovic, Patterson, "Direction-Optimizing
// Breadth-First Search", SC 2012): every unvisited vertex scans its own
// edges, four at a time, for a neighbour in the current frontier (level ==
// L) and stops at the first it finds.  On a symmetric graph a vertex's
// out-edges are its in-edges, so this claims exactly the vertices a
// top-down level would, with the same level.  Warps take 32-vertex words of
// the visited bitmap and own them for the level, so each sets its word's
// new bits with one plain store; claimed vertices are also queued, so a
// top-down level can follow.
template <bool kLocalBits, unsigned kQB>
__device__ __forceinline__ void bottom_up_level(BfsVisitorT<kLocalBits, kQB> &vis, const TravParams &p, unsigned L,
                                                unsigned gwarp, unsigned nwarps, unsigned lane)
{
    const uint32_t n = p.nnodes, nwords = (n + 31) >> 5;
    const int32_t cur = (int32_t)L;
    for (uint32_t w = gwarp; w < nwords; w += nwarps) {
        const uint32_t word = ld_bits<kLocalBits>(p.visited + w);
        if (word == 0xFFFFFFFFu) continue;  // warp uniform
        const uint32_t v = (w << 5) + lane;
        bool found = false;
        uint32_t par = 0, deg = 0;
        if (v < n && !((word >> lane) & 1u)) {
            const uint32_t s = __ldg(p.row_start + v), e = __ldg(p.row_start + v + 1);
            deg = e - s;
            for (uint32_t i = s; i < e && !found; i += 4) {
                uint32_t u[4];
                int32_t lv[4];
#pragma unroll
                for (int k = 0; k < 4; k++) u[k] = i + k < e ? ld_stream(p.edge_dst + i + k) : 0u;
#pragma unroll
                for (int k = 0; k < 4; k++) lv[k] = i + k < e ? __ldcg(p.out + u[k]) : -1;
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (!found && lv[k] == cur) {
                        found = true;
                        par = u[k];
                        vis.edges += k + 1;
                    }
                if (!found) vis.edges += min(4u, e - i);
            }
        }
        const uint32_t got = __ballot_sync(kFull, found);
        if (found) {
            p.out[v] = cur + 1;
            if (p.parent) p.parent[v] = par;
            vis.claimed++;
            vis.mf += deg;
        }
        if (lane == 0 && got) p.visited[w] = word | got;
        vis.q.push(found, v, lane);
    }
}

// ---------------------------------------------------------------------------
// Execution modes.  One traversal runs on a group of threads: the whole
// cooperative grid (GridMode, single queries) or one CTA (CtaMode, batched
// and served queries, whose control block lives in shared memory and whose
// barrier is __syncthreads).  The traversal bodies below are written once
// against this interface.
// ---------------------------------------------------------------------------
struct GridMode {
    static constexpr bool kGrid = true;
    GridSync gs;
    TraversalCtl *ctl;
    unsigned tid, nthreads, gwarp, nwarps;
    __device__ __forceinline__ bool sync() { return gs.sync(); }
    __device__ __forceinline__ unsigned ld(unsigned *p) const { return ld_relaxed_u32(p); }
    __device__ __forceinline__ unsigned long long ld64(unsigned long long *p) const { return ld_relaxed_u64(p); }
    __device__ __forceinline__ unsigned epoch() const { return gs.epoch; }
};

struct CtaMode {
    static constexpr bool kGrid = false;
    TraversalCtl *ctl;  // in shared memory, or the grid's control block while one CTA runs alone
    unsigned tid, nthreads, gwarp, nwarps, ep;
    // Every thread contributes its own view of the error word, so all threads
    // take the same decision even if an error is raised as the barrier opens.
    __device__ __forceinline__ bool sync()
    {
        ep++;
        return !__syncthreads_or(*(volatile unsigned *)&ctl->error != 0);
    }
    __device__ __forceinline__ unsigned ld(unsigned *p) const { return *(volatile unsigned *)p; }
    __device__ __forceinline__ unsigned long long ld64(unsigned long long *p) const
    {
        return *(volatile unsigned long long *)p;
    }
    __device__ __forceinline__ unsigned epoch() const { return ep; }
};

// ---------------------------------------------------------------------------
// BFS body
// ---------------------------------------------------------------------------
// Direction switch (Beamer et al.): go bottom-up once the frontier's edges
// exceed 1/kAlpha of the edges still unexplored, and back top-down once the
// frontier holds fewer than 1/kBeta of the vertices.
constexpr unsigned kAlpha = 14, kBeta = 24, kScan = 32;

// kLocalBits: p.visited points to shared memory (one CTA runs the traversal).
// warp_buf: this warp's kQB-entry push buffer.
template <class Mode, bool kLocalBits = false, unsigned kQB = kQueueBuf>
__device__ __forceinline__ void bfs_body(const TravParams &p, Mode &m, uint32_t *warp_buf)
{
    using Vis = BfsVisitorT<kLocalBits, kQB>;
    TraversalCtl *ctl = m.ctl;
    const unsigned lane = threadIdx.x & 31;
    const unsigned tid = m.tid, nthreads = m.nthreads, nwarps = m.nwarps, gwarp = m.gwarp;

    // Initialise (apps/bfs/kernel.cu:20-32): level 0 at src, INF elsewhere.
    const uint32_t n = p.nnodes, nwords = (n + 31) >> 5;
    for (uint32_t v = tid; v < n; v += nthreads) {
        p.out[v] = v == p.src ? 0 : (int32_t)kInf;
        if (p.parent) p.parent[v] = v == p.src ? p.src : GFT_NO_PARENT;
    }
    for (uint32_t w = tid; w < nwords; w += nthreads)
        p.visited[w] = (w == (p.src >> 5)) ? (1u << (p.src & 31)) : 0u;
    if (tid == 0) {
        p.q[0][0] = p.src;
        *u32_of(ctl->qlen[0]) = 1;
        // far_len[] carries, per level slot, the out-degree sum of the
        // frontier (BFS has no far pile).
        *u32_of(ctl->far_len[0]) = p.row_start[p.src + 1] - p.row_start[p.src];
    }
    if (!m.sync()) return;

    Vis vis;
    vis.edge_dst = p.edge_dst;
    // Skewed graphs sum the claimed vertices' out-degrees for the direction
    // switch; on uniform-degree graphs the frontier's size times the mean
    // degree is as good and costs no loads.
    vis.row_start = (p.dir_opt && !p.uniform) ? p.row_start : nullptr;
    vis.mf = 0;
    vis.visited = p.visited;
    vis.level = p.out;
    vis.parent = p.parent;
    vis.edges = 0;
    vis.claimed = 0;
    vis.vec = p.vec_ok;
    vis.q.buf = warp_buf;
    vis.q.count = 0;
    vis.q.cap = p.qcap;
    vis.q.err = &ctl->error;
    vis.q.err_where = &ctl->error_where;

    unsigned L = 0;
    bool bottom_up = false;
    unsigned long long m_seen = 0;  // out-degree sum of the frontiers reached so far
    unsigned long long n_seen = 0;  // vertices reached so far (uniform-degree estimate)
    unsigned n_prev = 0;            // previous frontier size
    const float n_f = (float)n, E_f = (float)p.nedges, mean_deg = E_f / fmaxf(1.f, n_f);
    // One CTA (bitmap in shared memory) on a uniform-degree graph: a warp
    // takes at least as many frontier vertices as one flattened step holds
    // at the mean degree (32 * kBatch edges).  A small frontier then keeps a
    // few warps busy with one step each, instead of every warp paying a
    // step's fixed cost for a handful of vertices; the level's critical path
    // is the same single step.  (256^2 grid, frontiers of at most 256
    // vertices: 16 per warp.)
    const unsigned min_grain =
        (kLocalBits && p.uniform)
            ? max(1u, min(32u, 32u * Vis::kBatch / max(1u, (unsigned)ceilf(mean_deg))))
            : 1u;
    // The frontier's out-degree sum is only gathered on skewed graphs.
    const bool sum_degrees = p.dir_opt && !p.uniform;
    for (;;) {
        const unsigned slot = L % 3, nslot = (L + 1) % 3, rslot = (L + 2) % 3;
        const unsigned n_in = m.ld(u32_of(ctl->qlen[slot]));
        if (n_in == 0) {
            if (tid == 0) trace_iter(L, 0);
            break;
        }
        if (p.dir_opt) {  // every thread reads the same counters: a uniform decision
            // Single-precision arithmetic: the switch is a heuristic, and
            // 64-bit divisions by n would cost about a microsecond per level.
            float mf, m_u;
            if (p.uniform) {
                n_seen += n_in;
                mf = (float)n_in * mean_deg;
                m_u = fmaxf(0.f, E_f - (float)n_seen * mean_deg);
            } else {
                const unsigned mfi = m.ld(u32_of(ctl->far_len[slot]));
                m_seen += mfi;
                mf = (float)mfi;
                m_u = fmaxf(0.f, E_f - (float)m_seen);
            }
            // A bottom-up level also pays a pass over the visited bitmap (one
            // word per 32 vertices), so the switch charges n / kScan edge
            // equivalents for it; and it needs a growing frontier.  On a
            // high-diameter graph the frontier stops growing long before the
            // unexplored edges run low, and most unvisited vertices are far
            // from it and would scan all their edges in vain.  A uniform-degree
            // graph also needs a frontier of n / kBeta vertices: its frontier
            // edges are an estimate, and a road network's frontier can wobble
            // upward past its peak.
            const bool big = (float)n_in * kBeta >= n_f;
            bottom_up = bottom_up ? big
                                  : n_in > n_prev && (big || !p.uniform) && mf > m_u / kAlpha + n_f / kScan;
        }
        n_prev = n_in;
        if (tid == 0) {
            trace_iter(L, n_in | ((unsigned long long)bottom_up << 32));
            *u32_of(ctl->qlen[rslot]) = 0;
            *u32_of(ctl->claim[rslot]) = 0;
            ctl->hub[rslot].v = 0;
            *u32_of(ctl->hub_claim[rslot]) = 0;
            *u32_of(ctl->far_len[rslot]) = 0;
        }
        vis.newlevel = (int)L + 1;
        vis.q.queue = sel2(p.q, (L + 1));
        vis.q.len = u32_of(ctl->qlen[nslot]);
        unsigned *mf_next = u32_of(ctl->far_len[nslot]);
        if (bottom_up) {
            bottom_up_level(vis, p, L, gwarp, nwarps, lane);
        } else {
            const unsigned grain = max(min_grain, pick_grain(n_in, nwarps, p.uniform));
            expand_frontier<Vis, BfsOwn>(vis, p, sel2(p.q, L), n_in, u32_of(ctl->claim[slot]), &ctl->hub[slot].v,
                                         grain, gwarp, nwarps, lane);
        }
        vis.q.flush(lane);
        if (sum_degrees) {
            warp_add_u32(mf_next, (unsigned)vis.mf, lane);
            vis.mf = 0;
        }
        if (!m.sync()) return;
        const unsigned long long hv = bottom_up ? 0ull : m.ld64(&ctl->hub[slot].v);
        if (hv) {
            expand_hubs<Vis, BfsOwn>(vis, p, (unsigned)(hv >> 32), (unsigned)hv, u32_of(ctl->hub_claim[slot]),
                                     gwarp, nwarps, lane);
            vis.q.flush(lane);
            if (sum_degrees) {
                warp_add_u32(mf_next, (unsigned)vis.mf, lane);
                vis.mf = 0;
            }
            if (!m.sync()) return;
        }
        L++;
    }
    warp_add_u64(&ctl->edges, vis.edges, lane);
    warp_add_u64(&ctl->reached, vis.claimed, lane);
    if (tid == 0) {
        ctl->levels = L;
        ctl->iterations = m.epoch();
    }
}

// ---------------------------------------------------------------------------
// SSSP body (near-far)
// ---------------------------------------------------------------------------
// Bucket fusion (as in GraphIt's delta-stepping, Zhang et al., CGO 2020): a
// warp that pushed v to the near pile in this iteration may expand v itself
// before the barrier, taking v back out of its push buffer.  It first
// claims v by lowering v's stamp from this iteration's near stamp to the
// fused stamp (a compare-and-swap with acquire semantics), then reads v's
// distance as the expansion's owner.  A later improvement of v raises the
// stamp back to near and, having found the fused stamp, queues v again; an
// improvement whose stamp went in before the claim is visible to the read
// after it (the improving thread's atomicMin had completed before it issued
// its stamp, and the claim is an acquire), so no improvement is lost.
// Piles larger than this are not fused: every warp is busy with them
// already, and chasing only lengthens the wait at the barrier (road
// 4096^2 with 128-entry push buffers: 3.88 ms fusing every pile, 3.66 ms
// up to 262144, 3.74 ms up to 65536, 3.92 ms up to 16384; with 256-entry
// buffers: 3.53 ms up to 524288, 3.57 ms up to 262144, 3.56 ms up to
// 131072 or 1048576).
constexpr unsigned kFuseMaxPile = 524288;

// Near-far loop state: bucket threshold (inclusive), iteration, phase, and
// the iteration that started the phase.
struct SsspState {
    unsigned long long T;
    unsigned I, P, Ps;
};

// Pile stamps (see SsspVisitorT): increasing with the iteration, never 0.
__device__ __forceinline__ uint32_t far_stamp_of(unsigned I) { return (I + 1u) << 2; }
__device__ __forceinline__ uint32_t fused_stamp_of(unsigned I) { return ((I + 1u) << 2) | 1u; }
__device__ __forceinline__ uint32_t near_stamp_of(unsigned I) { return ((I + 1u) << 2) | 2u; }

__device__ __forceinline__ uint32_t cas_acquire_u32(uint32_t *p, uint32_t cmp, uint32_t val)
{
    uint32_t old;
    asm volatile("atom.acquire.gpu.global.cas.b32 %0, [%1], %2, %3;"
                 : "=r"(old)
                 : "l"(p), "r"(cmp), "r"(val)
                 : "memory");
    return old;
}

// Is the coming iteration small enough for one CTA?  A near pile of at most
// p.cta_small vertices, or a far split (empty near pile) of a far pile that
// small.
template <class Mode>
__device__ __forceinline__ bool sssp_small(const TravParams &p, Mode &m, const SsspState &st, unsigned n_near)
{
    if (n_near) return n_near <= p.cta_small;
    return m.ld(u32_of(m.ctl->far_len[st.P % 3])) <= p.cta_small;
}

// One near-far iteration (apps/sssp/kernel.cu:177-306 for the relaxation):
// relax the near pile, or, when it is empty, split the far pile with the
// next threshold.  gwarp/nwarps are the caller's warp numbering for the
// work split (the grid's, or one CTA's).  Returns 0 to go on, 1 when the
// traversal is done (both piles empty), -1 when a barrier reported an error.
template <class Mode, class Vis>
__device__ __forceinline__ int sssp_iter(const TravParams &p, Mode &m, Vis &vis, SsspState &st, unsigned n_near,
                                         unsigned gwarp, unsigned nwarps)
{
    TraversalCtl *ctl = m.ctl;
    const unsigned lane = threadIdx.x & 31;
    const unsigned tid = m.tid;
    const unsigned I = st.I, P = st.P;
    const unsigned long long T = st.T;
    const unsigned slot = I % 3, nslot = (I + 1) % 3, rslot = (I + 2) % 3;
    if (tid == 0) {
        trace_iter(I, n_near | ((unsigned long long)m.ld(u32_of(ctl->far_len[P % 3])) << 32));
        *u32_of(ctl->qlen[rslot]) = 0;
        *u32_of(ctl->claim[rslot]) = 0;
        ctl->hub[rslot].v = 0;
        *u32_of(ctl->hub_claim[rslot]) = 0;
    }
    vis.nq.queue = sel2(p.q, (I + 1));
    vis.nq.len = u32_of(ctl->qlen[nslot]);
    if (n_near > 0) {
        // Relax the near pile (apps/sssp/kernel.cu:177-306).
        vis.threshold = (uint32_t)min(T, 0xFFFFFFFFull);
        vis.near_stamp = near_stamp_of(I);
        vis.phase_stamp = far_stamp_of(st.Ps);
        vis.far_min = kInf;
        vis.fq.queue = sel2(p.far, P);
        vis.fq.len = u32_of(ctl->far_len[P % 3]);
        expand_frontier<Vis, SsspOwn>(vis, p, sel2(p.q, I), n_near, u32_of(ctl->claim[slot]),
                                              &ctl->hub[slot].v, pick_grain(n_near, nwarps, p.uniform), gwarp, nwarps,
                                              lane);
        if constexpr (Vis::kFuse) {
            // Bucket fusion: expand up to p.fuse of this warp's fresh near
            // vertices now, newest first, instead of in the next iteration.
            unsigned budget = n_near <= kFuseMaxPile ? p.fuse : 0u;
            const uint32_t fused = fused_stamp_of(I);
            while (vis.nq.count && budget) {
                const unsigned take = min(32u, vis.nq.count);
                const unsigned base = vis.nq.count - take;
                __syncwarp();
                const uint32_t v = lane < take ? vis.nq.buf[base + lane] : 0u;
                __syncwarp();
                vis.nq.count = base;
                budget = budget > take ? budget - take : 0;
                // The claim: only this warp holds v in this iteration, so
                // the stamp is this iteration's near stamp.  Expanding v is
                // correct whatever the swap finds (a relaxation only ever
                // lowers distances); the swap is what re-queues v after a
                // later improvement.
                if (lane < take) cas_acquire_u32(p.qstamp + v, vis.near_stamp, fused);
                expand_lanes<Vis, SsspOwn>(vis, p, lane < take, v, &ctl->hub[slot].v, lane);
            }
        }
        vis.nq.flush(lane);
        vis.fq.flush(lane);
        unsigned fm = warp_min_u32(vis.far_min);
        if (lane == 0 && fm != kInf) atomicMin(u32_of(ctl->far_min[P % 3]), fm);
        if (!m.sync()) return -1;
        const unsigned long long hv = m.ld64(&ctl->hub[slot].v);
        if (hv) {
            vis.far_min = kInf;
            expand_hubs<Vis, SsspOwn>(vis, p, (unsigned)(hv >> 32), (unsigned)hv,
                                              u32_of(ctl->hub_claim[slot]), gwarp, nwarps, lane);
            vis.nq.flush(lane);
            vis.fq.flush(lane);
            fm = warp_min_u32(vis.far_min);
            if (lane == 0 && fm != kInf) atomicMin(u32_of(ctl->far_min[P % 3]), fm);
            if (!m.sync()) return -1;
        }
    } else {
        // Near pile drained: split the far pile with the next threshold.
        // This iteration starts phase P + 1; the vertices carried over to
        // its far pile get its phase stamp.
        const unsigned nf = m.ld(u32_of(ctl->far_len[P % 3]));
        if (nf == 0) return 1;
        const unsigned fmin = m.ld(u32_of(ctl->far_min[P % 3]));
        const unsigned long long T_old = T;
        unsigned long long T_new = T_old + p.delta;
        if (fmin != kInf && fmin > T_new)  // skip empty buckets
            T_new = T_old + (unsigned long long)p.delta * ((fmin - T_old + p.delta - 1) / p.delta);
        if (tid == 0) {
            *u32_of(ctl->far_len[(P + 2) % 3]) = 0;
            *u32_of(ctl->far_min[(P + 2) % 3]) = kInf;
        }
        vis.fq.queue = sel2(p.far, (P + 1));
        vis.fq.len = u32_of(ctl->far_len[(P + 1) % 3]);
        const uint32_t carry = far_stamp_of(I);
        const uint32_t *pile = sel2(p.far, P);
        unsigned local_min = kInf;
        const unsigned sgrain = pick_grain(nf, nwarps, p.uniform);
        const ChunkSched cs{(nf + sgrain - 1) / sgrain, nwarps, gwarp, lane, u32_of(ctl->claim[slot])};
        for (unsigned c = cs.first(); c < cs.nchunks; c = cs.next()) {
            const unsigned base = c * sgrain;
            const unsigned end = min(nf, base + sgrain);
            for (unsigned i0 = base; i0 < end; i0 += 32) {
                const unsigned idx = i0 + lane;
                uint32_t v = 0;
                unsigned d = kInf;
                if (idx < end) {
                    v = __ldcg(pile + idx);
                    d = __ldcg(vis.dist + v);
                }
                const bool live = idx < end && d > T_old;
                const bool to_near = live && d <= T_new;
                const bool to_far = live && d > T_new;
                if (to_far) {
                    p.qstamp[v] = carry;
                    local_min = min(local_min, d);
                }
                vis.nq.push(to_near, v, lane);
                vis.fq.push(to_far, v, lane);
            }
        }
        vis.nq.flush(lane);
        vis.fq.flush(lane);
        unsigned fm = warp_min_u32(local_min);
        if (lane == 0 && fm != kInf) atomicMin(u32_of(ctl->far_min[(P + 1) % 3]), fm);
        if (!m.sync()) return -1;
        st.T = T_new;
        st.P = P + 1;
        st.Ps = I;
    }
    st.I = I + 1;
    return 0;
}

// kSolo: a single query (the persistent grid or the single-CTA kernel):
// runs of small iterations may go to the first CTA of a grid launch (needs
// p.cta_small), and the visitor reads interleaved edges and fuses buckets.
// The batched kernel's jobs use the lean body.
// near_buf and far_buf: this warp's kQB-entry push buffers.
template <class Mode, bool kSolo = false, unsigned kQB = kQueueBuf>
__device__ __forceinline__ void sssp_body(const TravParams &p, Mode &m, uint32_t *near_buf, uint32_t *far_buf)
{
    TraversalCtl *ctl = m.ctl;
    const unsigned lane = threadIdx.x & 31;
    const unsigned tid = m.tid, nthreads = m.nthreads, nwarps = m.nwarps, gwarp = m.gwarp;
    uint32_t *dist = reinterpret_cast<uint32_t *>(p.out);

    // Initialise (apps/sssp/kernel.cu:23-35): 0 at src, INF elsewhere; the
    // distances are computed in place in the output array.
    const uint32_t n = p.nnodes;
    for (uint32_t v = tid; v < n; v += nthreads) {
        dist[v] = v == p.src ? 0u : kInf;
        p.qstamp[v] = 0;
    }
    if (tid == 0) {
        p.q[0][0] = p.src;
        *u32_of(ctl->qlen[0]) = 1;
        for (int i = 0; i < 3; i++) *u32_of(ctl->far_min[i]) = kInf;
    }
    if (!m.sync()) return;

    SsspVisitorT<kSolo, kQB> vis;
    vis.edge_dst = p.edge_dst;
    vis.edge_data = p.edge_data;
    vis.edge_dw = p.edge_dw;
    vis.dist = dist;
    vis.qstamp = p.qstamp;
    vis.edges = 0;
    vis.err = &ctl->error;
    vis.err_where = &ctl->error_where;
    vis.vec = p.vec_ok;
    vis.nq.buf = near_buf;
    vis.nq.count = 0;
    vis.nq.cap = p.qcap;
    vis.nq.err = &ctl->error;
    vis.nq.err_where = &ctl->error_where;
    vis.fq = vis.nq;
    vis.fq.buf = far_buf;

    SsspState st{p.delta, 0, 0, 0};
    for (;;) {
        const unsigned n_near = m.ld(u32_of(ctl->qlen[st.I % 3]));
        if (kSolo && Mode::kGrid && p.cta_small && sssp_small(p, m, st, n_near)) {
            // Small iterations: the first CTA runs them alone, with
            // __syncthreads as the barrier, while the other CTAs wait at the
            // grid barrier below; it hands the loop state over there.
            if (blockIdx.x == 0) {
                CtaMode cm{ctl, threadIdx.x, blockDim.x, threadIdx.x >> 5, blockDim.x >> 5, 0};
                unsigned nn = n_near;
                int r = 0;
                do {
                    r = sssp_iter(p, cm, vis, st, nn, threadIdx.x >> 5, blockDim.x >> 5);
                    if (r != 0) break;
                    nn = cm.ld(u32_of(ctl->qlen[st.I % 3]));
                } while (sssp_small(p, cm, st, nn));
                if (threadIdx.x == 0) {
                    ctl->handoff[0].v = st.T;
                    ctl->handoff[1].v = ((unsigned long long)(r > 0) << 63) | ((unsigned long long)st.P << 32) | st.I;
                    ctl->handoff[2].v = st.Ps;
                }
            }
            if (!m.sync()) return;
            const unsigned long long h1 = m.ld64(&ctl->handoff[1].v);
            st.T = m.ld64(&ctl->handoff[0].v);
            st.I = (unsigned)h1;
            st.P = (unsigned)(h1 >> 32) & 0x7FFFFFFFu;
            st.Ps = (unsigned)m.ld64(&ctl->handoff[2].v);
            if (h1 >> 63) break;
            continue;
        }
        const int r = sssp_iter(p, m, vis, st, n_near, gwarp, nwarps);
        if (r < 0) return;
        if (r > 0) break;
    }
    // Every CTA leaves the loop after the same barrier, so all relaxations are
    // done and the output array holds the distances.
    warp_add_u64(&ctl->edges, vis.edges, lane);
    if (tid == 0) {
        ctl->levels = st.P;
        ctl->iterations = m.epoch();
        ctl->threshold = (unsigned)min(st.T, 0xFFFFFFFFull);
    }
}

}  // namespace dev
}  // namespace gft
