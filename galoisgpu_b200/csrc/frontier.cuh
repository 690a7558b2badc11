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
struct TravParams {
    const uint32_t *__restrict__ row_start;
    const uint32_t *__restrict__ edge_dst;
    const int32_t *__restrict__ edge_data;  // SSSP; NULL = every weight 0
    uint32_t nnodes;
    uint32_t src;
    int32_t *out;       // level / dist
    uint32_t *parent;   // BFS parent or NULL
    uint32_t *visited;  // BFS bitmap
    uint32_t *q[2];     // frontier / near pile
    uint32_t *far[2];   // SSSP far pile
    unsigned long long *dt;  // SSSP: (dist << 32) | tag per vertex
    uint32_t *far_stamp;
    uint2 *hubs;
    uint32_t hub_cap;
    uint32_t hub_degree;
    uint32_t qcap;
    uint32_t delta;
    TraversalCtl *ctl;
    unsigned long long timeout_ns;
    int skip_block;
    int vec_ok;
};

// ---------------------------------------------------------------------------
// Visitors: what happens to one edge.
// ---------------------------------------------------------------------------
struct BfsOwn {
    uint32_t u;
};

struct BfsVisitor {
    const uint32_t *__restrict__ edge_dst;
    uint32_t *visited;
    int32_t *level;
    uint32_t *parent;
    int newlevel;
    WarpQueue q;
    unsigned long long edges;  // per lane
    unsigned long long claimed;
    bool vec;

    __device__ __forceinline__ BfsOwn owner(bool has, uint32_t u) const { return BfsOwn{u}; }
    __device__ __forceinline__ bool active(const BfsOwn &) const { return true; }
    __device__ __forceinline__ BfsOwn shfl(const BfsOwn &o, int lane) const
    {
        return BfsOwn{__shfl_sync(kFull, o.u, lane)};
    }

    __device__ __forceinline__ void visit(bool valid, uint32_t dst, const BfsOwn &o, unsigned lane)
    {
        bool mine = false;
        if (valid) {
            edges++;
            uint32_t w = dst >> 5, b = 1u << (dst & 31);
            if (!(__ldcg(visited + w) & b)) {
                mine = !(atomicOr(visited + w, b) & b);
                if (mine) {
                    level[dst] = newlevel;
                    if (parent) parent[dst] = o.u;
                    claimed++;
                }
            }
        }
        q.push(mine, dst, lane);
    }
    __device__ __forceinline__ void edge1(bool valid, uint32_t e, const BfsOwn &o, unsigned lane)
    {
        uint32_t d = valid ? ld_stream(edge_dst + e) : 0u;
        visit(valid, d, o, lane);
    }
    __device__ __forceinline__ void edge4(bool valid, uint32_t e, const BfsOwn &o, unsigned lane)
    {
        uint4 d = valid ? ld_stream4(edge_dst + e) : make_uint4(0, 0, 0, 0);
        visit(valid, d.x, o, lane);
        visit(valid, d.y, o, lane);
        visit(valid, d.z, o, lane);
        visit(valid, d.w, o, lane);
    }
};

struct SsspOwn {
    uint32_t u;
    uint32_t du;
};

// SSSP relaxation on a packed word per vertex, (dist << 32) | tag.  One
// 64-bit atomicMin both lowers the distance and records who lowered it: an
// improvement that leaves the vertex at or under the bucket threshold writes
// this iteration's odd near tag, and it queues the vertex only if the tag it
// replaced differs, so the near pile holds each vertex at most once per
// iteration without a separate stamp array or a second atomic.  An
// improvement above the threshold writes near_tag - 1 and is deduplicated in
// the far pile with a per-phase stamp.
struct SsspVisitor {
    const uint32_t *__restrict__ edge_dst;
    const int32_t *__restrict__ edge_data;
    unsigned long long *dt;
    uint32_t *far_stamp;
    uint32_t near_tag, far_tag;
    unsigned long long threshold;
    WarpQueue nq, fq;
    unsigned far_min;
    unsigned long long edges;
    unsigned *err, *err_where;
    bool vec;

    __device__ __forceinline__ SsspOwn owner(bool has, uint32_t u) const
    {
        return SsspOwn{u, has ? (uint32_t)(__ldcg(dt + u) >> 32) : kInf};
    }
    __device__ __forceinline__ bool active(const SsspOwn &o) const { return o.du != kInf; }
    __device__ __forceinline__ SsspOwn shfl(const SsspOwn &o, int lane) const
    {
        return SsspOwn{__shfl_sync(kFull, o.u, lane), __shfl_sync(kFull, o.du, lane)};
    }

    __device__ __forceinline__ void relax(bool valid, uint32_t v, uint32_t w, const SsspOwn &o, unsigned lane)
    {
        bool to_near = false, to_far = false;
        if (valid) {
            edges++;
            uint32_t nd = o.du + w;  // du < 2^31 and w < 2^32: no wrap in 32 bits is checked below
            if (nd >= kInf || nd < o.du) {
                raise_error(err, err_where, GFT_ERR_OVERFLOW, o.u);
            } else if (nd < (uint32_t)(__ldcg(dt + v) >> 32)) {
                const bool near = nd <= threshold;
                const unsigned long long mine = ((unsigned long long)nd << 32) | (near ? near_tag : near_tag - 1);
                const unsigned long long old = atomicMin(dt + v, mine);
                if (nd < (uint32_t)(old >> 32)) {
                    if (near) {
                        to_near = (uint32_t)old != near_tag;
                    } else {
                        far_min = min(far_min, nd);
                        to_far = atomicExch(far_stamp + v, far_tag) != far_tag;
                    }
                }
            }
        }
        nq.push(to_near, v, lane);
        fq.push(to_far, v, lane);
    }
    __device__ __forceinline__ void edge1(bool valid, uint32_t e, const SsspOwn &o, unsigned lane)
    {
        uint32_t d = 0, w = 0;
        if (valid) {
            d = ld_stream(edge_dst + e);
            if (edge_data) w = (uint32_t)__ldcs(edge_data + e);
        }
        relax(valid, d, w, o, lane);
    }
    __device__ __forceinline__ void edge4(bool valid, uint32_t e, const SsspOwn &o, unsigned lane)
    {
        uint4 d = make_uint4(0, 0, 0, 0), w = make_uint4(0, 0, 0, 0);
        if (valid) {
            d = ld_stream4(edge_dst + e);
            if (edge_data) w = __ldcs(reinterpret_cast<const uint4 *>(edge_data + e));
        }
        relax(valid, d.x, w.x, o, lane);
        relax(valid, d.y, w.y, o, lane);
        relax(valid, d.z, w.z, o, lane);
        relax(valid, d.w, w.w, o, lane);
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

// Expands the frontier `in[0, n)` in chunks of `grain` vertices.  Vertices
// of degree >= hub_degree are recorded in the hub list for the grid-wide hub
// phase instead.
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
            Own o = vis.owner(has, u);
            uint32_t start = 0, deg = 0;
            if (has && vis.active(o)) {
                start = __ldg(p.row_start + u);
                deg = __ldg(p.row_start + u + 1) - start;
            }
            if (deg >= p.hub_degree) {
                unsigned nch = (deg + kHubChunk - 1) / kHubChunk;
                unsigned long long old = atomicAdd(hub_ctr, (1ull << 32) | nch);
                unsigned h = (unsigned)(old >> 32);
                if (h < p.hub_cap) p.hubs[h] = make_uint2(u, (unsigned)old);
                else raise_error(&p.ctl->error, &p.ctl->error_where, GFT_ERR_OVERFLOW, h);
                deg = 0;
            }
            unsigned m = __ballot_sync(kFull, deg >= 32);
            while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t s = __shfl_sync(kFull, start, l), d = __shfl_sync(kFull, deg, l);
                warp_range(vis, s, d, vis.shfl(o, l), lane);
            }
            if (deg >= 32) deg = 0;
            warp_flatten(start, deg, lane, [&](bool valid, int j, uint32_t e) { vis.edge1(valid, e, vis.shfl(o, j), lane); });
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

__device__ __forceinline__ unsigned pick_grain(unsigned n, unsigned nwarps)
{
    // A frontier smaller than one 32-vertex chunk per warp is spread over
    // all warps, so a narrow frontier is not left to a few of them.
    if (n < nwarps * 32u) return max(1u, (n + nwarps - 1) / nwarps);
    unsigned per = n / (nwarps * 32u * 4u);
    return 32u * max(1u, min(8u, per));
}

// ---------------------------------------------------------------------------
// Execution modes.  One traversal runs on a group of threads: the whole
// cooperative grid (GridMode, single queries) or one CTA (CtaMode, batched
// and served queries, whose control block lives in shared memory and whose
// barrier is __syncthreads).  The traversal bodies below are written once
// against this interface.
// ---------------------------------------------------------------------------
struct GridMode {
    GridSync gs;
    TraversalCtl *ctl;
    unsigned tid, nthreads, gwarp, nwarps;
    __device__ __forceinline__ bool sync() { return gs.sync(); }
    __device__ __forceinline__ unsigned ld(unsigned *p) const { return ld_relaxed_u32(p); }
    __device__ __forceinline__ unsigned long long ld64(unsigned long long *p) const { return ld_relaxed_u64(p); }
    __device__ __forceinline__ unsigned epoch() const { return gs.epoch; }
};

struct CtaMode {
    TraversalCtl *ctl;  // in shared memory
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
template <class Mode>
__device__ __forceinline__ void bfs_body(const TravParams &p, Mode &m, uint32_t *warp_buf)
{
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
    }
    if (!m.sync()) return;

    BfsVisitor vis;
    vis.edge_dst = p.edge_dst;
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
    for (;;) {
        const unsigned slot = L % 3, nslot = (L + 1) % 3, rslot = (L + 2) % 3;
        const unsigned n_in = m.ld(u32_of(ctl->qlen[slot]));
        if (n_in == 0) break;
        if (tid == 0) {
            *u32_of(ctl->qlen[rslot]) = 0;
            *u32_of(ctl->claim[rslot]) = 0;
            ctl->hub[rslot].v = 0;
            *u32_of(ctl->hub_claim[rslot]) = 0;
        }
        vis.newlevel = (int)L + 1;
        vis.q.queue = sel2(p.q, (L + 1));
        vis.q.len = u32_of(ctl->qlen[nslot]);
        expand_frontier<BfsVisitor, BfsOwn>(vis, p, sel2(p.q, L), n_in, u32_of(ctl->claim[slot]), &ctl->hub[slot].v,
                                            pick_grain(n_in, nwarps), gwarp, nwarps, lane);
        vis.q.flush(lane);
        if (!m.sync()) return;
        const unsigned long long hv = m.ld64(&ctl->hub[slot].v);
        if (hv) {
            expand_hubs<BfsVisitor, BfsOwn>(vis, p, (unsigned)(hv >> 32), (unsigned)hv, u32_of(ctl->hub_claim[slot]),
                                            gwarp, nwarps, lane);
            vis.q.flush(lane);
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
template <class Mode>
__device__ __forceinline__ void sssp_body(const TravParams &p, Mode &m, uint32_t *near_buf, uint32_t *far_buf)
{
    TraversalCtl *ctl = m.ctl;
    const unsigned lane = threadIdx.x & 31;
    const unsigned tid = m.tid, nthreads = m.nthreads, nwarps = m.nwarps, gwarp = m.gwarp;
    unsigned long long *dt = p.dt;

    // Initialise (apps/sssp/kernel.cu:23-35): 0 at src, INF elsewhere.
    const uint32_t n = p.nnodes;
    for (uint32_t v = tid; v < n; v += nthreads) {
        dt[v] = v == p.src ? 0ull : ((unsigned long long)kInf << 32);
        p.far_stamp[v] = 0;
    }
    if (tid == 0) {
        p.q[0][0] = p.src;
        *u32_of(ctl->qlen[0]) = 1;
        for (int i = 0; i < 3; i++) *u32_of(ctl->far_min[i]) = kInf;
    }
    if (!m.sync()) return;

    SsspVisitor vis;
    vis.edge_dst = p.edge_dst;
    vis.edge_data = p.edge_data;
    vis.dt = dt;
    vis.far_stamp = p.far_stamp;
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

    unsigned long long T = p.delta;  // current bucket threshold (inclusive)
    unsigned I = 0, P = 0;           // iteration, phase
    for (;;) {
        const unsigned slot = I % 3, nslot = (I + 1) % 3, rslot = (I + 2) % 3;
        const unsigned n_near = m.ld(u32_of(ctl->qlen[slot]));
        if (tid == 0) {
            *u32_of(ctl->qlen[rslot]) = 0;
            *u32_of(ctl->claim[rslot]) = 0;
            ctl->hub[rslot].v = 0;
            *u32_of(ctl->hub_claim[rslot]) = 0;
        }
        vis.nq.queue = sel2(p.q, (I + 1));
        vis.nq.len = u32_of(ctl->qlen[nslot]);
        if (n_near > 0) {
            // Relax the near pile (apps/sssp/kernel.cu:177-306).
            vis.threshold = T;
            vis.near_tag = 2 * I + 3;  // odd, distinct per iteration, never the initial 0
            vis.far_tag = P + 1;
            vis.far_min = kInf;
            vis.fq.queue = sel2(p.far, P);
            vis.fq.len = u32_of(ctl->far_len[P % 3]);
            expand_frontier<SsspVisitor, SsspOwn>(vis, p, sel2(p.q, I), n_near, u32_of(ctl->claim[slot]),
                                                  &ctl->hub[slot].v, pick_grain(n_near, nwarps), gwarp, nwarps, lane);
            vis.nq.flush(lane);
            vis.fq.flush(lane);
            unsigned fm = warp_min_u32(vis.far_min);
            if (lane == 0 && fm != kInf) atomicMin(u32_of(ctl->far_min[P % 3]), fm);
            if (!m.sync()) return;
            const unsigned long long hv = m.ld64(&ctl->hub[slot].v);
            if (hv) {
                vis.far_min = kInf;
                expand_hubs<SsspVisitor, SsspOwn>(vis, p, (unsigned)(hv >> 32), (unsigned)hv,
                                                  u32_of(ctl->hub_claim[slot]), gwarp, nwarps, lane);
                vis.nq.flush(lane);
                vis.fq.flush(lane);
                fm = warp_min_u32(vis.far_min);
                if (lane == 0 && fm != kInf) atomicMin(u32_of(ctl->far_min[P % 3]), fm);
                if (!m.sync()) return;
            }
        } else {
            // Near pile drained: split the far pile with the next threshold.
            const unsigned nf = m.ld(u32_of(ctl->far_len[P % 3]));
            if (nf == 0) break;
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
            const uint32_t *pile = sel2(p.far, P);
            unsigned local_min = kInf;
            const unsigned sgrain = pick_grain(nf, nwarps);
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
                        d = (uint32_t)(__ldcg(dt + v) >> 32);
                    }
                    const bool live = idx < end && d > T_old;
                    const bool to_near = live && d <= T_new;
                    const bool to_far = live && d > T_new;
                    if (to_far) {
                        p.far_stamp[v] = P + 2;
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
            if (!m.sync()) return;
            T = T_new;
            P++;
        }
        I++;
    }
    // Every CTA leaves the loop after the same barrier, so all relaxations are
    // done: write the int32 distances.
    for (uint32_t v = tid; v < n; v += nthreads) p.out[v] = (int32_t)(uint32_t)(__ldcg(dt + v) >> 32);
    warp_add_u64(&ctl->edges, vis.edges, lane);
    if (tid == 0) {
        ctl->levels = P;
        ctl->iterations = m.epoch();
        ctl->threshold = (unsigned)min(T, 0xFFFFFFFFull);
    }
}

}  // namespace dev
}  // namespace gft
