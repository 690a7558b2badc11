// traversal.cu -- persistent, cooperative BFS and near-far SSSP kernels for
// sm_100a and their C-ABI launchers (gft_bfs, gft_sssp, *_host).
//
// One launch runs a whole query, like the reference's gg_main_pipe_1_gpu_gb
// (apps/bfs/kernel.cu:312-334, apps/sssp/kernel.cu:355-391), but:
//   * the grid is launched cooperatively and sized from the occupancy API,
//     so it is co-resident by construction, and every grid barrier is a
//     bounded wait (traverse.cuh GridSync);
//   * BFS claims each vertex exactly once with atomicOr on a visited bitmap
//     (V/8 bytes, L2 resident), instead of the reference's racy
//     check-then-write on level[] (apps/bfs/kernel.cu:194-199), so the
//     frontier never holds duplicates and a V-sized queue cannot overflow;
//   * frontier vertices are expanded at three granularities chosen per
//     vertex from its degree: small lists are flattened across the warp
//     (thread granularity), lists of >= 32 edges are streamed by the whole
//     warp with 16-byte loads, and lists of >= hub_degree edges are split in
//     chunks over the whole grid after the vertex phase;
//   * pushes are warp aggregated through shared memory (WarpQueue);
//   * SSSP keeps the reference's near/far structure and its relaxation
//     (dist[u] + w compared, then atomicMin, apps/sssp/kernel.cu:244-259),
//     but splits the far pile by threshold with per-vertex phase stamps
//     (no separate duplicate-removal pass, apps/sssp/kernel.cu:36-66) and
//     skips empty buckets.
#include <string.h>

#include <algorithm>

#include "gft_internal.h"
#include "traverse.cuh"

namespace gft {
namespace dev {

constexpr uint32_t kHubChunk = 2048;  // edges of a hub handled per warp claim
constexpr unsigned kInf = 0x7FFFFFFFu;

__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p) { return __ldcs(p); }
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
    uint32_t *near_stamp, *far_stamp;
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

struct SsspVisitor {
    const uint32_t *__restrict__ edge_dst;
    const int32_t *__restrict__ edge_data;
    unsigned *dist;
    uint32_t *near_stamp, *far_stamp;
    uint32_t near_tag, far_tag;
    unsigned long long threshold;
    WarpQueue nq, fq;
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

    __device__ __forceinline__ void relax(bool valid, uint32_t v, uint32_t w, const SsspOwn &o, unsigned lane)
    {
        bool to_near = false, to_far = false;
        if (valid) {
            edges++;
            uint32_t nd = o.du + w;  // du < 2^31 and w < 2^32: no wrap in 32 bits is checked below
            if (nd >= kInf || nd < o.du) {
                raise_error(err, err_where, GFT_ERR_OVERFLOW, o.u);
            } else if (nd < __ldcg(dist + v)) {
                unsigned old = atomicMin(dist + v, nd);
                if (nd < old) {
                    if (nd <= threshold) {
                        to_near = atomicExch(near_stamp + v, near_tag) != near_tag;
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
    unsigned per = n / (nwarps * 32u * 4u);
    return 32u * max(1u, min(8u, per));
}

// ---------------------------------------------------------------------------
// BFS
// ---------------------------------------------------------------------------
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) bfs_persistent(TravParams p)
{
    constexpr int NW = BLOCK / 32;
    __shared__ uint32_t s_buf[NW][64];
    TraversalCtl *ctl = p.ctl;
    if ((int)blockIdx.x == p.skip_block) return;  // test hook: this CTA never arrives

    const unsigned lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned tid = blockIdx.x * BLOCK + threadIdx.x, nthreads = gridDim.x * BLOCK;
    const unsigned nwarps = nthreads / 32, gwarp = tid / 32;
    GridSync gs{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, gridDim.x, 0, p.timeout_ns};

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
    if (!gs.sync()) return;

    BfsVisitor vis;
    vis.edge_dst = p.edge_dst;
    vis.visited = p.visited;
    vis.level = p.out;
    vis.parent = p.parent;
    vis.edges = 0;
    vis.claimed = 0;
    vis.vec = p.vec_ok;
    vis.q.buf = s_buf[wib];
    vis.q.count = 0;
    vis.q.cap = p.qcap;
    vis.q.err = &ctl->error;
    vis.q.err_where = &ctl->error_where;

    unsigned L = 0;
    for (;;) {
        const unsigned slot = L % 3, nslot = (L + 1) % 3, rslot = (L + 2) % 3;
        const unsigned n_in = ld_relaxed_u32(u32_of(ctl->qlen[slot]));
        if (n_in == 0) break;
        if (tid == 0) {
            *u32_of(ctl->qlen[rslot]) = 0;
            *u32_of(ctl->claim[rslot]) = 0;
            ctl->hub[rslot].v = 0;
            *u32_of(ctl->hub_claim[rslot]) = 0;
        }
        vis.newlevel = (int)L + 1;
        vis.q.queue = p.q[(L + 1) & 1];
        vis.q.len = u32_of(ctl->qlen[nslot]);
        expand_frontier<BfsVisitor, BfsOwn>(vis, p, p.q[L & 1], n_in, u32_of(ctl->claim[slot]), &ctl->hub[slot].v,
                                            pick_grain(n_in, nwarps), gwarp, nwarps, lane);
        vis.q.flush(lane);
        if (!gs.sync()) return;
        const unsigned long long hv = ld_relaxed_u64(&ctl->hub[slot].v);
        if (hv) {
            expand_hubs<BfsVisitor, BfsOwn>(vis, p, (unsigned)(hv >> 32), (unsigned)hv, u32_of(ctl->hub_claim[slot]),
                                            gwarp, nwarps, lane);
            vis.q.flush(lane);
            if (!gs.sync()) return;
        }
        L++;
    }
    warp_add_u64(&ctl->edges, vis.edges, lane);
    warp_add_u64(&ctl->reached, vis.claimed, lane);
    if (tid == 0) {
        ctl->levels = L;
        ctl->iterations = gs.epoch;
    }
}

// ---------------------------------------------------------------------------
// SSSP (near-far)
// ---------------------------------------------------------------------------
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) sssp_persistent(TravParams p)
{
    constexpr int NW = BLOCK / 32;
    __shared__ uint32_t s_near[NW][64];
    __shared__ uint32_t s_far[NW][64];
    TraversalCtl *ctl = p.ctl;
    if ((int)blockIdx.x == p.skip_block) return;

    const unsigned lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned tid = blockIdx.x * BLOCK + threadIdx.x, nthreads = gridDim.x * BLOCK;
    const unsigned nwarps = nthreads / 32, gwarp = tid / 32;
    GridSync gs{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, gridDim.x, 0, p.timeout_ns};
    unsigned *dist = reinterpret_cast<unsigned *>(p.out);

    // Initialise (apps/sssp/kernel.cu:23-35): 0 at src, INF elsewhere.
    const uint32_t n = p.nnodes;
    for (uint32_t v = tid; v < n; v += nthreads) {
        dist[v] = v == p.src ? 0u : kInf;
        p.near_stamp[v] = 0;
        p.far_stamp[v] = 0;
    }
    if (tid == 0) {
        p.q[0][0] = p.src;
        *u32_of(ctl->qlen[0]) = 1;
        for (int i = 0; i < 3; i++) *u32_of(ctl->far_min[i]) = kInf;
    }
    if (!gs.sync()) return;

    SsspVisitor vis;
    vis.edge_dst = p.edge_dst;
    vis.edge_data = p.edge_data;
    vis.dist = dist;
    vis.near_stamp = p.near_stamp;
    vis.far_stamp = p.far_stamp;
    vis.edges = 0;
    vis.err = &ctl->error;
    vis.err_where = &ctl->error_where;
    vis.vec = p.vec_ok;
    vis.nq.buf = s_near[wib];
    vis.nq.count = 0;
    vis.nq.cap = p.qcap;
    vis.nq.err = &ctl->error;
    vis.nq.err_where = &ctl->error_where;
    vis.fq = vis.nq;
    vis.fq.buf = s_far[wib];

    unsigned long long T = p.delta;  // current bucket threshold (inclusive)
    unsigned I = 0, P = 0;           // iteration, phase
    for (;;) {
        const unsigned slot = I % 3, nslot = (I + 1) % 3, rslot = (I + 2) % 3;
        const unsigned n_near = ld_relaxed_u32(u32_of(ctl->qlen[slot]));
        if (tid == 0) {
            *u32_of(ctl->qlen[rslot]) = 0;
            *u32_of(ctl->claim[rslot]) = 0;
            ctl->hub[rslot].v = 0;
            *u32_of(ctl->hub_claim[rslot]) = 0;
        }
        vis.nq.queue = p.q[(I + 1) & 1];
        vis.nq.len = u32_of(ctl->qlen[nslot]);
        if (n_near > 0) {
            // Relax the near pile (apps/sssp/kernel.cu:177-306).
            vis.threshold = T;
            vis.near_tag = I + 1;
            vis.far_tag = P + 1;
            vis.far_min = kInf;
            vis.fq.queue = p.far[P & 1];
            vis.fq.len = u32_of(ctl->far_len[P % 3]);
            expand_frontier<SsspVisitor, SsspOwn>(vis, p, p.q[I & 1], n_near, u32_of(ctl->claim[slot]),
                                                  &ctl->hub[slot].v, pick_grain(n_near, nwarps), gwarp, nwarps, lane);
            vis.nq.flush(lane);
            vis.fq.flush(lane);
            unsigned fm = warp_min_u32(vis.far_min);
            if (lane == 0 && fm != kInf) atomicMin(u32_of(ctl->far_min[P % 3]), fm);
            if (!gs.sync()) return;
            const unsigned long long hv = ld_relaxed_u64(&ctl->hub[slot].v);
            if (hv) {
                vis.far_min = kInf;
                expand_hubs<SsspVisitor, SsspOwn>(vis, p, (unsigned)(hv >> 32), (unsigned)hv,
                                                  u32_of(ctl->hub_claim[slot]), gwarp, nwarps, lane);
                vis.nq.flush(lane);
                vis.fq.flush(lane);
                fm = warp_min_u32(vis.far_min);
                if (lane == 0 && fm != kInf) atomicMin(u32_of(ctl->far_min[P % 3]), fm);
                if (!gs.sync()) return;
            }
        } else {
            // Near pile drained: split the far pile with the next threshold.
            const unsigned nf = ld_relaxed_u32(u32_of(ctl->far_len[P % 3]));
            if (nf == 0) break;
            const unsigned fmin = ld_relaxed_u32(u32_of(ctl->far_min[P % 3]));
            const unsigned long long T_old = T;
            unsigned long long T_new = T_old + p.delta;
            if (fmin != kInf && fmin > T_new)  // skip empty buckets
                T_new = T_old + (unsigned long long)p.delta * ((fmin - T_old + p.delta - 1) / p.delta);
            if (tid == 0) {
                *u32_of(ctl->far_len[(P + 2) % 3]) = 0;
                *u32_of(ctl->far_min[(P + 2) % 3]) = kInf;
            }
            vis.fq.queue = p.far[(P + 1) & 1];
            vis.fq.len = u32_of(ctl->far_len[(P + 1) % 3]);
            const uint32_t *pile = p.far[P & 1];
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
                        d = __ldcg(dist + v);
                    }
                    const bool live = idx < end && d > T_old;
                    const bool to_near = live && d <= T_new;
                    const bool to_far = live && d > T_new;
                    if (to_near) p.near_stamp[v] = I + 1;
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
            if (!gs.sync()) return;
            T = T_new;
            P++;
        }
        I++;
    }
    warp_add_u64(&ctl->edges, vis.edges, lane);
    if (tid == 0) {
        ctl->levels = P;
        ctl->iterations = gs.epoch;
        ctl->threshold = (unsigned)min(T, 0xFFFFFFFFull);
    }
}

// SSSP parent tree from final distances: parent[v] = some u with
// dist[u] + w(u, v) == dist[v].
__global__ void parent_init(uint32_t *parent, uint32_t n, uint32_t src)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        parent[v] = v == src ? src : GFT_NO_PARENT;
}

__global__ void sssp_parent_assign(const uint32_t *__restrict__ row_start, const uint32_t *__restrict__ edge_dst,
                                   const int32_t *__restrict__ edge_data, const int32_t *__restrict__ dist,
                                   uint32_t *parent, uint32_t n, uint32_t src)
{
    const unsigned lane = threadIdx.x & 31;
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = gridDim.x * blockDim.x / 32;
    for (uint32_t u = warp; u < n; u += nwarps) {
        const int32_t du = dist[u];
        if (du == (int32_t)kInf) continue;
        const uint32_t s = row_start[u], e = row_start[u + 1];
        for (uint32_t i = s + lane; i < e; i += 32) {
            const uint32_t v = edge_dst[i];
            const int64_t w = edge_data ? edge_data[i] : 0;
            if (v != src && (int64_t)du + w == (int64_t)dist[v]) parent[v] = u;
        }
    }
}

// V_r and E_r of a result array.
__global__ void reach_stats_kernel(const uint32_t *__restrict__ row_start, const int32_t *__restrict__ val, uint32_t n,
                                   unsigned long long *out)
{
    unsigned long long vr = 0, er = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        if (val[v] != (int32_t)kInf) {
            vr++;
            er += row_start[v + 1] - row_start[v];
        }
    const unsigned lane = threadIdx.x & 31;
    warp_add_u64(out, vr, lane);
    warp_add_u64(out + 1, er, lane);
}

}  // namespace dev

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

// Defaults from the autotuner on a B200 (RMAT-24 BFS, RMAT-20 SSSP and the
// 4096^2 road grid): 1024-thread CTAs for BFS, 512 for SSSP, two CTAs per
// SM, and vertices of degree >= 256 split across the grid.
constexpr uint32_t kDefaultBlockBfs = 1024;
constexpr uint32_t kDefaultBlockSssp = 512;
constexpr uint32_t kDefaultBlocksPerSm = 2;
constexpr uint32_t kDefaultHubDegree = 256;
constexpr uint32_t kDefaultTimeoutMs = 20000;

const void *bfs_kernel_for(int block)
{
    switch (block) {
    case 256: return (const void *)dev::bfs_persistent<256>;
    case 512: return (const void *)dev::bfs_persistent<512>;
    case 1024: return (const void *)dev::bfs_persistent<1024>;
    }
    return nullptr;
}

const void *sssp_kernel_for(int block)
{
    switch (block) {
    case 256: return (const void *)dev::sssp_persistent<256>;
    case 512: return (const void *)dev::sssp_persistent<512>;
    case 1024: return (const void *)dev::sssp_persistent<1024>;
    }
    return nullptr;
}

struct Tune {
    uint32_t block, bps, hub, timeout_ms;
    int skip;
};

Tune resolve_tuning(const gft_tuning *t, bool is_sssp)
{
    Tune r{is_sssp ? kDefaultBlockSssp : kDefaultBlockBfs, kDefaultBlocksPerSm, kDefaultHubDegree, kDefaultTimeoutMs,
           -1};
    if (t) {
        if (t->block_threads) r.block = t->block_threads;
        if (t->blocks_per_sm) r.bps = t->blocks_per_sm;
        if (t->hub_degree) r.hub = t->hub_degree;
        if (t->timeout_ms) r.timeout_ms = t->timeout_ms;
        r.skip = t->test_skip_block;
    }
    return r;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

gft_status finish(gft_engine *e, cudaStream_t stream, const LaunchShape &shape, gft_stats *stats, const char *what)
{
    TraversalCtl *hctl = reinterpret_cast<TraversalCtl *>(e->host_ctl);
    const size_t cold = offsetof(TraversalCtl, error);
    GFT_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char *>(hctl) + cold, reinterpret_cast<char *>(e->ctl.ptr) + cold,
                                 sizeof(TraversalCtl) - cold, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    if (hctl->error)
        return fail((gft_status)hctl->error, "%s: device reported %s (site %u)", what,
                    gft_status_string((gft_status)hctl->error), hctl->error_where);
    if (stats) {
        float ms = 0;
        GFT_CUDA_TRY(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
        stats->levels = hctl->levels;
        stats->iterations = hctl->iterations;
        stats->edges_scanned = hctl->edges;
        stats->pushes = hctl->pushes;
        stats->vertices_reached = hctl->reached;
        stats->kernel_ms = ms;
        stats->grid_blocks = shape.blocks;
        stats->block_threads = shape.block_threads;
    }
    return GFT_OK;
}

}  // namespace

gft_status run_traversal(bool is_sssp, gft_engine *e, const gft_graph *g, uint32_t src, int32_t delta, int32_t *d_out,
                         uint32_t *d_parent, const gft_tuning *tune, cudaStream_t stream, gft_stats *stats)
{
    const char *what = is_sssp ? "gft_sssp" : "gft_bfs";
    GFT_TRY(check_engine_graph(e, g));
    const DeviceGraph &G = g->g;
    if (!d_out) return fail(GFT_ERR_INVALID_ARG, "%s: output pointer is NULL", what);
    if (src >= G.nnodes) return fail(GFT_ERR_INVALID_ARG, "%s: source %u out of range (nnodes %u)", what, src, G.nnodes);
    if (is_sssp && delta <= 0) return fail(GFT_ERR_INVALID_ARG, "%s: delta must be > 0 (got %d)", what, delta);
    Tune t = resolve_tuning(tune, is_sssp);
    const void *kern = is_sssp ? sssp_kernel_for(t.block) : bfs_kernel_for(t.block);
    if (!kern) return fail(GFT_ERR_INVALID_ARG, "%s: block_threads must be 256, 512 or 1024", what);
    if (t.hub < 32) t.hub = 32;
    GFT_CUDA_TRY(cudaSetDevice(e->device));
    LaunchShape shape;
    GFT_TRY(resolve_shape(e, kern, (int)t.block, (int)t.bps, 0, &shape));

    // Scratch layout.
    const uint32_t n = G.nnodes;
    const uint32_t qcap = n;
    const uint32_t hub_cap = std::min<uint64_t>(n, (uint64_t)G.nedges / t.hub + 1);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += align256(bytes);
        return o;
    };
    size_t o_q0 = take((size_t)qcap * 4), o_q1 = take((size_t)qcap * 4);
    size_t o_hubs = take((size_t)hub_cap * 8);
    size_t o_vis = 0, o_f0 = 0, o_f1 = 0, o_ns = 0, o_fs = 0;
    if (is_sssp) {
        o_f0 = take((size_t)qcap * 4);
        o_f1 = take((size_t)qcap * 4);
        o_ns = take((size_t)n * 4);
        o_fs = take((size_t)n * 4);
    } else {
        o_vis = take((size_t)((n + 31) / 32) * 4);
    }
    GFT_TRY(e->scratch.ensure(off));
    char *base = reinterpret_cast<char *>(e->scratch.ptr);

    dev::TravParams p{};
    p.row_start = G.row_start;
    p.edge_dst = G.edge_dst;
    p.edge_data = G.edge_data;
    p.nnodes = n;
    p.src = src;
    p.out = d_out;
    p.parent = is_sssp ? nullptr : d_parent;
    p.q[0] = reinterpret_cast<uint32_t *>(base + o_q0);
    p.q[1] = reinterpret_cast<uint32_t *>(base + o_q1);
    p.hubs = reinterpret_cast<uint2 *>(base + o_hubs);
    if (is_sssp) {
        p.far[0] = reinterpret_cast<uint32_t *>(base + o_f0);
        p.far[1] = reinterpret_cast<uint32_t *>(base + o_f1);
        p.near_stamp = reinterpret_cast<uint32_t *>(base + o_ns);
        p.far_stamp = reinterpret_cast<uint32_t *>(base + o_fs);
    } else {
        p.visited = reinterpret_cast<uint32_t *>(base + o_vis);
    }
    p.hub_cap = hub_cap;
    p.hub_degree = t.hub;
    p.qcap = qcap;
    p.delta = (uint32_t)delta;
    p.ctl = reinterpret_cast<TraversalCtl *>(e->ctl.ptr);
    p.timeout_ns = (unsigned long long)t.timeout_ms * 1000000ull;
    p.skip_block = t.skip;
    p.vec_ok = ((uintptr_t)G.edge_dst % 16 == 0) && (!G.edge_data || (uintptr_t)G.edge_data % 16 == 0);

    GFT_CUDA_TRY(cudaMemsetAsync(e->ctl.ptr, 0, sizeof(TraversalCtl), stream));
    void *args[] = {&p};
    GFT_CUDA_TRY(cudaEventRecord(e->ev0, stream));
    GFT_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(shape.blocks), dim3(shape.block_threads), args, 0, stream));
    GFT_CUDA_TRY(cudaEventRecord(e->ev1, stream));
    if (is_sssp && d_parent) {
        dev::parent_init<<<e->sms * 4, 256, 0, stream>>>(d_parent, n, src);
        GFT_CUDA_TRY(cudaGetLastError());
        dev::sssp_parent_assign<<<e->sms * 8, 256, 0, stream>>>(G.row_start, G.edge_dst, G.edge_data, d_out, d_parent,
                                                                  n, src);
        GFT_CUDA_TRY(cudaGetLastError());
    }
    return finish(e, stream, shape, stats, what);
}

gft_status reach_stats(const gft_graph *g, const int32_t *d_val, cudaStream_t stream, uint64_t *v_r, uint64_t *e_r)
{
    unsigned long long *d = nullptr, h[2] = {0, 0};
    GFT_CUDA_TRY(cudaSetDevice(g->g.device));
    GFT_CUDA_TRY(cudaMallocAsync(&d, 16, stream));
    GFT_CUDA_TRY(cudaMemsetAsync(d, 0, 16, stream));
    dev::reach_stats_kernel<<<592, 256, 0, stream>>>(g->g.row_start, d_val, g->g.nnodes, d);
    cudaError_t le = cudaGetLastError();
    GFT_CUDA_TRY(cudaMemcpyAsync(h, d, 16, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaFreeAsync(d, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    GFT_CUDA_TRY(le);
    if (v_r) *v_r = h[0];
    if (e_r) *e_r = h[1];
    return GFT_OK;
}

}  // namespace gft

using namespace gft;

extern "C" {

gft_status gft_bfs(gft_engine *e, const gft_graph *g, uint32_t src, int32_t *d_level, uint32_t *d_parent,
                   const gft_tuning *tune, void *stream, gft_stats *stats)
{
    if (!e) return fail(GFT_ERR_INVALID_ARG, "gft_bfs: engine is NULL");
    std::lock_guard<std::mutex> lk(e->mu);
    return run_traversal(false, e, g, src, 0, d_level, d_parent, tune, (cudaStream_t)stream, stats);
}

gft_status gft_sssp(gft_engine *e, const gft_graph *g, uint32_t src, int32_t delta, int32_t *d_dist,
                    uint32_t *d_parent, const gft_tuning *tune, void *stream, gft_stats *stats)
{
    if (!e) return fail(GFT_ERR_INVALID_ARG, "gft_sssp: engine is NULL");
    std::lock_guard<std::mutex> lk(e->mu);
    return run_traversal(true, e, g, src, delta, d_dist, d_parent, tune, (cudaStream_t)stream, stats);
}

static gft_status run_host(bool is_sssp, gft_engine *e, const gft_graph *g, uint32_t src, int32_t delta,
                           int32_t *h_out, uint32_t *h_parent, const gft_tuning *tune, void *stream_, gft_stats *stats)
{
    const char *what = is_sssp ? "gft_sssp_host" : "gft_bfs_host";
    if (!e) return fail(GFT_ERR_INVALID_ARG, "%s: engine is NULL", what);
    if (!h_out) return fail(GFT_ERR_INVALID_ARG, "%s: output pointer is NULL", what);
    std::lock_guard<std::mutex> lk(e->mu);
    GFT_TRY(check_engine_graph(e, g));
    cudaStream_t stream = (cudaStream_t)stream_;
    const size_t n = g->g.nnodes;
    GFT_TRY(e->aux.ensure(align256(n * 4) + (h_parent ? align256(n * 4) : 0)));
    int32_t *d_out = reinterpret_cast<int32_t *>(e->aux.ptr);
    uint32_t *d_par = h_parent ? reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(e->aux.ptr) + align256(n * 4))
                               : nullptr;
    GFT_TRY(run_traversal(is_sssp, e, g, src, delta, d_out, d_par, tune, stream, stats));
    GFT_CUDA_TRY(cudaMemcpyAsync(h_out, d_out, n * 4, cudaMemcpyDeviceToHost, stream));
    if (h_parent) GFT_CUDA_TRY(cudaMemcpyAsync(h_parent, d_par, n * 4, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    return GFT_OK;
}

gft_status gft_bfs_host(gft_engine *e, const gft_graph *g, uint32_t src, int32_t *h_level, uint32_t *h_parent,
                        const gft_tuning *tune, void *stream, gft_stats *stats)
{
    return run_host(false, e, g, src, 0, h_level, h_parent, tune, stream, stats);
}

gft_status gft_sssp_host(gft_engine *e, const gft_graph *g, uint32_t src, int32_t delta, int32_t *h_dist,
                         uint32_t *h_parent, const gft_tuning *tune, void *stream, gft_stats *stats)
{
    return run_host(true, e, g, src, delta, h_dist, h_parent, tune, stream, stats);
}

gft_status gft_reach_stats(const gft_graph *g, const int32_t *d_val, void *stream, uint64_t *v_r, uint64_t *e_r)
{
    if (!g || !d_val) return fail(GFT_ERR_INVALID_ARG, "gft_reach_stats: null argument");
    return reach_stats(g, d_val, (cudaStream_t)stream, v_r, e_r);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free BFS (gft_bfs_noalloc)
//
// For callers that must not allocate device memory themselves or through
// the library: code running while another component owns the device's
// memory (a caching allocator that has reserved the free memory, or a
// framework that forbids allocations outside its own pool), and hot paths
// where cudaMalloc / cudaFree are not allowed because of their implicit
// synchronisation.  The traversal scratch (control block, two frontier
// queues, visited bitmap, hub list) lives in one file-scope device array of
// fixed size, sized for graphs of up to kNoAllocMaxNodes vertices; every GPU
// that loads libgft holds it until the process exits.
//
// The array's name is only a host-side stand-in in host code, so its device
// address is looked up once per device with cudaGetSymbolAddress (with that
// device current) on the first call for that device; make that first call
// before any stream capture.  All calls share the array: the control block
// is cleared on the call's stream before the launch, and calls whose work
// overlaps on the GPU race on the scratch, so serialise them (one stream, or
// events between streams).
// ---------------------------------------------------------------------------
namespace gft {
namespace {

constexpr uint32_t kNoAllocMaxNodes = 1u << 20;  // 1,048,576 vertices
constexpr int kNoAllocBlock = 512;

constexpr size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kNoAllocCtlBytes = na_align(sizeof(TraversalCtl));
constexpr size_t kNoAllocQueueBytes = na_align((size_t)kNoAllocMaxNodes * 4);
constexpr size_t kNoAllocBitmapBytes = na_align((size_t)(kNoAllocMaxNodes / 32) * 4);
constexpr size_t kNoAllocHubBytes = na_align((size_t)kNoAllocMaxNodes * 8);
constexpr size_t kNoAllocBytes = kNoAllocCtlBytes + 2 * kNoAllocQueueBytes + kNoAllocBitmapBytes + kNoAllocHubBytes;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void *g_noalloc_addr[256];

gft_status noalloc_scratch(int device, char **out)
{
    if (device < 0 || device >= 256) return fail(GFT_ERR_INVALID_ARG, "gft_bfs_noalloc: device %d", device);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(GFT_ERR_CUDA, "gft_bfs_noalloc: cudaGetSymbolAddress failed on device %d: %s", device,
                        cudaGetErrorString(e));
        g_noalloc_addr[device] = p;
    }
    *out = static_cast<char *>(g_noalloc_addr[device]);
    return GFT_OK;
}

}  // namespace
}  // namespace gft

extern "C" gft_status gft_bfs_noalloc(const gft_graph *g, uint32_t src, int32_t *d_level, uint32_t *d_parent,
                                      const gft_tuning *tune, void *stream_, gft_stats *stats)
{
    using namespace gft;
    if (!g || !d_level) return fail(GFT_ERR_INVALID_ARG, "gft_bfs_noalloc: null argument");
    const DeviceGraph &G = g->g;
    if (G.nnodes > kNoAllocMaxNodes)
        return fail(GFT_ERR_INVALID_ARG, "gft_bfs_noalloc: %u vertices exceed the fixed scratch limit of %u",
                    G.nnodes, kNoAllocMaxNodes);
    if (src >= G.nnodes)
        return fail(GFT_ERR_INVALID_ARG, "gft_bfs_noalloc: source %u out of range (nnodes %u)", src, G.nnodes);
    uint32_t hub = (tune && tune->hub_degree) ? std::max<uint32_t>(tune->hub_degree, 32) : 4096;
    uint32_t timeout_ms = (tune && tune->timeout_ms) ? tune->timeout_ms : 20000;
    cudaStream_t stream = (cudaStream_t)stream_;
    GFT_CUDA_TRY(cudaSetDevice(G.device));
    char *base = nullptr;
    GFT_TRY(noalloc_scratch(G.device, &base));

    const void *kern = (const void *)dev::bfs_persistent<kNoAllocBlock>;
    int sms = 0, occ = 0;
    GFT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, G.device));
    GFT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kNoAllocBlock, 0));
    if (occ <= 0) return fail(GFT_ERR_NOT_SUPPORTED, "gft_bfs_noalloc: kernel cannot be resident");
    const int blocks = sms * std::min(occ, 2);

    dev::TravParams p{};
    p.row_start = G.row_start;
    p.edge_dst = G.edge_dst;
    p.edge_data = nullptr;
    p.nnodes = G.nnodes;
    p.src = src;
    p.out = d_level;
    p.parent = d_parent;
    p.ctl = reinterpret_cast<TraversalCtl *>(base);
    p.q[0] = reinterpret_cast<uint32_t *>(base + kNoAllocCtlBytes);
    p.q[1] = reinterpret_cast<uint32_t *>(base + kNoAllocCtlBytes + kNoAllocQueueBytes);
    p.visited = reinterpret_cast<uint32_t *>(base + kNoAllocCtlBytes + 2 * kNoAllocQueueBytes);
    p.hubs = reinterpret_cast<uint2 *>(base + kNoAllocCtlBytes + 2 * kNoAllocQueueBytes + kNoAllocBitmapBytes);
    p.hub_cap = (uint32_t)std::min<uint64_t>(G.nnodes, (uint64_t)G.nedges / hub + 1);
    p.hub_degree = hub;
    p.qcap = G.nnodes;
    p.timeout_ns = (unsigned long long)timeout_ms * 1000000ull;
    p.skip_block = -1;
    p.vec_ok = ((uintptr_t)G.edge_dst % 16 == 0);

    // The control block must start at zero for every call.
    GFT_CUDA_TRY(cudaMemsetAsync(p.ctl, 0, sizeof(TraversalCtl), stream));
    void *args[] = {&p};
    GFT_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(kNoAllocBlock), args, 0, stream));
    TraversalCtl h;
    const size_t cold = offsetof(TraversalCtl, error);
    GFT_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char *>(&h) + cold, reinterpret_cast<char *>(p.ctl) + cold,
                                 sizeof(TraversalCtl) - cold, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h.error)
        return fail((gft_status)h.error, "gft_bfs_noalloc: device reported %s (site %u)",
                    gft_status_string((gft_status)h.error), h.error_where);
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->levels = h.levels;
        stats->iterations = h.iterations;
        stats->edges_scanned = h.edges;
        stats->vertices_reached = h.reached + 1;
        stats->grid_blocks = blocks;
        stats->block_threads = kNoAllocBlock;
    }
    return GFT_OK;
}
