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

#include "frontier.cuh"
#include "gft_internal.h"

namespace gft {
namespace dev {

constexpr int kCtaBlock = 1024;  // threads of the single-CTA kernels

// ---------------------------------------------------------------------------
// Single-query kernels: the whole cooperative grid is one group.
// ---------------------------------------------------------------------------
// Push buffers of the grid-wide kernels (the queue tile, QB entries per
// warp) are a template parameter: 64, 128 or 256, picked per launch
// (gft_tuning.queue_tile).  BFS defaults to 256 (one buffer per warp, at
// most 32 KB per CTA), as the grid-wide SSSP kernel.
constexpr unsigned kBfsGridQueueBuf = 256;

template <int BLOCK, unsigned QB>
// Resident threads per SM the grid BFS kernel's register budget is set for:
// 2048 (32 registers a thread, 42 bytes spilled).  A 64-register build
// (1024, no spills) was slower on RMAT-24 BFS: best 0.89 ms against 0.70 ms
// (512 x 4) and 0.74 ms (1024 x 2); more warps in flight hide more of the
// traversal's memory latency than the spills cost.
#ifndef GFT_BFS_THREADS_PER_SM
#define GFT_BFS_THREADS_PER_SM 2048
#endif
__global__ void __launch_bounds__(BLOCK, GFT_BFS_THREADS_PER_SM / BLOCK) bfs_persistent(TravParams p)
{
    __shared__ uint32_t s_buf[BLOCK / 32][QB];
    if ((int)blockIdx.x == p.skip_block) return;  // test hook: this CTA never arrives
    TraversalCtl *ctl = p.ctl;
    const unsigned tid = blockIdx.x * BLOCK + threadIdx.x, nthreads = gridDim.x * BLOCK;
    GridMode m{{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, gridDim.x, 0, p.timeout_ns},
               ctl, tid, nthreads, tid / 32, nthreads / 32};
    bfs_body<GridMode, false, QB>(p, m, s_buf[threadIdx.x >> 5]);
}

// Default push buffers of the grid-wide SSSP kernel: 256 entries per warp up
// to 512 threads per CTA (32 KB), halving the reservations on the piles'
// length counters (road 4096^2: 3.74 -> 3.60 ms; 64 entries: 4.80 ms);
// 1024-thread CTAs keep 128, the most that fits in 48 KB of static shared
// memory (near and far buffers).
template <int BLOCK>
constexpr unsigned kSsspGridQueueBuf = BLOCK <= 512 ? 256 : kQueueBuf;

template <int BLOCK, unsigned QB>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) sssp_persistent(TravParams p)
{
    static_assert(2 * (BLOCK / 32) * QB * 4 <= 48 * 1024, "near and far buffers exceed static shared memory");
    __shared__ uint32_t s_near[BLOCK / 32][QB];
    __shared__ uint32_t s_far[BLOCK / 32][QB];
    if ((int)blockIdx.x == p.skip_block) return;
    TraversalCtl *ctl = p.ctl;
    const unsigned tid = blockIdx.x * BLOCK + threadIdx.x, nthreads = gridDim.x * BLOCK;
    GridMode m{{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, gridDim.x, 0, p.timeout_ns},
               ctl, tid, nthreads, tid / 32, nthreads / 32};
    sssp_body<GridMode, true, QB>(p, m, s_near[threadIdx.x >> 5], s_far[threadIdx.x >> 5]);
}

// ---------------------------------------------------------------------------
// Single-CTA kernels for small graphs.  A small graph's frontiers are small
// and its levels many (the 256^2 grid: 511 levels of at most 256 vertices),
// so a grid barrier per level dominates.  One CTA runs the whole traversal
// with its control block in shared memory and __syncthreads as the barrier
// (CtaMode, as the batched kernel's small jobs), then copies the results to
// the engine's control block.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void publish_cta_result(const TraversalCtl &s, TraversalCtl *g)
{
    g->error = s.error;
    g->error_where = s.error_where;
    g->levels = s.levels;
    g->iterations = s.iterations;
    g->threshold = s.threshold;
    g->edges = s.edges;
    g->pushes = s.pushes;
    g->reached = s.reached;
}

// Graphs of at most this many vertices keep the BFS visited bitmap in the
// CTA's shared memory (16 KB): every probe and claim of a level then stays
// on the SM.
constexpr uint32_t kCtaLocalBitsNodes = 1u << 17;

template <bool kLocalBits>
__global__ void __launch_bounds__(kCtaBlock, 1) bfs_single_cta(TravParams p)
{
    __shared__ TraversalCtl s_ctl;
    __shared__ uint32_t s_buf[kCtaBlock / 32][kQueueBuf];
    __shared__ uint32_t s_bits[kLocalBits ? kCtaLocalBitsNodes / 32 : 1];
    for (unsigned i = threadIdx.x; i < sizeof(TraversalCtl) / 4; i += kCtaBlock)
        reinterpret_cast<unsigned *>(&s_ctl)[i] = 0;
    __syncthreads();
    TraversalCtl *gctl = p.ctl;
    p.ctl = &s_ctl;
    if (kLocalBits) p.visited = s_bits;  // bfs_body clears the first (nnodes + 31) / 32 words
    CtaMode m{&s_ctl, threadIdx.x, kCtaBlock, threadIdx.x >> 5, kCtaBlock / 32, 0};
    bfs_body<CtaMode, kLocalBits>(p, m, s_buf[threadIdx.x >> 5]);
    __syncthreads();
    if (threadIdx.x == 0) publish_cta_result(s_ctl, gctl);
}

// ---------------------------------------------------------------------------
// One CTA, a thread per frontier vertex: BFS on small graphs of uniform low
// degree (grids, road networks).  Their levels are many and their frontiers
// a few hundred vertices, so a level costs its critical path, and the
// general kernel's balancing (prefix sums and shuffle searches over the
// warp's edges, per-warp queue buffers) costs more than the few edges it
// balances.  The visited bitmap and the first kLaneQueueHead entries of both
// frontier queues live in shared memory; a queue's later entries go to the
// engine's global queue at the same index.  With the graph's BFS slots (16
// bytes per vertex holding its up to 4 destinations, all inside the graph),
// a vertex's edges are one load instead of a row lookup and then an edge
// load, and its four claims go out with no range check; a vertex of more
// edges (or any vertex of a graph without slots) is walked through the CSR
// four edges at a time.  A level is: slot loads, claims in shared memory,
// one shared atomic per warp step for the appends, one __syncthreads.  The
// level costs about the instructions of its longest warp, so the common
// path keeps them few: edges are counted per vertex, and a warp step whose
// appends all fit the shared queue head stores them with no per-vertex
// check.  Always top-down: levels are the same in either direction, and
// these graphs' frontiers stay small.
// ---------------------------------------------------------------------------
constexpr uint32_t kLaneQueueHead = 8192;
constexpr size_t kLaneSmemBytes = (kCtaLocalBitsNodes / 32 + 2 * (size_t)kLaneQueueHead) * 4;

// One warp step's appends: claimed destinations v[k] (mine[k]) of frontier
// vertex u go to the next frontier and get their level.  Each vertex is
// claimed once, so a level appends fewer than qcap = nnodes entries.
template <bool kParent>
__device__ __forceinline__ void lanes_append(const TravParams &p, const bool (&mine)[4], const uint32_t (&v)[4],
                                             uint32_t u, unsigned *len_next, uint32_t *out_head,
                                             uint32_t *out_tail, int32_t level, unsigned *err, unsigned lane,
                                             unsigned &claimed)
{
    unsigned mask[4], total = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        mask[k] = __ballot_sync(kFull, mine[k]);
        total += __popc(mask[k]);
    }
    if (total == 0) return;  // warp uniform
    unsigned at = 0;
    if (lane == 0) {
        at = atomicAdd(len_next, total);
        claimed += total;
    }
    at = __shfl_sync(kFull, at, 0);
    const unsigned lt = lanemask_lt();
    if (at + total <= kLaneQueueHead) {  // warp uniform
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (mine[k]) {
                out_head[at + __popc(mask[k] & lt)] = v[k];
                p.out[v[k]] = level;
                if (kParent) p.parent[v[k]] = u;
            }
            at += __popc(mask[k]);
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (mine[k]) {
            const unsigned slot = at + __popc(mask[k] & lt);
            if (slot < kLaneQueueHead)
                out_head[slot] = v[k];
            else if (slot < p.qcap)
                out_tail[slot] = v[k];
            else
                atomicCAS(err, 0u, (unsigned)GFT_ERR_OVERFLOW);
            p.out[v[k]] = level;
            if (kParent) p.parent[v[k]] = u;
        }
        at += __popc(mask[k]);
    }
}

template <int BLOCK, bool kParent>
__global__ void __launch_bounds__(BLOCK, 1) bfs_cta_lanes(TravParams p)
{
    extern __shared__ __align__(16) uint32_t s_lane[];
    uint32_t *bits = s_lane;
    uint32_t *const head0 = bits + kCtaLocalBitsNodes / 32, *const head1 = head0 + kLaneQueueHead;
    __shared__ unsigned s_len[3];
    __shared__ unsigned s_err;
    const unsigned tid = threadIdx.x, lane = tid & 31;
    const uint32_t n = p.nnodes, nwords = (n + 31) >> 5;
    for (uint32_t v = tid; v < n; v += BLOCK) {
        p.out[v] = v == p.src ? 0 : (int32_t)kInf;
        if (kParent) p.parent[v] = v == p.src ? p.src : GFT_NO_PARENT;
    }
    for (uint32_t w = tid; w < nwords; w += BLOCK) bits[w] = w == (p.src >> 5) ? 1u << (p.src & 31) : 0u;
    if (tid == 0) {
        head0[0] = p.src;
        s_len[0] = 1;
        s_len[1] = 0;
        s_len[2] = 0;
        s_err = 0;
    }
    __syncthreads();

    const uint4 *__restrict__ slots = p.bfs_slots;
    const uint4 none = make_uint4(kBfsSlotNone, kBfsSlotNone, kBfsSlotNone, kBfsSlotNone);
    // Per-thread counts fit 32 bits: graphs here have at most 2^17 vertices
    // of at most kUniformDegree edges.
    unsigned edges = 0, claimed = 0;
    unsigned L = 0;
    // Lengths are triple-buffered: s_len[c] is read by every thread at the
    // top of a level, s_len[nx] collects the level's appends, and s_len[cl]
    // (read at the top of the previous level, before its barrier) is
    // cleared for the next level; the three rotate each level, as the two
    // queues swap.
    unsigned c = 0, nx = 1, cl = 2;
    const uint32_t *in_head = head0, *in_tail = p.q[0];
    uint32_t *out_head = head1, *out_tail = p.q[1];
    for (;;) {
        const unsigned n_in = *(volatile unsigned *)&s_len[c];
        if (n_in == 0) break;
        if (tid == 0) s_len[cl] = 0;
        unsigned *len_next = &s_len[nx];
        const int32_t next_level = (int32_t)L + 1;
        for (unsigned base = tid - lane; base < n_in; base += BLOCK) {  // warp-uniform trip count
            const unsigned i = base + lane;
            uint32_t u = 0;
            uint4 sl = none;
            bool csr = false;
            if (i < n_in) {
                u = i < kLaneQueueHead ? in_head[i] : __ldcg(in_tail + i);
                if (slots) sl = __ldg(slots + u);
                csr = !slots || sl.x == kBfsSlotWide;
                if (csr) sl = none;
            }
            // Slot destinations.  The four claims go out together, with no
            // probe first: a shared-memory atomic costs about what a load
            // does, and this keeps one shared round trip per step.
            {
                const uint32_t v[4] = {sl.x, sl.y, sl.z, sl.w};
                bool mine[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const bool valid = v[k] != kBfsSlotNone;
                    const uint32_t b = 1u << (v[k] & 31);
                    uint32_t old = b;
                    if (valid) old = atomicOr(bits + (v[k] >> 5), b);
                    mine[k] = !(old & b);
                    edges += valid;
                }
                lanes_append<kParent>(p, mine, v, u, len_next, out_head, out_tail, next_level, &s_err, lane,
                                      claimed);
            }
            // Vertices read through the CSR, four edges a step.
            if (__any_sync(kFull, csr)) {
                uint32_t s = 0, deg = 0;
                if (csr) {
                    s = __ldg(p.row_start + u);
                    deg = __ldg(p.row_start + u + 1) - s;
                }
                edges += deg;
                const unsigned max_deg = __reduce_max_sync(kFull, deg);
                for (unsigned j = 0; j < max_deg; j += 4) {
                    uint32_t v[4];
                    bool mine[4];
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        v[k] = j + k < deg ? __ldg(p.edge_dst + s + j + k) : 0u;
                        mine[k] = false;
                        if (j + k < deg) {
                            const uint32_t b = 1u << (v[k] & 31);
                            if (v[k] < n)
                                mine[k] = !(atomicOr(bits + (v[k] >> 5), b) & b);
                            else
                                atomicCAS(&s_err, 0u, (unsigned)GFT_ERR_FORMAT);
                        }
                    }
                    lanes_append<kParent>(p, mine, v, u, len_next, out_head, out_tail, next_level, &s_err, lane,
                                          claimed);
                }
            }
        }
        // An error (a destination outside the graph, a queue overrun) skips
        // the access it found and is reported after the traversal, so the
        // level ends with a plain barrier.
        __syncthreads();
        L++;
        const unsigned c0 = c;
        c = nx;
        nx = cl;
        cl = c0;
        const uint32_t *ih = in_head, *it = in_tail;
        in_head = out_head;
        in_tail = out_tail;
        out_head = const_cast<uint32_t *>(ih);
        out_tail = const_cast<uint32_t *>(it);
    }
    warp_add_u64(&p.ctl->edges, edges, lane);
    warp_add_u64(&p.ctl->reached, claimed, lane);
    if (tid == 0) {
        p.ctl->levels = L;
        p.ctl->iterations = L + 1;  // barriers, as the general kernel counts them
        if (s_err) p.ctl->error = s_err;
    }
}

#ifndef GFT_LANES_BLOCK
#define GFT_LANES_BLOCK 0  // 0: chosen from the vertex count
#endif
__host__ __forceinline__ int lanes_block_for(uint32_t nnodes)
{
    if (GFT_LANES_BLOCK) return GFT_LANES_BLOCK;
    // Idle warps still pay for every level's loop top and barrier: the
    // 256^2 grid (frontiers <= 256) is fastest at 256 threads, the 362^2
    // road graph (random sources, frontiers of 700 and more) at 1024.
    // Graphs here have at most kCtaLocalBitsNodes vertices.
    return nnodes <= (1u << 16) ? 256 : 1024;
}
template <bool kParent>
__host__ inline const void *lanes_kernel_for(int block)
{
    return block <= 256   ? (const void *)bfs_cta_lanes<256, kParent>
           : block <= 512 ? (const void *)bfs_cta_lanes<512, kParent>
                          : (const void *)bfs_cta_lanes<1024, kParent>;
}
__host__ inline const void *lanes_kernel_for(int block, bool parent)
{
    return parent ? lanes_kernel_for<true>(block) : lanes_kernel_for<false>(block);
}
__host__ inline bool is_lanes_kernel(const void *k)
{
    for (int b : {256, 512, 1024})
        if (k == lanes_kernel_for<false>(b) || k == lanes_kernel_for<true>(b)) return true;
    return false;
}

__global__ void __launch_bounds__(kCtaBlock, 1) sssp_single_cta(TravParams p)
{
    __shared__ TraversalCtl s_ctl;
    __shared__ uint32_t s_near[kCtaBlock / 32][kQueueBuf];
    __shared__ uint32_t s_far[kCtaBlock / 32][kQueueBuf];
    for (unsigned i = threadIdx.x; i < sizeof(TraversalCtl) / 4; i += kCtaBlock)
        reinterpret_cast<unsigned *>(&s_ctl)[i] = 0;
    __syncthreads();
    TraversalCtl *gctl = p.ctl;
    p.ctl = &s_ctl;
    CtaMode m{&s_ctl, threadIdx.x, kCtaBlock, threadIdx.x >> 5, kCtaBlock / 32, 0};
    sssp_body<CtaMode, true>(p, m, s_near[threadIdx.x >> 5], s_far[threadIdx.x >> 5]);
    __syncthreads();
    if (threadIdx.x == 0) publish_cta_result(s_ctl, gctl);
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
// SSSP iterations of at most this many vertices (near pile, or far pile at a
// split) run on the grid's first CTA alone, by default on graphs of uniform
// degree: a __syncthreads saves the grid barrier, but one CTA's warps take
// longer over the pile, so only tiny piles gain (road 4096^2: 4.81 ->
// 4.73 ms at 256, slower from 1024 up; R-MAT gains nothing).
constexpr uint32_t kDefaultCtaSmall = 256;
// SSSP near vertices a warp may expand itself in the iteration that found
// them (bucket fusion, on piles of at most dev::kFuseMaxPile vertices), by
// default on graphs of uniform degree.  Road 4096^2, 3 sources: 4.11 ms
// without (delta 40000), 3.66 ms at 256 with delta 20000 (iterations
// 203 -> ~70); road 2048^2 gains ~20%; R-MAT loses (4.0 -> 4.4 ms on
// RMAT-22), where a warp's chased vertices are hubs' neighbourhoods and
// unbalance the grid.
constexpr uint32_t kDefaultFuse = 256;
// Graphs up to this size run on one CTA by default: their frontiers are
// small enough for 1024 threads, and a __syncthreads per level is several
// times cheaper than a grid barrier (BFS on the 256^2 grid: 511 levels).
constexpr uint32_t kCtaMaxNodes = 1u << 17;
constexpr uint32_t kCtaMaxEdges = 1u << 19;

template <int BLOCK>
const void *bfs_kernel_tile(uint32_t tile)
{
    switch (tile) {
    case 64: return (const void *)dev::bfs_persistent<BLOCK, 64>;
    case 128: return (const void *)dev::bfs_persistent<BLOCK, 128>;
    case 256: return (const void *)dev::bfs_persistent<BLOCK, 256>;
    }
    return nullptr;
}

// Grid-wide BFS kernel for a CTA size and queue tile (0: the default tile);
// NULL for a combination that is not built.
const void *bfs_kernel_for(int block, uint32_t tile)
{
    if (!tile) tile = dev::kBfsGridQueueBuf;
    switch (block) {
    case 256: return bfs_kernel_tile<256>(tile);
    case 512: return bfs_kernel_tile<512>(tile);
    case 1024: return bfs_kernel_tile<1024>(tile);
    }
    return nullptr;
}

template <int BLOCK>
const void *sssp_kernel_tile(uint32_t tile)
{
    switch (tile) {
    case 64: return (const void *)dev::sssp_persistent<BLOCK, 64>;
    case 128: return (const void *)dev::sssp_persistent<BLOCK, 128>;
    case 256:
        if constexpr (BLOCK <= 512) return (const void *)dev::sssp_persistent<BLOCK, 256>;
        break;
    }
    return nullptr;
}

// Grid-wide SSSP kernel for a CTA size and queue tile (0: the default tile,
// dev::kSsspGridQueueBuf); 1024-thread CTAs take tiles of at most 128.
const void *sssp_kernel_for(int block, uint32_t tile)
{
    switch (block) {
    case 256: return sssp_kernel_tile<256>(tile ? tile : dev::kSsspGridQueueBuf<256>);
    case 512: return sssp_kernel_tile<512>(tile ? tile : dev::kSsspGridQueueBuf<512>);
    case 1024: return sssp_kernel_tile<1024>(tile ? tile : dev::kSsspGridQueueBuf<1024>);
    }
    return nullptr;
}

struct Tune {
    uint32_t block, bps, hub, timeout_ms;
    int skip;
    uint32_t max_blocks;
    uint32_t direction;
    uint32_t cta_small;
    uint32_t fuse;
    uint32_t tile;         // push-buffer entries per warp of the grid kernels (0 = default)
    uint32_t warp_degree;  // degree from which a warp expands a vertex by itself
};

Tune resolve_tuning(const gft_tuning *t, bool is_sssp)
{
    Tune r{is_sssp ? kDefaultBlockSssp : kDefaultBlockBfs, kDefaultBlocksPerSm, kDefaultHubDegree, kDefaultTimeoutMs,
           -1, 0, 0, 0, 0, 0, dev::kDefaultWarpDegree};
    if (t) {
        if (t->block_threads) r.block = t->block_threads;
        if (t->blocks_per_sm) r.bps = t->blocks_per_sm;
        if (t->hub_degree) r.hub = t->hub_degree;
        if (t->timeout_ms) r.timeout_ms = t->timeout_ms;
        r.skip = t->test_skip_block;
        r.max_blocks = t->max_blocks;
        r.direction = t->direction;
        r.cta_small = t->cta_small;
        r.fuse = t->fuse_budget;
        r.tile = t->queue_tile;
        if (t->warp_degree) r.warp_degree = t->warp_degree;
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
    // Graphs the engine owns get the interleaved edge pairs; a wrapped graph
    // (the caller's arrays, adopted without a copy) keeps that promise and
    // is read from the separate arrays.
    if (is_sssp && G.edge_data && !G.edge_dw && !G.wrapped)
        GFT_TRY(ensure_edge_pairs(const_cast<gft_graph *>(g), stream));
    Tune t = resolve_tuning(tune, is_sssp);
    const void *kern = is_sssp ? sssp_kernel_for(t.block, t.tile) : bfs_kernel_for(t.block, t.tile);
    if (!kern)
        return fail(GFT_ERR_INVALID_ARG,
                    "%s: block_threads must be 256, 512 or 1024 and queue_tile 0, 64, 128 or 256 "
                    "(SSSP at 1024 threads: at most 128)",
                    what);
    if (t.hub < 32) t.hub = 32;
    DeviceScope device_scope(e->device);
    GFT_CUDA_TRY(device_scope.err);
    // One CTA for small graphs (max_blocks 0 = automatic) or on request
    // (max_blocks 1); the whole cooperative grid otherwise.
    const bool single = t.max_blocks == 1 || (t.max_blocks == 0 && t.skip < 0 && G.nnodes <= kCtaMaxNodes &&
                                              G.nedges <= kCtaMaxEdges);
    LaunchShape shape;
    size_t dyn_smem = 0;
    if (single) {
        shape.block_threads = dev::kCtaBlock;
        shape.blocks = 1;
        shape.blocks_per_sm = 1;
        shape.sms = e->sms;
        if (is_sssp) {
            kern = (const void *)dev::sssp_single_cta;
        } else if (G.nnodes <= dev::kCtaLocalBitsNodes && G.max_degree <= kUniformDegree) {
            // Thread per frontier vertex, bitmap and queue heads in shared memory.
            // A level costs about the instructions its warps issue, and the
            // idle ones issue too: size the CTA to the frontiers, which on
            // these graphs stay near the square root of the vertex count.
            const int lanes_block = dev::lanes_block_for(G.nnodes);
            shape.block_threads = lanes_block;
            kern = dev::lanes_kernel_for(lanes_block, d_parent != nullptr);
            dyn_smem = dev::kLaneSmemBytes;
            if (!G.wrapped) GFT_TRY(ensure_bfs_slots(const_cast<gft_graph *>(g), stream));
            GFT_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem));
        } else {
            kern = G.nnodes <= dev::kCtaLocalBitsNodes ? (const void *)dev::bfs_single_cta<true>
                                                       : (const void *)dev::bfs_single_cta<false>;
        }
    } else {
        GFT_TRY(resolve_shape(e, kern, (int)t.block, (int)t.bps, 0, &shape));
        if (t.max_blocks && (uint32_t)shape.blocks > t.max_blocks) shape.blocks = (int)t.max_blocks;
    }

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
    size_t o_vis = 0, o_f0 = 0, o_f1 = 0, o_qs = 0;
    if (is_sssp) {
        // Distances are computed in place in d_out; per vertex the engine
        // keeps only a pile stamp.
        o_f0 = take((size_t)qcap * 4);
        o_f1 = take((size_t)qcap * 4);
        o_qs = take((size_t)n * 4);
    } else {
        o_vis = take((size_t)((n + 31) / 32) * 4);
    }
    GFT_TRY(e->scratch.ensure(off));
    char *base = reinterpret_cast<char *>(e->scratch.ptr);

    dev::TravParams p{};
    p.row_start = G.row_start;
    p.edge_dst = G.edge_dst;
    p.edge_data = G.edge_data;
    p.edge_dw = is_sssp ? G.edge_dw : nullptr;
    p.bfs_slots = dev::is_lanes_kernel(kern) ? G.bfs_slots : nullptr;
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
        p.qstamp = reinterpret_cast<uint32_t *>(base + o_qs);
    } else {
        p.visited = reinterpret_cast<uint32_t *>(base + o_vis);
    }
    p.hub_cap = hub_cap;
    p.hub_degree = t.hub;
    p.warp_degree = t.warp_degree;
    p.qcap = qcap;
    p.delta = (uint32_t)delta;
    p.ctl = reinterpret_cast<TraversalCtl *>(e->ctl.ptr);
    p.timeout_ns = (unsigned long long)t.timeout_ms * 1000000ull;
    p.skip_block = t.skip;
    p.vec_ok = ((uintptr_t)G.edge_dst % 16 == 0) && (!G.edge_data || (uintptr_t)G.edge_data % 16 == 0);
    p.nedges = G.nedges;
    p.dir_opt = !is_sssp && G.symmetric && t.direction == 0;
    p.uniform = G.max_degree <= kUniformDegree;
    if (is_sssp && !single)
        p.cta_small = t.cta_small == UINT32_MAX ? 0 : t.cta_small ? t.cta_small : p.uniform ? kDefaultCtaSmall : 0;
    if (is_sssp) p.fuse = t.fuse == UINT32_MAX ? 0 : t.fuse ? t.fuse : p.uniform ? kDefaultFuse : 0;

    GFT_CUDA_TRY(cudaMemsetAsync(e->ctl.ptr, 0, sizeof(TraversalCtl), stream));
    void *args[] = {&p};
    GFT_CUDA_TRY(cudaEventRecord(e->ev0, stream));
    if (single)
        GFT_CUDA_TRY(cudaLaunchKernel(kern, dim3(1), dim3(shape.block_threads), args, dyn_smem, stream));
    else
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
    DeviceScope device_scope(g->g.device);
    GFT_CUDA_TRY(device_scope.err);
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

// k queries on one graph with results to the host: query i writes device
// buffer i % 2, and its copy to row i runs on the engine's copy stream while
// query i + 1 runs on `stream`.  Query i + 2 waits for copy i before it
// reuses the buffer.
static gft_status run_host_many(bool is_sssp, gft_engine *e, const gft_graph *g, const uint32_t *sources, uint32_t k,
                                int32_t delta, int32_t *h_out, const gft_tuning *tune, void *stream_, gft_stats *stats)
{
    const char *what = is_sssp ? "gft_sssp_host_many" : "gft_bfs_host_many";
    if (!e) return fail(GFT_ERR_INVALID_ARG, "%s: engine is NULL", what);
    if (k && (!sources || !h_out)) return fail(GFT_ERR_INVALID_ARG, "%s: sources or output pointer is NULL", what);
    std::lock_guard<std::mutex> lk(e->mu);
    GFT_TRY(check_engine_graph(e, g));
    const size_t n = g->g.nnodes;
    for (uint32_t i = 0; i < k; i++)
        if (sources[i] >= n)
            return fail(GFT_ERR_INVALID_ARG, "%s: source %u (query %u) out of range (nnodes %zu)", what, sources[i], i,
                        n);
    if (is_sssp && delta <= 0) return fail(GFT_ERR_INVALID_ARG, "%s: delta must be > 0 (got %d)", what, delta);
    if (k == 0) return GFT_OK;
    cudaStream_t stream = (cudaStream_t)stream_;
    DeviceScope device_scope(e->device);
    GFT_CUDA_TRY(device_scope.err);
    if (!e->copy_stream) GFT_CUDA_TRY(cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking));
    for (int b = 0; b < 2; b++) {
        if (!e->result_ready[b]) GFT_CUDA_TRY(cudaEventCreateWithFlags(&e->result_ready[b], cudaEventDisableTiming));
        if (!e->copy_done[b]) GFT_CUDA_TRY(cudaEventCreateWithFlags(&e->copy_done[b], cudaEventDisableTiming));
    }
    const size_t row = align256(n * 4);
    GFT_TRY(e->aux.ensure(2 * row));
    char *base = reinterpret_cast<char *>(e->aux.ptr);
    gft_status st = GFT_OK;
    cudaError_t ce = cudaSuccess;
    for (uint32_t i = 0; i < k && st == GFT_OK && ce == cudaSuccess; i++) {
        const int b = i & 1;
        int32_t *d_out = reinterpret_cast<int32_t *>(base + b * row);
        if (i >= 2) ce = cudaStreamWaitEvent(stream, e->copy_done[b], 0);
        if (ce != cudaSuccess) break;
        st = run_traversal(is_sssp, e, g, sources[i], delta, d_out, nullptr, tune, stream, stats ? stats + i : nullptr);
        if (st != GFT_OK) break;
        ce = cudaEventRecord(e->result_ready[b], stream);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->copy_stream, e->result_ready[b], 0);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(h_out + (size_t)i * n, d_out, n * 4, cudaMemcpyDeviceToHost, e->copy_stream);
        if (ce == cudaSuccess) ce = cudaEventRecord(e->copy_done[b], e->copy_stream);
    }
    // No copy into the caller's rows stays in flight after the call.
    const cudaError_t se = cudaStreamSynchronize(e->copy_stream);
    if (st != GFT_OK) return st;
    GFT_CUDA_TRY(ce);
    GFT_CUDA_TRY(se);
    return GFT_OK;
}

gft_status gft_bfs_host_many(gft_engine *e, const gft_graph *g, const uint32_t *sources, uint32_t k, int32_t *h_out,
                             const gft_tuning *tune, void *stream, gft_stats *stats)
{
    return run_host_many(false, e, g, sources, k, 0, h_out, tune, stream, stats);
}

gft_status gft_sssp_host_many(gft_engine *e, const gft_graph *g, const uint32_t *sources, uint32_t k, int32_t delta,
                              int32_t *h_out, const gft_tuning *tune, void *stream, gft_stats *stats)
{
    return run_host_many(true, e, g, sources, k, delta, h_out, tune, stream, stats);
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
    DeviceScope device_scope(G.device);
    GFT_CUDA_TRY(device_scope.err);
    char *base = nullptr;
    GFT_TRY(noalloc_scratch(G.device, &base));

    const void *kern = (const void *)dev::bfs_persistent<kNoAllocBlock, dev::kBfsGridQueueBuf>;
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
    // The same schedule choices as gft_bfs: static chunks on uniform-degree
    // graphs, bottom-up levels on a graph marked symmetric (they use only the
    // bitmap and queues above).
    p.nedges = G.nedges;
    p.uniform = G.max_degree <= kUniformDegree;
    p.dir_opt = G.symmetric && !(tune && tune->direction != 0);

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

#ifdef GFT_TRACE
extern "C" GFT_API int gft_debug_trace(unsigned long long *host, int max_records)
{
    const int n = max_records < 8192 ? max_records : 8192;
    return cudaMemcpyFromSymbol(host, gft::dev::g_trace, sizeof(unsigned long long) * 2 * n) == cudaSuccess ? n : -1;
}
#endif
