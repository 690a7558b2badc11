// mis.cu -- maximal independent set (gft_mis): the reference's apps/mis on
// the engine's frontier core.
//
// The reference (apps/mis/kernel.cu) gives every vertex a priority from one
// xorshift128 stream per thread of its launch grid (gen_prio_gpu, :18-41:
// thread t starts from (SEED1..SEED4) ^ t and gives its k-th output to
// vertex t + k * nthreads) and then runs rounds over a worklist that starts
// with every vertex (:151-169):
//   mark   a worklist vertex is MARKED when no out-neighbour other than
//          itself that is not NON_INDEPENDENT beats it in (priority, id)
//          order: larger unsigned priority, then larger id (:65-103);
//   drop   a worklist vertex that is MARKED, or has a MARKED out-neighbour,
//          leaves the worklist, and an unmarked one becomes NON_INDEPENDENT
//          (:104-149).
// A vertex marked during a mark pass is still not NON_INDEPENDENT and a
// vertex excluded during a drop pass is still not MARKED, so no decision
// depends on the schedule: the set is a function of the priorities.
//
// Here one persistent cooperative launch runs every round (two grid
// barriers per round), or one CTA for a small graph.  Each vertex has one
// 64-bit word, priority << 32 | state, so testing a neighbour is one 8-byte
// load that answers both passes' questions.  Worklist vertices go one per
// lane; a lane scans a list of fewer than 32 edges alone and stops at the
// first deciding neighbour, and the whole warp scans a longer one 32 edges
// at a time.  Survivors are appended with the warp-aggregated queue.
#include <string.h>

#include <algorithm>

#include "frontier.cuh"
#include "gft_internal.h"

namespace gft {
namespace dev {

constexpr uint32_t kMisUnmarked = 0;  // apps/mis/kernel.cu:9-11
constexpr uint32_t kMisMarked = 1;
constexpr uint32_t kMisExcluded = 2;  // NON_INDEPENDENT
// SEED1..SEED4, apps/mis/kernel.cu:13-16.
constexpr uint32_t kMisSeed1 = 0x12345678u, kMisSeed2 = 0xabbdef12u, kMisSeed3 = 0xcafe1234u,
                   kMisSeed4 = 0x09832516u;
constexpr int kMisBlock = 1024;

struct MisParams {
    TravParams t;              // graph, queues, control block
    unsigned long long *word;  // per vertex: priority << 32 | state
    int32_t *out;              // per vertex state, as the reference's node_data
    uint32_t prio_threads;     // priority streams (the reference's launch size)
};

__device__ __forceinline__ uint32_t mis_state(unsigned long long w) { return (uint32_t)w; }
__device__ __forceinline__ uint32_t mis_prio(unsigned long long w) { return (uint32_t)(w >> 32); }
__device__ __forceinline__ void mis_set_state(unsigned long long *word, uint32_t v, uint32_t s)
{
    __stcg(reinterpret_cast<uint32_t *>(word + v), s);  // the low half of the little-endian word
}

// Does neighbour d decide vertex u?  Mark pass: d beats u.  Drop pass: d is
// MARKED.
template <bool MARK>
__device__ __forceinline__ bool mis_decides(uint32_t u, uint32_t pu, uint32_t d, unsigned long long wd)
{
    if (MARK)
        return d != u && mis_state(wd) != kMisExcluded &&
               (mis_prio(wd) > pu || (mis_prio(wd) == pu && d > u));
    return mis_state(wd) == kMisMarked;
}

// One pass over the worklist `in[0, n)`.  Mark: undecided (unbeaten)
// vertices become MARKED.  Drop: MARKED vertices and those with a MARKED
// neighbour leave (unmarked ones become NON_INDEPENDENT); the rest are
// appended to q.
template <bool MARK, class Mode>
__device__ __forceinline__ void mis_pass(const MisParams &mp, Mode &m, const uint32_t *in, uint32_t n,
                                         unsigned *claim, WarpQueue &q, unsigned long long &scanned)
{
    const TravParams &p = mp.t;
    const unsigned lane = threadIdx.x & 31;
    const unsigned grain = pick_grain(n, m.nwarps, p.uniform);
    const ChunkSched cs{(n + grain - 1) / grain, m.nwarps, m.gwarp, lane, claim};
    for (unsigned c = cs.first(); c < cs.nchunks; c = cs.next()) {
        const unsigned base = c * grain;
        const unsigned end = min(n, base + grain);
        for (unsigned i0 = base; i0 < end; i0 += 32) {
            const unsigned idx = i0 + lane;
            const bool has = idx < end;
            uint32_t u = 0, start = 0, deg = 0, pu = 0;
            bool decided = false, live = has;
            if (has) {
                u = __ldcg(in + idx);
                const unsigned long long wu = __ldcg(mp.word + u);
                pu = mis_prio(wu);
                if (!MARK && mis_state(wu) == kMisMarked) {
                    live = false;  // leaves the worklist, stays in the set
                } else {
                    start = __ldg(p.row_start + u);
                    deg = __ldg(p.row_start + u + 1) - start;
                }
            }
            // Lists of >= 32 edges: the whole warp, 32 edges a step, stops
            // at the first deciding neighbour.
            unsigned heavy = __ballot_sync(kFull, live && deg >= 32);
            while (heavy) {
                const int l = __ffs(heavy) - 1;
                heavy &= heavy - 1;
                const uint32_t hu = __shfl_sync(kFull, u, l), hs = __shfl_sync(kFull, start, l);
                const uint32_t hd = __shfl_sync(kFull, deg, l), hp = __shfl_sync(kFull, pu, l);
                bool found = false;
                for (uint32_t e0 = 0; e0 < hd && !found; e0 += 32) {
                    bool mine = false;
                    if (e0 + lane < hd) {
                        const uint32_t d = __ldcs(p.edge_dst + hs + e0 + lane);
                        mine = mis_decides<MARK>(hu, hp, d, __ldcg(mp.word + d));
                        scanned++;
                    }
                    found = __any_sync(kFull, mine);
                }
                if (lane == l) decided = found;
            }
            if (live && deg < 32) {
                for (uint32_t e = start; e < start + deg && !decided; e++) {
                    const uint32_t d = __ldcs(p.edge_dst + e);
                    decided = mis_decides<MARK>(u, pu, d, __ldcg(mp.word + d));
                    scanned++;
                }
            }
            if (MARK) {
                if (live && !decided) mis_set_state(mp.word, u, kMisMarked);
            } else {
                if (live && decided) mis_set_state(mp.word, u, kMisExcluded);
                q.push(live && !decided, u, lane);
            }
        }
    }
    if (!MARK) q.flush(lane);
}

template <class Mode>
__device__ __forceinline__ void mis_body(const MisParams &mp, Mode &m, uint32_t *warp_buf)
{
    const TravParams &p = mp.t;
    TraversalCtl *ctl = m.ctl;
    const unsigned lane = threadIdx.x & 31;
    const unsigned tid = m.tid, nthreads = m.nthreads;
    const uint32_t n = p.nnodes;

    // Priorities (apps/mis/kernel.cu:18-41), state UNMARKED, and a worklist
    // of every vertex (init_wl, :49-63).
    const uint32_t streams = min(mp.prio_threads, n);
    for (uint32_t s = tid; s < streams; s += nthreads) {
        uint32_t x = kMisSeed1 ^ s, y = kMisSeed2 ^ s, z = kMisSeed3 ^ s, w = kMisSeed4 ^ s;
        for (uint64_t v = s; v < n; v += mp.prio_threads) {
            // Marsaglia's xorshift128 ("Xorshift RNGs", J. Stat. Softw. 8(14), 2003).
            const uint32_t t = x ^ (x << 11);
            x = y;
            y = z;
            z = w;
            w = w ^ (w >> 19) ^ t ^ (t >> 8);
            mp.word[v] = ((unsigned long long)w << 32) | kMisUnmarked;
        }
    }
    for (uint32_t v = tid; v < n; v += nthreads) p.q[0][v] = v;
    if (tid == 0) *u32_of(ctl->qlen[0]) = n;
    if (!m.sync()) return;

    WarpQueue q;
    q.buf = warp_buf;
    q.count = 0;
    q.cap = p.qcap;
    q.err = &ctl->error;
    q.err_where = &ctl->error_where;
    unsigned long long scanned = 0, pops = 0;  // pops: thread 0's tally of worklist entries
    unsigned L = 0;
    for (;;) {
        const unsigned slot = L % 3, nslot = (L + 1) % 3, rslot = (L + 2) % 3;
        const unsigned n_in = m.ld(u32_of(ctl->qlen[slot]));
        if (n_in == 0) break;
        pops += n_in;
        if (tid == 0) {
            *u32_of(ctl->qlen[rslot]) = 0;
            *u32_of(ctl->claim[rslot]) = 0;
            *u32_of(ctl->hub_claim[rslot]) = 0;
        }
        const uint32_t *in = sel2(p.q, L);
        mis_pass<true>(mp, m, in, n_in, u32_of(ctl->claim[slot]), q, scanned);
        if (!m.sync()) return;
        q.queue = sel2(p.q, L + 1);
        q.len = u32_of(ctl->qlen[nslot]);
        mis_pass<false>(mp, m, in, n_in, u32_of(ctl->hub_claim[slot]), q, scanned);
        if (!m.sync()) return;
        L++;
    }
    // node_data for the caller, and the set's size.
    unsigned long long members = 0;
    for (uint32_t v = tid; v < n; v += nthreads) {
        const uint32_t s = mis_state(__ldcg(mp.word + v));
        mp.out[v] = (int32_t)s;
        members += s == kMisMarked;
    }
    warp_add_u64(&ctl->edges, scanned, lane);
    warp_add_u64(&ctl->reached, members, lane);
    if (tid == 0) {
        ctl->levels = L;
        ctl->iterations = m.epoch();
        ctl->pushes = pops;
    }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 2048 / BLOCK) mis_persistent(MisParams mp)
{
    __shared__ uint32_t s_buf[BLOCK / 32][kQueueBuf];
    TraversalCtl *ctl = mp.t.ctl;
    const unsigned tid = blockIdx.x * BLOCK + threadIdx.x, nthreads = gridDim.x * BLOCK;
    GridMode m{{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, gridDim.x, 0,
                mp.t.timeout_ns},
               ctl, tid, nthreads, tid / 32, nthreads / 32};
    mis_body(mp, m, s_buf[threadIdx.x >> 5]);
}

// Small graphs: one CTA, control block in shared memory, __syncthreads as
// the barrier; the counters are copied to the engine's control block.
__global__ void __launch_bounds__(kMisBlock, 1) mis_single_cta(MisParams mp)
{
    __shared__ TraversalCtl s_ctl;
    __shared__ uint32_t s_buf[kMisBlock / 32][kQueueBuf];
    for (unsigned i = threadIdx.x; i < sizeof(TraversalCtl) / 4; i += kMisBlock)
        reinterpret_cast<unsigned *>(&s_ctl)[i] = 0;
    __syncthreads();
    TraversalCtl *gctl = mp.t.ctl;
    mp.t.ctl = &s_ctl;
    CtaMode m{&s_ctl, threadIdx.x, kMisBlock, threadIdx.x >> 5, kMisBlock / 32, 0};
    mis_body(mp, m, s_buf[threadIdx.x >> 5]);
    __syncthreads();
    if (threadIdx.x == 0) {
        gctl->error = s_ctl.error;
        gctl->error_where = s_ctl.error_where;
        gctl->levels = s_ctl.levels;
        gctl->iterations = s_ctl.iterations;
        gctl->edges = s_ctl.edges;
        gctl->reached = s_ctl.reached;
        gctl->pushes = s_ctl.pushes;
    }
}

}  // namespace dev
}  // namespace gft

namespace gft {
namespace {

// Graphs up to this size run on one CTA by default (as the single-query
// traversals do): their rounds are many and small.
constexpr uint32_t kMisCtaMaxNodes = 1u << 17;
constexpr uint32_t kMisCtaMaxEdges = 1u << 19;

const void *mis_kernel_for(int block)
{
    switch (block) {
    case 256: return (const void *)dev::mis_persistent<256>;
    case 512: return (const void *)dev::mis_persistent<512>;
    case 1024: return (const void *)dev::mis_persistent<1024>;
    }
    return nullptr;
}

gft_status run_mis(gft_engine *e, const gft_graph *g, int32_t *d_state, uint32_t prio_threads,
                   const gft_tuning *tune, cudaStream_t stream, gft_stats *stats)
{
    GFT_TRY(check_engine_graph(e, g));
    if (!d_state) return fail(GFT_ERR_INVALID_ARG, "gft_mis: state pointer is NULL");
    const DeviceGraph &G = g->g;
    const int block = (tune && tune->block_threads) ? (int)tune->block_threads : 1024;
    const int bps = (tune && tune->blocks_per_sm) ? (int)tune->blocks_per_sm : 2;
    const uint32_t max_blocks = tune ? tune->max_blocks : 0;
    DeviceScope device_scope(e->device);
    GFT_CUDA_TRY(device_scope.err);
    // The reference's priority grid: kernel_sizing's 8 CTAs of 256 threads
    // per SM (skelapp/skel.cu:37-43, apps/mis/kernel.cu:225).
    if (prio_threads == 0) prio_threads = 8u * (uint32_t)e->sms * 256u;
    const uint32_t n = G.nnodes;
    const bool single = max_blocks == 1 || (max_blocks == 0 && n <= kMisCtaMaxNodes && G.nedges <= kMisCtaMaxEdges);
    LaunchShape shape;
    const void *kern;
    if (single) {
        kern = (const void *)dev::mis_single_cta;
        shape.block_threads = dev::kMisBlock;
        shape.blocks = 1;
        shape.blocks_per_sm = 1;
        shape.sms = e->sms;
    } else {
        kern = mis_kernel_for(block);
        if (!kern) return fail(GFT_ERR_INVALID_ARG, "gft_mis: block_threads must be 256, 512 or 1024");
        GFT_TRY(resolve_shape(e, kern, block, bps, 0, &shape));
        if (max_blocks && (uint32_t)shape.blocks > max_blocks) shape.blocks = (int)max_blocks;
    }
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (std::max<size_t>(bytes, 8) + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_q0 = take((size_t)n * 4), o_q1 = take((size_t)n * 4), o_word = take((size_t)n * 8);
    GFT_TRY(e->scratch.ensure(off));
    char *base = static_cast<char *>(e->scratch.ptr);
    dev::MisParams mp{};
    dev::TravParams &p = mp.t;
    p.row_start = G.row_start;
    p.edge_dst = G.edge_dst;
    p.nnodes = n;
    p.q[0] = reinterpret_cast<uint32_t *>(base + o_q0);
    p.q[1] = reinterpret_cast<uint32_t *>(base + o_q1);
    p.qcap = n;
    p.ctl = reinterpret_cast<TraversalCtl *>(e->ctl.ptr);
    p.timeout_ns = (unsigned long long)((tune && tune->timeout_ms) ? tune->timeout_ms : 20000) * 1000000ull;
    p.skip_block = -1;
    p.nedges = G.nedges;
    p.uniform = G.max_degree <= kUniformDegree;
    mp.word = reinterpret_cast<unsigned long long *>(base + o_word);
    mp.out = d_state;
    mp.prio_threads = prio_threads;
    GFT_CUDA_TRY(cudaMemsetAsync(e->ctl.ptr, 0, sizeof(TraversalCtl), stream));
    void *args[] = {&mp};
    GFT_CUDA_TRY(cudaEventRecord(e->ev0, stream));
    if (single)
        GFT_CUDA_TRY(cudaLaunchKernel(kern, dim3(1), dim3(shape.block_threads), args, 0, stream));
    else
        GFT_CUDA_TRY(
            cudaLaunchCooperativeKernel(kern, dim3(shape.blocks), dim3(shape.block_threads), args, 0, stream));
    GFT_CUDA_TRY(cudaEventRecord(e->ev1, stream));
    TraversalCtl *h = reinterpret_cast<TraversalCtl *>(e->host_ctl);
    const size_t cold = offsetof(TraversalCtl, error);
    GFT_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char *>(h) + cold, reinterpret_cast<char *>(e->ctl.ptr) + cold,
                                 sizeof(TraversalCtl) - cold, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h->error)
        return fail((gft_status)h->error, "gft_mis: device reported %s (site %u)",
                    gft_status_string((gft_status)h->error), h->error_where);
    if (stats) {
        memset(stats, 0, sizeof *stats);
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev0, e->ev1);
        stats->levels = h->levels;
        stats->iterations = h->iterations;
        stats->vertices_reached = h->reached;
        stats->edges_scanned = h->edges;
        stats->pushes = h->pushes;
        stats->kernel_ms = ms;
        stats->grid_blocks = shape.blocks;
        stats->block_threads = shape.block_threads;
    }
    return GFT_OK;
}

}  // namespace
}  // namespace gft

using namespace gft;

extern "C" {

gft_status gft_mis(gft_engine *e, const gft_graph *g, int32_t *d_state, uint32_t prio_threads,
                   const gft_tuning *tune, void *stream, gft_stats *stats)
{
    if (!e) return fail(GFT_ERR_INVALID_ARG, "gft_mis: engine is NULL");
    std::lock_guard<std::mutex> lk(e->mu);
    return run_mis(e, g, d_state, prio_threads, tune, (cudaStream_t)stream, stats);
}

gft_status gft_mis_host(gft_engine *e, const gft_graph *g, int32_t *h_state, uint32_t prio_threads,
                        const gft_tuning *tune, void *stream_, gft_stats *stats)
{
    if (!e) return fail(GFT_ERR_INVALID_ARG, "gft_mis_host: engine is NULL");
    if (!h_state) return fail(GFT_ERR_INVALID_ARG, "gft_mis_host: output pointer is NULL");
    std::lock_guard<std::mutex> lk(e->mu);
    GFT_TRY(check_engine_graph(e, g));
    DeviceScope device_scope(g->g.device);
    GFT_CUDA_TRY(device_scope.err);
    cudaStream_t stream = (cudaStream_t)stream_;
    const size_t n = g->g.nnodes;
    GFT_TRY(e->aux.ensure(std::max<size_t>(n * 4, 256)));
    int32_t *d_state = reinterpret_cast<int32_t *>(e->aux.ptr);
    GFT_TRY(run_mis(e, g, d_state, prio_threads, tune, stream, stats));
    GFT_CUDA_TRY(cudaMemcpyAsync(h_state, d_state, n * 4, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    return GFT_OK;
}

}  // extern "C"
