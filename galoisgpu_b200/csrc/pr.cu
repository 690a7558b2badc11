// pr.cu -- PageRank by residual push (gft_pr): the reference's apps/pr on
// the engine's frontier core.
//
// The reference (apps/pr/kernel.cu) keeps a rank and a residual per vertex:
//   init   rank = 1 - ALPHA; every vertex adds (float)(1.0 / outdeg) to its
//          neighbours' residuals (init_1, :26-47); each residual is scaled
//          by (1 - ALPHA) * ALPHA in double precision (init_2, :49-63); every
//          vertex is on the first worklist;
//   step   a worklist vertex takes its residual r (atomicExch to 0), adds it
//          to its rank, and adds r * ALPHA / outdeg to each neighbour's
//          residual; a neighbour whose residual crosses EPSILON from below
//          joins the next worklist (pagerank_main, :127-236);
// until the worklist is empty (:271-305).  Here the same steps run in one
// persistent cooperative launch on the frontier machinery of frontier.cuh:
// the per-vertex expansion tiers (flattened, warp, grid-wide hubs), the
// warp-aggregated queue, and the bounded grid barrier.
//
// One rule differs, for the hardware: the worklist of the next round is every
// vertex whose residual exceeds EPSILON when the round ends, collected by a
// sweep of the residuals after the round's barrier, instead of the vertices
// whose residual crossed EPSILON during a push.  A push then needs no return
// value, so it is a fire-and-forget float reduction in L2 instead of an
// atomic whose result the warp waits for (the crossing test).  Each vertex
// is listed once, so it has one popper per round and its rank needs no
// atomic.  Two consequences: a residual that rounds to exactly EPSILON, which
// the reference's crossing test never queues again (its later residual never
// reaches its rank), is picked up once it grows; and at the end every
// residual is at most EPSILON.  Float addition in schedule order makes the
// last bits of the ranks run-dependent, as in the reference.
#include <string.h>

#include <algorithm>

#include "frontier.cuh"
#include "gft_internal.h"

namespace gft {
namespace dev {

constexpr float kPrAlpha = 0.85f;       // apps/pr/kernel.cu:19
constexpr float kPrEpsilon = 0.000001f;  // apps/pr/kernel.cu:20

// Float add to global memory with no return value (a reduction performed in
// L2): the issuing warp does not wait for it.
__device__ __forceinline__ void red_add_f32(float *p, float v)
{
    asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

struct PrOwn {
    uint32_t u;
    float upd;  // what each of u's edges adds to its destination's residual
};

// Init: every vertex adds (float)(1.0 / outdeg) along its edges.
struct PrInitVisitor {
    static constexpr int kBatch = 2;
    static constexpr bool kEarlyRow = false;  // owner() reads only the degree
    const uint32_t *__restrict__ row_start;
    const uint32_t *__restrict__ edge_dst;
    float *residual;
    WarpQueue q;  // unused: init pushes nothing
    unsigned long long edges;
    bool vec;

    __device__ __forceinline__ PrOwn owner(bool has, uint32_t u) const
    {
        if (!has) return PrOwn{u, 0.f};
        const uint32_t deg = __ldg(row_start + u + 1) - __ldg(row_start + u);
        return PrOwn{u, deg ? (float)(1.0 / deg) : 0.f};
    }
    __device__ __forceinline__ bool active(const PrOwn &o) const { return o.upd != 0.f; }
    __device__ __forceinline__ PrOwn shfl(const PrOwn &o, int lane) const
    {
        return PrOwn{__shfl_sync(kFull, o.u, lane), __shfl_sync(kFull, o.upd, lane)};
    }
    template <int K>
    __device__ __forceinline__ void addK(const bool (&valid)[K], const uint32_t (&d)[K], const PrOwn (&o)[K])
    {
#pragma unroll
        for (int k = 0; k < K; k++)
            if (valid[k]) {
                red_add_f32(residual + d[k], o[k].upd);
                edges++;
            }
    }
    template <int K>
    __device__ __forceinline__ void edgeK(const bool (&valid)[K], const uint32_t (&e)[K], const PrOwn (&o)[K],
                                          unsigned lane)
    {
        uint32_t d[K];
#pragma unroll
        for (int k = 0; k < K; k++) d[k] = valid[k] ? __ldcs(edge_dst + e[k]) : 0u;
        addK<K>(valid, d, o);
    }
    __device__ __forceinline__ void edge1(bool valid, uint32_t e, const PrOwn &o, unsigned lane)
    {
        const bool v[1] = {valid};
        const uint32_t ee[1] = {e};
        const PrOwn oo[1] = {o};
        edgeK<1>(v, ee, oo, lane);
    }
    __device__ __forceinline__ void edge4(bool valid, uint32_t e, const PrOwn &o, unsigned lane)
    {
        const uint4 x = valid ? __ldcs(reinterpret_cast<const uint4 *>(edge_dst + e)) : make_uint4(0, 0, 0, 0);
        const bool v[4] = {valid, valid, valid, valid};
        const uint32_t d[4] = {x.x, x.y, x.z, x.w};
        const PrOwn oo[4] = {o, o, o, o};
        addK<4>(v, d, oo);
    }
};

// One push step.  owner() pops the vertex (its only side effect), except in
// the hub phase, where the hub's update was stored when it was popped.  A
// push is a float add whose result is not used (a fire-and-forget reduction
// in L2): the next worklist is built after the round from the residuals
// themselves, so no push waits for the residual it changed.
struct PrVisitor {
    static constexpr int kBatch = 4;
    static constexpr bool kEarlyRow = true;  // owner() pops the residual
    const uint32_t *__restrict__ row_start;
    const uint32_t *__restrict__ edge_dst;
    float *rank, *residual, *hub_upd;
    uint32_t hub_degree;
    bool hub_phase;
    unsigned long long edges;
    bool vec;

    __device__ __forceinline__ PrOwn owner(bool has, uint32_t u)
    {
        if (!has) return PrOwn{u, 0.f};
        if (hub_phase) return PrOwn{u, __ldcg(hub_upd + u)};
        const float r = __uint_as_float(atomicExch(reinterpret_cast<unsigned *>(residual + u), 0u));
        rank[u] += r;  // a worklist lists a vertex once: one popper per round
        const uint32_t deg = __ldg(row_start + u + 1) - __ldg(row_start + u);
        const float upd = deg ? r * kPrAlpha / (float)deg : 0.f;
        if (deg >= hub_degree) hub_upd[u] = upd;
        return PrOwn{u, upd};
    }
    __device__ __forceinline__ bool active(const PrOwn &o) const { return o.upd != 0.f; }
    __device__ __forceinline__ PrOwn shfl(const PrOwn &o, int lane) const
    {
        return PrOwn{__shfl_sync(kFull, o.u, lane), __shfl_sync(kFull, o.upd, lane)};
    }
    template <int K>
    __device__ __forceinline__ void edgeK(const bool (&valid)[K], const uint32_t (&e)[K], const PrOwn (&o)[K],
                                          unsigned lane)
    {
        uint32_t d[K];
#pragma unroll
        for (int k = 0; k < K; k++) d[k] = valid[k] ? __ldcs(edge_dst + e[k]) : 0u;
#pragma unroll
        for (int k = 0; k < K; k++)
            if (valid[k]) {
                red_add_f32(residual + d[k], o[k].upd);
                edges++;
            }
    }
    __device__ __forceinline__ void edge1(bool valid, uint32_t e, const PrOwn &o, unsigned lane)
    {
        const bool v[1] = {valid};
        const uint32_t ee[1] = {e};
        const PrOwn oo[1] = {o};
        edgeK<1>(v, ee, oo, lane);
    }
    __device__ __forceinline__ void edge4(bool valid, uint32_t e, const PrOwn &o, unsigned lane)
    {
        const uint4 x = valid ? __ldcs(reinterpret_cast<const uint4 *>(edge_dst + e)) : make_uint4(0, 0, 0, 0);
        if (valid) {
            red_add_f32(residual + x.x, o.upd);
            red_add_f32(residual + x.y, o.upd);
            red_add_f32(residual + x.z, o.upd);
            red_add_f32(residual + x.w, o.upd);
            edges += 4;
        }
    }
};

struct PrParams {
    TravParams t;  // graph, queues, hubs, control block (expansion machinery)
    float *rank, *residual, *hub_upd;
    uint32_t max_iterations;
};

// Appends every vertex whose residual exceeds EPSILON to the next worklist
// (each vertex once, so a worklist never lists a vertex twice).  Runs between
// two grid barriers, when no push is in flight.
__device__ __forceinline__ void pr_collect(const float *residual, uint32_t n, WarpQueue &q, unsigned gwarp,
                                           unsigned nwarps, unsigned lane)
{
    for (uint32_t base = gwarp * 32u; base < n; base += nwarps * 32u) {
        const uint32_t v = base + lane;
        const bool has = v < n;
        const float r = has ? __ldcg(residual + v) : 0.f;
        q.push(has && r > kPrEpsilon, v, lane);
    }
    q.flush(lane);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 2048 / BLOCK) pr_persistent(PrParams pp)
{
    __shared__ uint32_t s_buf[BLOCK / 32][kQueueBuf];
    const TravParams &p = pp.t;
    TraversalCtl *ctl = p.ctl;
    const unsigned lane = threadIdx.x & 31;
    const unsigned tid = blockIdx.x * BLOCK + threadIdx.x, nthreads = gridDim.x * BLOCK;
    const unsigned gwarp = tid / 32, nwarps = nthreads / 32;
    GridMode m{{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, gridDim.x, 0, p.timeout_ns},
               ctl, tid, nthreads, gwarp, nwarps};
    const uint32_t n = p.nnodes;

    // Init (apps/pr/kernel.cu:26-63).
    for (uint32_t v = tid; v < n; v += nthreads) {
        pp.rank[v] = (float)(1.0 - (double)kPrAlpha);
        pp.residual[v] = 0.f;
        p.q[0][v] = v;
    }
    if (tid == 0) *u32_of(ctl->qlen[0]) = n;
    if (!m.sync()) return;
    {
        PrInitVisitor iv{p.row_start, p.edge_dst, pp.residual, WarpQueue{}, 0, p.vec_ok != 0};
        expand_frontier<PrInitVisitor, PrOwn>(iv, p, p.q[0], n, u32_of(ctl->claim[0]), &ctl->hub[0].v,
                                              pick_grain(n, nwarps, p.uniform), gwarp, nwarps, lane);
        if (!m.sync()) return;
        const unsigned long long hv = m.ld64(&ctl->hub[0].v);
        if (hv) {
            expand_hubs<PrInitVisitor, PrOwn>(iv, p, (unsigned)(hv >> 32), (unsigned)hv,
                                              u32_of(ctl->hub_claim[0]), gwarp, nwarps, lane);
            if (!m.sync()) return;
        }
    }
    for (uint32_t v = tid; v < n; v += nthreads)
        pp.residual[v] = (float)((double)pp.residual[v] * ((1.0 - (double)kPrAlpha) * (double)kPrAlpha));
    if (tid == 0) {
        ctl->hub[0].v = 0;
        *u32_of(ctl->claim[0]) = 0;
        *u32_of(ctl->hub_claim[0]) = 0;
    }
    if (!m.sync()) return;

    PrVisitor vis;
    vis.row_start = p.row_start;
    vis.edge_dst = p.edge_dst;
    vis.rank = pp.rank;
    vis.residual = pp.residual;
    vis.hub_upd = pp.hub_upd;
    vis.hub_degree = p.hub_degree;
    vis.hub_phase = false;
    vis.edges = 0;
    vis.vec = p.vec_ok != 0;
    WarpQueue q;
    q.buf = s_buf[threadIdx.x >> 5];
    q.count = 0;
    q.cap = p.qcap;
    q.err = &ctl->error;
    q.err_where = &ctl->error_where;

    // Round L: pop and push the worklist Q(L) (its hubs in a grid-wide second
    // phase), then collect Q(L+1) from the residuals.
    unsigned L = 0;
    unsigned long long pops = 0;  // worklist entries processed (thread 0's tally)
    for (;;) {
        const unsigned slot = L % 3, nslot = (L + 1) % 3, rslot = (L + 2) % 3;
        const unsigned n_in = m.ld(u32_of(ctl->qlen[slot]));
        if (n_in == 0 || L >= pp.max_iterations) break;
        pops += n_in;
        if (tid == 0) {
            *u32_of(ctl->qlen[rslot]) = 0;
            *u32_of(ctl->claim[rslot]) = 0;
            ctl->hub[rslot].v = 0;
            *u32_of(ctl->hub_claim[rslot]) = 0;
        }
        vis.hub_phase = false;
        expand_frontier<PrVisitor, PrOwn>(vis, p, sel2(p.q, L), n_in, u32_of(ctl->claim[slot]), &ctl->hub[slot].v,
                                          pick_grain(n_in, nwarps, p.uniform), gwarp, nwarps, lane);
        if (!m.sync()) return;
        const unsigned long long hv = m.ld64(&ctl->hub[slot].v);
        if (hv) {
            vis.hub_phase = true;
            expand_hubs<PrVisitor, PrOwn>(vis, p, (unsigned)(hv >> 32), (unsigned)hv, u32_of(ctl->hub_claim[slot]),
                                          gwarp, nwarps, lane);
            if (!m.sync()) return;
        }
        q.queue = sel2(p.q, (L + 1));
        q.len = u32_of(ctl->qlen[nslot]);
        pr_collect(pp.residual, n, q, gwarp, nwarps, lane);
        if (!m.sync()) return;
        L++;
    }
    warp_add_u64(&ctl->edges, vis.edges, lane);
    if (tid == 0) {
        ctl->levels = L;
        ctl->iterations = m.epoch();
        ctl->pushes = pops;
    }
}

}  // namespace dev
}  // namespace gft

namespace gft {
namespace {

const void *pr_kernel_for(int block)
{
    switch (block) {
    case 256: return (const void *)dev::pr_persistent<256>;
    case 512: return (const void *)dev::pr_persistent<512>;
    case 1024: return (const void *)dev::pr_persistent<1024>;
    }
    return nullptr;
}

gft_status run_pr(gft_engine *e, const gft_graph *g, float *d_rank, uint32_t max_iterations, const gft_tuning *tune,
                  cudaStream_t stream, gft_stats *stats)
{
    GFT_TRY(check_engine_graph(e, g));
    if (!d_rank) return fail(GFT_ERR_INVALID_ARG, "gft_pr: rank pointer is NULL");
    const DeviceGraph &G = g->g;
    const int block = (tune && tune->block_threads) ? (int)tune->block_threads : 1024;
    const int bps = (tune && tune->blocks_per_sm) ? (int)tune->blocks_per_sm : 2;
    const uint32_t hub = std::max<uint32_t>(32, (tune && tune->hub_degree) ? tune->hub_degree : 256);
    const void *kern = pr_kernel_for(block);
    if (!kern) return fail(GFT_ERR_INVALID_ARG, "gft_pr: block_threads must be 256, 512 or 1024");
    DeviceScope device_scope(e->device);
    GFT_CUDA_TRY(device_scope.err);
    LaunchShape shape;
    GFT_TRY(resolve_shape(e, kern, block, bps, 0, &shape));
    const uint32_t n = G.nnodes;
    const uint32_t hub_cap = std::max<uint32_t>(1, std::min<uint64_t>(n, (uint64_t)G.nedges / hub + 1));
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (std::max<size_t>(bytes, 4) + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_q0 = take((size_t)n * 4), o_q1 = take((size_t)n * 4), o_hubs = take((size_t)hub_cap * 8),
                 o_res = take((size_t)n * 4), o_upd = take((size_t)n * 4);
    GFT_TRY(e->scratch.ensure(off));
    char *base = static_cast<char *>(e->scratch.ptr);
    dev::PrParams pp{};
    dev::TravParams &p = pp.t;
    p.row_start = G.row_start;
    p.edge_dst = G.edge_dst;
    p.nnodes = n;
    p.q[0] = reinterpret_cast<uint32_t *>(base + o_q0);
    p.q[1] = reinterpret_cast<uint32_t *>(base + o_q1);
    p.hubs = reinterpret_cast<uint2 *>(base + o_hubs);
    p.hub_cap = hub_cap;
    p.hub_degree = hub;
    p.qcap = n;
    p.ctl = reinterpret_cast<TraversalCtl *>(e->ctl.ptr);
    p.timeout_ns = (unsigned long long)((tune && tune->timeout_ms) ? tune->timeout_ms : 20000) * 1000000ull;
    p.skip_block = -1;
    p.vec_ok = (uintptr_t)G.edge_dst % 16 == 0;
    p.nedges = G.nedges;
    p.uniform = G.max_degree <= kUniformDegree;
    pp.rank = d_rank;
    pp.residual = reinterpret_cast<float *>(base + o_res);
    pp.hub_upd = reinterpret_cast<float *>(base + o_upd);
    pp.max_iterations = max_iterations;
    GFT_CUDA_TRY(cudaMemsetAsync(e->ctl.ptr, 0, sizeof(TraversalCtl), stream));
    void *args[] = {&pp};
    GFT_CUDA_TRY(cudaEventRecord(e->ev0, stream));
    GFT_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(shape.blocks), dim3(shape.block_threads), args, 0, stream));
    GFT_CUDA_TRY(cudaEventRecord(e->ev1, stream));
    TraversalCtl *h = reinterpret_cast<TraversalCtl *>(e->host_ctl);
    const size_t cold = offsetof(TraversalCtl, error);
    GFT_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char *>(h) + cold, reinterpret_cast<char *>(e->ctl.ptr) + cold,
                                 sizeof(TraversalCtl) - cold, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h->error)
        return fail((gft_status)h->error, "gft_pr: device reported %s (site %u)", gft_status_string((gft_status)h->error),
                    h->error_where);
    if (stats) {
        memset(stats, 0, sizeof *stats);
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev0, e->ev1);
        stats->levels = h->levels;
        stats->iterations = h->iterations;
        stats->vertices_reached = n;
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

gft_status gft_pr(gft_engine *e, const gft_graph *g, float *d_rank, uint32_t max_iterations, const gft_tuning *tune,
                  void *stream, gft_stats *stats)
{
    if (!e) return fail(GFT_ERR_INVALID_ARG, "gft_pr: engine is NULL");
    std::lock_guard<std::mutex> lk(e->mu);
    return run_pr(e, g, d_rank, max_iterations, tune, (cudaStream_t)stream, stats);
}

gft_status gft_pr_host(gft_engine *e, const gft_graph *g, float *h_rank, uint32_t max_iterations,
                       const gft_tuning *tune, void *stream_, gft_stats *stats)
{
    if (!e) return fail(GFT_ERR_INVALID_ARG, "gft_pr_host: engine is NULL");
    if (!h_rank) return fail(GFT_ERR_INVALID_ARG, "gft_pr_host: output pointer is NULL");
    std::lock_guard<std::mutex> lk(e->mu);
    GFT_TRY(check_engine_graph(e, g));
    DeviceScope device_scope(g->g.device);
    GFT_CUDA_TRY(device_scope.err);
    cudaStream_t stream = (cudaStream_t)stream_;
    const size_t n = g->g.nnodes;
    GFT_TRY(e->aux.ensure(std::max<size_t>(n * 4, 256)));
    float *d_rank = reinterpret_cast<float *>(e->aux.ptr);
    GFT_TRY(run_pr(e, g, d_rank, max_iterations, tune, stream, stats));
    GFT_CUDA_TRY(cudaMemcpyAsync(h_rank, d_rank, n * 4, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    return GFT_OK;
}

}  // extern "C"
