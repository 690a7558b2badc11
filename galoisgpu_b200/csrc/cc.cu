// cc.cu -- connected components (gft_cc) on the engine's device graphs:
// the reference's apps/cc on the same frontier core.
//
// The reference (apps/cc/kernel.cu:630-723) hooks roots along every edge
// with racy plain stores, alternating high-to-low and low-to-high passes
// (:266-330), and pointer-jumps until nothing changes, with one grid-wide
// pass over all edges per round.  Here every edge is joined once, by a
// lock-free union-find:
//   find   follows parent links to the root, halving the path as it goes
//          (each link is replaced by the grandparent, always an ancestor);
//   union  finds both roots a < b and swings b's self-link to a with
//          atomicCAS; if b stopped being a root meanwhile the CAS fails and
//          the union retries from b's new parent.
// Links only ever point to a smaller vertex id, so a component's smallest
// vertex is never hooked and ends up as the root of the whole component:
// after a final compression every vertex is labelled with the smallest
// vertex id of its (weakly) connected component.  Unlike the reference's
// labels, these do not depend on the schedule.
//
// Launches, on the caller's stream.  On a graph marked symmetric, the sampled
// pass of Afforest (Sutton, Ben-Nun, Barak, IPDPS 2018): init; each vertex
// joins its first two neighbours; flatten; one CTA samples 1024 labels for
// the giant component; hook of the remaining edges of every vertex outside
// it; hook of those vertices' hub edges; compress + count.  Otherwise every
// edge is hooked: init; hook; hub hook; compress + count.  The hook flattens
// the edge lists of 32 vertices across the warp; vertices of degree >=
// kCcHubDegree go to a hub list, whose edges are hooked in kCcHubChunk-edge
// chunks.
#include <string.h>

#include <algorithm>

#include "gft_internal.h"
#include "traverse.cuh"

namespace gft {
namespace dev {

constexpr uint32_t kCcHubDegree = 2048;  // vertices with at least this many edges are split into chunks
constexpr uint32_t kCcHubChunk = 2048;

// Root of x.  Parent links are read from L2 (other SMs change them) and
// halved on the way: label[x] <- label[label[x]], an ancestor of x at the
// time of the read and therefore forever (trees only grow at the root).
__device__ __forceinline__ uint32_t cc_find(uint32_t *label, uint32_t x)
{
    uint32_t p = __ldcg(label + x);
    while (p != x) {
        const uint32_t g = __ldcg(label + p);
        if (g == p) return p;
        label[x] = g;
        x = g;
        p = __ldcg(label + x);
    }
    return x;
}

// Joins the components of u and v; the larger root is linked under the
// smaller one.
__device__ __forceinline__ void cc_union(uint32_t *label, uint32_t u, uint32_t v)
{
    uint32_t a = cc_find(label, u), b = cc_find(label, v);
    while (a != b) {
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicCAS(label + b, b, a);
        if (old == b) return;
        b = cc_find(label, old);
        a = cc_find(label, a);
    }
}

__global__ void cc_init(uint32_t *label, uint32_t n, unsigned long long *counters)
{
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    for (uint32_t v = tid; v < n; v += nthreads) label[v] = v;
    if (tid < 4) counters[tid] = 0;
}

// counters[0] = (hubs << 32) | hub chunks, counters[1] = edges joined,
// counters[2] = components.
// mode 0: every edge, each undirected edge once on a graph marked symmetric
//         (half_edges).  mode 1 (sampled, symmetric graphs only): the edges
//         from index `first` on of every vertex outside the sampled giant
//         component (its compressed label differs from *giant), in both
//         directions, since the other endpoint may be skipped.
__global__ void cc_hook(const uint32_t *__restrict__ row_start, const uint32_t *__restrict__ edge_dst, uint32_t n,
                        uint32_t *label, uint2 *hubs, uint32_t hub_cap, int half_edges, uint32_t first,
                        const uint32_t *giant, unsigned long long *counters, unsigned *error)
{
    const unsigned lane = threadIdx.x & 31;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t skip = giant ? __ldcg(giant) : 0xFFFFFFFFu;
    unsigned long long joined = 0;
    for (uint32_t base = gwarp * 32; base < n; base += nwarps * 32) {  // warp-uniform trip count
        const uint32_t u = base + lane;
        uint32_t start = 0, deg = 0;
        if (u < n && (!giant || __ldcg(label + u) != skip)) {
            start = __ldg(row_start + u);
            deg = __ldg(row_start + u + 1) - start;
            const uint32_t d0 = min(deg, first);
            start += d0;
            deg -= d0;
        }
        if (deg >= kCcHubDegree) {
            const unsigned nch = (deg + kCcHubChunk - 1) / kCcHubChunk;
            const unsigned long long old = atomicAdd(counters, (1ull << 32) | nch);
            const unsigned h = (unsigned)(old >> 32);
            if (h < hub_cap) hubs[h] = make_uint2(u, (unsigned)old);  // its edges from `first` on
            else atomicExch(error, (unsigned)GFT_ERR_OVERFLOW);
            deg = 0;
        }
        // Flatten the lanes' edge lists: the g-th edge of the block belongs
        // to the last lane whose exclusive degree prefix is <= g.
        const uint32_t incl = warp_incl_sum(deg, lane);
        const uint32_t total = __shfl_sync(kFull, incl, 31), excl = incl - deg;
        for (uint32_t g0 = 0; g0 < total; g0 += 32) {
            const uint32_t g = g0 + lane;
            int j = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1)
                if (__shfl_sync(kFull, excl, j + step) <= g) j += step;
            const uint32_t ostart = __shfl_sync(kFull, start, j), oexcl = __shfl_sync(kFull, excl, j);
            if (g < total) {
                const uint32_t src = base + j, dst = __ldcs(edge_dst + ostart + (g - oexcl));
                if (!half_edges || dst < src) {
                    cc_union(label, src, dst);
                    joined++;
                }
            }
        }
    }
    warp_add_u64(counters + 1, joined, lane);
}

// Hub edges: chunk c belongs to hub h with hubs[h].y <= c < hubs[h+1].y.
__global__ void cc_hook_hubs(const uint32_t *__restrict__ row_start, const uint32_t *__restrict__ edge_dst,
                             uint32_t *label, const uint2 *hubs, uint32_t hub_cap, int half_edges, uint32_t first,
                             unsigned long long *counters)
{
    const unsigned lane = threadIdx.x & 31;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const unsigned long long hv = __ldcg(counters);
    const uint32_t nh = min((uint32_t)(hv >> 32), hub_cap), nc = (uint32_t)hv;
    unsigned long long joined = 0;
    for (uint32_t c = gwarp; c < nc && nh; c += nwarps) {
        uint32_t lo = 0, hi = nh;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (hubs[mid].y <= c) lo = mid;
            else hi = mid;
        }
        const uint32_t u = hubs[lo].x, start = __ldg(row_start + u) + first,
                       deg = __ldg(row_start + u + 1) - start;
        const uint32_t off = (c - hubs[lo].y) * kCcHubChunk, len = min(kCcHubChunk, deg - off);
        for (uint32_t i = lane; i < len; i += 32) {
            const uint32_t dst = __ldcs(edge_dst + start + off + i);
            if (!half_edges || dst < u) {
                cc_union(label, u, dst);
                joined++;
            }
        }
    }
    warp_add_u64(counters + 1, joined, lane);
}

// Sampled pass, step 1: each vertex joins its first kCcSampleEdges
// neighbours (a thread per vertex; bounded work whatever the degree).  One
// flatten follows both rounds: a flatten between them was measured slower
// on both RMAT-24 and the 4096^2 road grid.
constexpr uint32_t kCcSampleEdges = 2;

__global__ void cc_neighbour_rounds(const uint32_t *__restrict__ row_start, const uint32_t *__restrict__ edge_dst,
                                    uint32_t n, uint32_t *label, unsigned long long *counters)
{
    const unsigned lane = threadIdx.x & 31;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    unsigned long long joined = 0;
    for (uint32_t r = 0; r < kCcSampleEdges; r++)
        for (uint32_t v = tid; v < n; v += nthreads) {
            const uint32_t s = __ldg(row_start + v);
            if (s + r < __ldg(row_start + v + 1)) {
                cc_union(label, v, __ldcs(edge_dst + s + r));
                joined++;
            }
        }
    warp_add_u64(counters + 1, joined, lane);
}

// Every label becomes its root (no union runs concurrently).
__global__ void cc_flatten(uint32_t *label, uint32_t n)
{
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    for (uint32_t v = tid; v < n; v += nthreads) {
        uint32_t r = v, p;
        while ((p = __ldcg(label + r)) != r) r = p;
        label[v] = r;
    }
}

// Sampled pass, step 2: the most frequent label among kCcSamples vertices
// drawn with a fixed multiplicative hash (one CTA).  A tie or a poor sample
// only skips fewer edges later; correctness never depends on it.
constexpr int kCcSamples = 1024;

__global__ void __launch_bounds__(kCcSamples, 1) cc_sample_giant(const uint32_t *label, uint32_t n, uint32_t *giant)
{
    __shared__ uint32_t s_lab[kCcSamples];
    __shared__ unsigned long long s_best;
    const uint32_t i = threadIdx.x;
    const uint32_t v = (uint32_t)(((unsigned long long)(i * 2654435761u + 12345u) * n) >> 32);
    s_lab[i] = n ? __ldcg(label + v) : 0;
    if (i == 0) s_best = 0;
    __syncthreads();
    uint32_t count = 0;
    for (int j = 0; j < kCcSamples; j++) count += s_lab[j] == s_lab[i];
    atomicMax(&s_best, ((unsigned long long)count << 32) | (0xFFFFFFFFu - s_lab[i]));
    __syncthreads();
    if (i == 0) *giant = 0xFFFFFFFFu - (uint32_t)s_best;
}

// Final labels.  No union runs any more, so the walk to the root only
// reads: a halving store here could land on a vertex whose own thread has
// already written its root and put back a non-root ancestor.  Each vertex's
// label is written by its own thread only, always with the root, so other
// walks that pass through it only get shorter.
__global__ void cc_compress(uint32_t *label, uint32_t n, unsigned long long *counters)
{
    const unsigned lane = threadIdx.x & 31;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    unsigned long long roots = 0;
    for (uint32_t v = tid; v < n; v += nthreads) {
        uint32_t r = v, p;
        while ((p = __ldcg(label + r)) != r) r = p;
        label[v] = r;
        roots += r == v;
    }
    warp_add_u64(counters + 2, roots, lane);
}

}  // namespace dev

namespace {

gft_status run_cc(gft_engine *e, const gft_graph *g, int32_t *d_label, const gft_tuning *tune, cudaStream_t stream,
                  gft_stats *stats, uint64_t *components)
{
    GFT_TRY(check_engine_graph(e, g));
    if (!d_label) return fail(GFT_ERR_INVALID_ARG, "gft_cc: label pointer is NULL");
    const DeviceGraph &G = g->g;
    DeviceScope device_scope(e->device);
    GFT_CUDA_TRY(device_scope.err);
    const uint32_t n = G.nnodes;
    const uint32_t hub_cap = std::max<uint32_t>(1, std::min<uint64_t>(n, (uint64_t)G.nedges / dev::kCcHubDegree + 1));
    const size_t o_ctr = 0, o_err = 256, o_giant = 320, o_hubs = 512;
    GFT_TRY(e->scratch.ensure(o_hubs + (size_t)hub_cap * sizeof(uint2)));
    char *base = static_cast<char *>(e->scratch.ptr);
    unsigned long long *ctr = reinterpret_cast<unsigned long long *>(base + o_ctr);
    unsigned *err = reinterpret_cast<unsigned *>(base + o_err);
    uint32_t *giant = reinterpret_cast<uint32_t *>(base + o_giant);
    uint2 *hubs = reinterpret_cast<uint2 *>(base + o_hubs);
    uint32_t *label = reinterpret_cast<uint32_t *>(d_label);
    const int block = 256;
    const int blocks = e->sms * 8;
    (void)tune;  // the launch shape is fixed: 8 CTAs of 256 threads per SM
    GFT_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(unsigned), stream));
    GFT_CUDA_TRY(cudaEventRecord(e->ev0, stream));
    dev::cc_init<<<blocks, block, 0, stream>>>(label, n, ctr);
    GFT_CUDA_TRY(cudaGetLastError());
    if (G.symmetric) {
        // Sampled pass (Sutton, Ben-Nun, Barak, "Optimizing Parallel Graph
        // Connectivity Computation via Subgraph Sampling", IPDPS 2018): join
        // each vertex with its first neighbours, find the giant component
        // from a sample, then join the remaining edges of the vertices
        // outside it only.  An edge (v, w) skipped at v, which lies in the
        // giant component, is joined at w unless w lies there too: on a
        // symmetric graph every edge is also w's edge.
        dev::cc_neighbour_rounds<<<blocks, block, 0, stream>>>(G.row_start, G.edge_dst, n, label, ctr);
        GFT_CUDA_TRY(cudaGetLastError());
        dev::cc_flatten<<<blocks, block, 0, stream>>>(label, n);
        GFT_CUDA_TRY(cudaGetLastError());
        dev::cc_sample_giant<<<1, dev::kCcSamples, 0, stream>>>(label, n, giant);
        GFT_CUDA_TRY(cudaGetLastError());
        dev::cc_hook<<<blocks, block, 0, stream>>>(G.row_start, G.edge_dst, n, label, hubs, hub_cap, 0,
                                                   dev::kCcSampleEdges, giant, ctr, err);
        GFT_CUDA_TRY(cudaGetLastError());
        dev::cc_hook_hubs<<<blocks, block, 0, stream>>>(G.row_start, G.edge_dst, label, hubs, hub_cap, 0,
                                                        dev::kCcSampleEdges, ctr);
    } else {
        dev::cc_hook<<<blocks, block, 0, stream>>>(G.row_start, G.edge_dst, n, label, hubs, hub_cap, 0, 0, nullptr,
                                                   ctr, err);
        GFT_CUDA_TRY(cudaGetLastError());
        dev::cc_hook_hubs<<<blocks, block, 0, stream>>>(G.row_start, G.edge_dst, label, hubs, hub_cap, 0, 0, ctr);
    }
    GFT_CUDA_TRY(cudaGetLastError());
    dev::cc_compress<<<blocks, block, 0, stream>>>(label, n, ctr);
    GFT_CUDA_TRY(cudaGetLastError());
    GFT_CUDA_TRY(cudaEventRecord(e->ev1, stream));
    unsigned long long h[3] = {0, 0, 0};
    unsigned herr = 0;
    GFT_CUDA_TRY(cudaMemcpyAsync(h, ctr, sizeof h, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    if (herr) return fail((gft_status)herr, "gft_cc: hub list overflow");
    if (components) *components = h[2];
    if (stats) {
        memset(stats, 0, sizeof *stats);
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev0, e->ev1);
        stats->levels = 1;
        stats->iterations = G.symmetric ? 7 : 4;  // kernel launches
        stats->vertices_reached = n;
        stats->edges_scanned = h[1];
        stats->kernel_ms = ms;
        stats->grid_blocks = blocks;
        stats->block_threads = block;
    }
    return GFT_OK;
}

}  // namespace
}  // namespace gft

using namespace gft;

extern "C" {

gft_status gft_cc(gft_engine *e, const gft_graph *g, int32_t *d_label, const gft_tuning *tune, void *stream,
                  gft_stats *stats, uint64_t *components)
{
    if (!e) return fail(GFT_ERR_INVALID_ARG, "gft_cc: engine is NULL");
    std::lock_guard<std::mutex> lk(e->mu);
    return run_cc(e, g, d_label, tune, (cudaStream_t)stream, stats, components);
}

gft_status gft_cc_host(gft_engine *e, const gft_graph *g, int32_t *h_label, const gft_tuning *tune, void *stream_,
                       gft_stats *stats, uint64_t *components)
{
    if (!e) return fail(GFT_ERR_INVALID_ARG, "gft_cc_host: engine is NULL");
    if (!h_label) return fail(GFT_ERR_INVALID_ARG, "gft_cc_host: output pointer is NULL");
    std::lock_guard<std::mutex> lk(e->mu);
    GFT_TRY(check_engine_graph(e, g));
    cudaStream_t stream = (cudaStream_t)stream_;
    const size_t n = g->g.nnodes;
    GFT_TRY(e->aux.ensure(std::max<size_t>(n * 4, 256)));
    int32_t *d_label = reinterpret_cast<int32_t *>(e->aux.ptr);
    GFT_TRY(run_cc(e, g, d_label, tune, stream, stats, components));
    GFT_CUDA_TRY(cudaMemcpyAsync(h_label, d_label, n * 4, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    return GFT_OK;
}

}  // extern "C"
