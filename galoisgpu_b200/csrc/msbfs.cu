// msbfs.cu -- multi-source BFS (gft_msbfs): up to 256 BFS queries on one
// graph in one persistent, cooperative launch.  No counterpart in the
// reference, which runs one source per process.
//
// Every vertex carries W = ceil(k / 32) words of bits, one bit per source:
// `seen` (sources that reached it) and, per level L, the frontier plane
// F_L (sources that reached it exactly at level L).  The planes are the
// result: level(source i, v) is the L whose plane has bit i set at v, so
// recording levels costs no writes beyond the frontier itself, and
// gft_msbfs_levels turns one source's planes into the int32 level array
// gft_bfs would produce.
//
// Each level runs in one of two directions, chosen from the edges leaving
// the frontier (m_f) against the graph's edges (Beamer, Asanovic,
// Patterson, "Direction-Optimizing Breadth-First Search", SC 2012):
//   top-down  (m_f small): a warp per frontier vertex u ORs F_L[u] & ~seen[v]
//             into next[v] for each neighbour v, then a commit pass over
//             the touched vertices moves next -> F_{L+1} and seen;
//   bottom-up (m_f large): a warp per vertex v ORs F_L[u] over its
//             neighbours u, restricted to the sources v still lacks, and
//             stops as soon as it has them all.  Uses v's out-edges as its
//             in-edges, so it requires a symmetric graph (flag
//             GFT_MSBFS_SYMMETRIC); without the flag every level runs
//             top-down.
#include <string.h>

#include <algorithm>

#include "gft_internal.h"
#include "traverse.cuh"

namespace gft {
namespace dev {

constexpr int kMaxWords = 8;  // 256 sources

struct MsParams {
    const uint32_t *__restrict__ row_start;
    const uint32_t *__restrict__ edge_dst;
    uint32_t nnodes, nedges;
    uint32_t k, words;         // sources, words per vertex
    const uint32_t *sources;   // device copy, k entries
    uint32_t *planes;          // (max_levels) x nnodes x words
    uint32_t max_levels;
    uint32_t *seen, *next;     // nnodes x words each (next zeroed)
    uint32_t *queue[2];        // frontier vertices per level
    uint32_t *touched;         // top-down: vertices given new bits
    uint32_t *tstamp;          // top-down: level + 1 at which v was last touched
    uint32_t symmetric;
    uint32_t alpha;            // bottom-up when m_f * alpha > nedges
    TraversalCtl *ctl;
    unsigned long long timeout_ns;
};

__device__ __forceinline__ uint32_t *row(uint32_t *base, uint32_t v, uint32_t words) { return base + (size_t)v * words; }

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) msbfs_kernel(MsParams p)
{
    TraversalCtl *ctl = p.ctl;
    const unsigned lane = threadIdx.x & 31;
    const unsigned tid = blockIdx.x * BLOCK + threadIdx.x, nthreads = gridDim.x * BLOCK;
    const unsigned gwarp = tid / 32, nwarps = nthreads / 32;
    GridSync gs{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, gridDim.x, 0, p.timeout_ns};
    const uint32_t n = p.nnodes, W = p.words;
    const size_t plane_words = (size_t)n * W;
    // Warp-aggregated appends (one reservation per flush) for the next
    // frontier and the top-down touched list.
    __shared__ uint32_t s_next[BLOCK / 32][kQueueBuf];
    __shared__ uint32_t s_touch[BLOCK / 32][kQueueBuf];
    WarpQueue nq{s_next[threadIdx.x >> 5], 0, nullptr, nullptr, n, &ctl->error, &ctl->error_where};
    WarpQueue tq{s_touch[threadIdx.x >> 5], 0, p.touched, nullptr, n, &ctl->error, &ctl->error_where};
    // counters: qlen[slot] frontier size, claim[slot] touched count,
    // hub[slot].v frontier edge count m_f.

    // Level 0: the sources themselves.
    for (size_t i = tid; i < plane_words; i += nthreads) {
        p.seen[i] = 0;
        p.planes[i] = 0;
    }
    if (!gs.sync()) return;
    if (tid == 0) {
        for (uint32_t i = 0; i < p.k; i++) {
            const uint32_t s = p.sources[i];
            row(p.seen, s, W)[i / 32] |= 1u << (i % 32);
            row(p.planes, s, W)[i / 32] |= 1u << (i % 32);
        }
        uint32_t nq = 0;
        unsigned long long mf = 0;
        for (uint32_t i = 0; i < p.k; i++) {
            const uint32_t s = p.sources[i];
            bool dup = false;
            for (uint32_t j = 0; j < i; j++) dup |= p.sources[j] == s;
            if (dup) continue;
            p.queue[0][nq++] = s;
            mf += p.row_start[s + 1] - p.row_start[s];
        }
        *u32_of(ctl->qlen[0]) = nq;
        ctl->hub[0].v = mf;
    }
    if (!gs.sync()) return;

    uint32_t L = 0;
    for (;;) {
        const unsigned slot = L % 3, nslot = (L + 1) % 3, rslot = (L + 2) % 3;
        const uint32_t nf = ld_relaxed_u32(u32_of(ctl->qlen[slot]));
        if (nf == 0) break;
        if (L + 1 >= p.max_levels) {
            if (tid == 0) raise_error(&ctl->error, &ctl->error_where, GFT_ERR_OVERFLOW, L + 1);
            gs.sync();
            return;
        }
        const unsigned long long mf = ld_relaxed_u64(&ctl->hub[slot].v);
        if (tid == 0) {
            *u32_of(ctl->qlen[rslot]) = 0;
            *u32_of(ctl->claim[rslot]) = 0;
            ctl->hub[rslot].v = 0;
        }
        const uint32_t *F = p.planes + (size_t)L * plane_words;
        uint32_t *Fn = p.planes + (size_t)(L + 1) * plane_words;
        uint32_t *qn = p.queue[(L + 1) & 1];
        unsigned *qn_len = u32_of(ctl->qlen[nslot]);
        unsigned long long *mf_next = &ctl->hub[nslot].v;
        nq.queue = qn;
        nq.len = qn_len;
        tq.len = u32_of(ctl->claim[slot]);
        unsigned long long my_mf = 0;
        const bool bottom_up = p.symmetric && mf * p.alpha > p.nedges;
        if (bottom_up) {
            // Dense pass: every vertex's next plane entry is written (0 when
            // nothing new), so the plane needs no clearing.
            for (uint32_t v = gwarp; v < n; v += nwarps) {
                uint32_t *sv = row(p.seen, v, W);
                uint32_t need[kMaxWords], acc[kMaxWords];
                bool any = false;
#pragma unroll
                for (int w = 0; w < kMaxWords; w++) {
                    need[w] = 0;
                    acc[w] = 0;
                    if (w < (int)W) {
                        const uint32_t valid = (w < (int)(p.k / 32)) ? ~0u : ((1u << (p.k % 32)) - 1);
                        need[w] = ~__ldcg(sv + w) & valid;
                        any |= need[w] != 0;
                    }
                }
                const uint32_t s = p.row_start[v], e = p.row_start[v + 1];
                if (any) {
                    for (uint32_t b = s; b < e; b += 32) {
                        if (b + lane < e) {
                            const uint32_t *fu = F + (size_t)__ldcs(p.edge_dst + b + lane) * W;
#pragma unroll
                            for (int w = 0; w < kMaxWords; w++)
                                if (w < (int)W && need[w]) acc[w] |= __ldcg(fu + w) & need[w];
                        }
                        bool done = true;
#pragma unroll
                        for (int w = 0; w < kMaxWords; w++) {
                            if (w < (int)W) {
#pragma unroll
                                for (int o = 16; o > 0; o >>= 1) acc[w] |= __shfl_xor_sync(kFull, acc[w], o);
                                done &= acc[w] == need[w];
                            }
                        }
                        if (done) break;
                    }
                }
                bool got = false;
                if (lane < W) {
                    uint32_t a = 0;
#pragma unroll
                    for (int w = 0; w < kMaxWords; w++)
                        if (w == (int)lane) a = acc[w];
                    row(Fn, v, W)[lane] = a;
                    if (a) sv[lane] |= a;
                }
#pragma unroll
                for (int w = 0; w < kMaxWords; w++) got |= acc[w] != 0;
                if (got && lane == 0) my_mf += e - s;
                nq.push(got && lane == 0, v, lane);
            }
        } else {
            // Top-down: clear the next plane, expand, commit.
            for (size_t i = tid; i < plane_words; i += nthreads) Fn[i] = 0;
            if (!gs.sync()) return;
            const uint32_t *q = p.queue[L & 1];
            for (uint32_t qi = gwarp; qi < nf; qi += nwarps) {
                const uint32_t u = __ldcg(q + qi);
                uint32_t fu[kMaxWords];
#pragma unroll
                for (int w = 0; w < kMaxWords; w++) fu[w] = w < (int)W ? __ldcg(F + (size_t)u * W + w) : 0u;
                const uint32_t s = p.row_start[u], e = p.row_start[u + 1];
                for (uint32_t eb = s; eb < e; eb += 32) {  // warp-uniform trip count
                    const uint32_t ei = eb + lane;
                    bool touched = false;
                    uint32_t v = 0;
                    if (ei < e) {
                        v = __ldcs(p.edge_dst + ei);
                        uint32_t *sv = row(p.seen, v, W), *nv = row(p.next, v, W);
#pragma unroll
                        for (int w = 0; w < kMaxWords; w++) {
                            if (w < (int)W && fu[w]) {
                                const uint32_t b = fu[w] & ~__ldcg(sv + w);
                                if (b) {
                                    atomicOr(nv + w, b);
                                    touched = true;
                                }
                            }
                        }
                        touched = touched && atomicExch(p.tstamp + v, L + 1) != L + 1;
                    }
                    tq.push(touched, v, lane);
                }
            }
            tq.flush(lane);
            if (!gs.sync()) return;
            const uint32_t nt = ld_relaxed_u32(u32_of(ctl->claim[slot]));
            for (uint32_t b = gwarp * 32; b < nt; b += nwarps * 32) {  // warp-uniform trip count
                const uint32_t ti = b + lane;
                bool got = false;
                uint32_t v = 0;
                if (ti < nt) {
                    v = __ldcg(p.touched + ti);
                    uint32_t *sv = row(p.seen, v, W), *nv = row(p.next, v, W), *fv = row(Fn, v, W);
                    for (uint32_t w = 0; w < W; w++) {
                        const uint32_t nb = __ldcg(nv + w) & ~__ldcg(sv + w);
                        nv[w] = 0;
                        if (nb) {
                            fv[w] = nb;
                            sv[w] |= nb;
                            got = true;
                        }
                    }
                    if (got) my_mf += p.row_start[v + 1] - p.row_start[v];
                }
                nq.push(got, v, lane);
            }
        }
        nq.flush(lane);
        warp_add_u64(mf_next, my_mf, lane);
        if (!gs.sync()) return;
        L++;
    }
    if (tid == 0) {
        ctl->levels = L;  // planes 0..L-1 hold the levels
        ctl->iterations = gs.epoch;
    }
}

// Level of source i at every vertex, from the planes.
__global__ void msbfs_levels_kernel(const uint32_t *__restrict__ planes, uint32_t nnodes, uint32_t words,
                                    uint32_t levels, uint32_t i, int32_t *out)
{
    const uint32_t w = i / 32, bit = 1u << (i % 32);
    const size_t plane_words = (size_t)nnodes * words;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nnodes; v += gridDim.x * blockDim.x) {
        int32_t lv = 0x7FFFFFFF;
        for (uint32_t L = 0; L < levels; L++)
            if (planes[(size_t)L * plane_words + (size_t)v * words + w] & bit) {
                lv = (int32_t)L;
                break;
            }
        out[v] = lv;
    }
}

}  // namespace dev
}  // namespace gft

using namespace gft;

extern "C" {

size_t gft_msbfs_plane_bytes(uint32_t nnodes, uint32_t k)
{
    return (size_t)nnodes * ((k + 31) / 32) * 4;
}

gft_status gft_msbfs(gft_engine *e, const gft_graph *g, const uint32_t *h_sources, uint32_t k, uint32_t *d_planes,
                     uint32_t max_levels, uint32_t flags, void *stream_, gft_stats *stats)
{
    if (!e || !g || !h_sources || !d_planes) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs: null argument");
    if (k == 0 || k > 256) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs: k must be 1..256 (got %u)", k);
    if (max_levels < 2) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs: max_levels must be >= 2");
    std::lock_guard<std::mutex> lk(e->mu);
    GFT_TRY(check_engine_graph(e, g));
    const DeviceGraph &G = g->g;
    for (uint32_t i = 0; i < k; i++)
        if (h_sources[i] >= G.nnodes) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs: source %u out of range", i);
    cudaStream_t stream = (cudaStream_t)stream_;
    GFT_CUDA_TRY(cudaSetDevice(e->device));
    const uint32_t W = (k + 31) / 32;
    const size_t vwords = (size_t)G.nnodes * W;
    auto a256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += a256(bytes);
        return o;
    };
    const size_t o_seen = take(vwords * 4), o_next = take(vwords * 4), o_q0 = take((size_t)G.nnodes * 4),
                 o_q1 = take((size_t)G.nnodes * 4), o_t = take((size_t)G.nnodes * 4),
                 o_ts = take((size_t)G.nnodes * 4), o_src = take((size_t)k * 4);
    GFT_TRY(e->scratch.ensure(off));
    char *base = static_cast<char *>(e->scratch.ptr);
    const void *kern = (const void *)dev::msbfs_kernel<512>;
    LaunchShape shape;
    GFT_TRY(resolve_shape(e, kern, 512, 2, 0, &shape));
    dev::MsParams p{};
    p.row_start = G.row_start;
    p.edge_dst = G.edge_dst;
    p.nnodes = G.nnodes;
    p.nedges = G.nedges;
    p.k = k;
    p.words = W;
    p.sources = reinterpret_cast<uint32_t *>(base + o_src);
    p.planes = d_planes;
    p.max_levels = max_levels;
    p.seen = reinterpret_cast<uint32_t *>(base + o_seen);
    p.next = reinterpret_cast<uint32_t *>(base + o_next);
    p.queue[0] = reinterpret_cast<uint32_t *>(base + o_q0);
    p.queue[1] = reinterpret_cast<uint32_t *>(base + o_q1);
    p.touched = reinterpret_cast<uint32_t *>(base + o_t);
    p.tstamp = reinterpret_cast<uint32_t *>(base + o_ts);
    p.symmetric = (flags & GFT_MSBFS_SYMMETRIC) ? 1u : 0u;
    p.alpha = 16;
    p.ctl = reinterpret_cast<TraversalCtl *>(e->ctl.ptr);
    p.timeout_ns = 20000ull * 1000000ull;
    GFT_CUDA_TRY(cudaMemcpyAsync(base + o_src, h_sources, (size_t)k * 4, cudaMemcpyHostToDevice, stream));
    GFT_CUDA_TRY(cudaMemsetAsync(base + o_next, 0, vwords * 4, stream));
    GFT_CUDA_TRY(cudaMemsetAsync(base + o_ts, 0, (size_t)G.nnodes * 4, stream));
    GFT_CUDA_TRY(cudaMemsetAsync(e->ctl.ptr, 0, sizeof(TraversalCtl), stream));
    void *args[] = {&p};
    GFT_CUDA_TRY(cudaEventRecord(e->ev0, stream));
    GFT_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(shape.blocks), dim3(512), args, 0, stream));
    GFT_CUDA_TRY(cudaEventRecord(e->ev1, stream));
    TraversalCtl *h = reinterpret_cast<TraversalCtl *>(e->host_ctl);
    const size_t cold = offsetof(TraversalCtl, error);
    GFT_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char *>(h) + cold, reinterpret_cast<char *>(e->ctl.ptr) + cold,
                                 sizeof(TraversalCtl) - cold, cudaMemcpyDeviceToHost, stream));
    GFT_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h->error)
        return fail((gft_status)h->error, "gft_msbfs: device reported %s (site %u)",
                    gft_status_string((gft_status)h->error), h->error_where);
    if (stats) {
        memset(stats, 0, sizeof *stats);
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev0, e->ev1);
        stats->levels = h->levels;
        stats->iterations = h->iterations;
        stats->kernel_ms = ms;
        stats->grid_blocks = shape.blocks;
        stats->block_threads = 512;
    }
    return GFT_OK;
}

gft_status gft_msbfs_levels(const uint32_t *d_planes, uint32_t nnodes, uint32_t k, uint32_t levels, uint32_t i,
                            int32_t *d_out, void *stream)
{
    if (!d_planes || !d_out || i >= k || k > 256) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs_levels: bad argument");
    dev::msbfs_levels_kernel<<<1184, 256, 0, (cudaStream_t)stream>>>(d_planes, nnodes, (k + 31) / 32, levels, i,
                                                                      d_out);
    GFT_CUDA_TRY(cudaGetLastError());
    return GFT_OK;
}

}  // extern "C"
