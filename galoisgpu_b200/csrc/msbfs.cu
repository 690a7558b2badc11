// msbfs.cu -- multi-source BFS (gft_msbfs): up to 256 BFS queries on one
// graph in one persistent, cooperative launch.  No counterpart in the
// reference, which runs one source per process.
//
// Every vertex carries a row of WP words of bits, one bit per source (WP =
// ceil(k / 32) rounded up to 1, 2, 4 or 8, so a row is one aligned vector
// load): `seen` (sources that reached it) and, per level L, the frontier
// plane F_L (sources that reached it exactly at level L).  The planes are the
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
//   bottom-up (m_f large): each vertex v ORs F_L[u] over its neighbours u,
//             restricted to the sources v still lacks, and stops once it has
//             them all.  A thread takes a vertex of at most kThreadDegree
//             edges (checking four edges at a time); the warp takes larger
//             ones together.  Uses v's out-edges as its in-edges, so it
//             requires a symmetric graph (flag GFT_MSBFS_SYMMETRIC); without
//             the flag every level runs top-down.
#include <string.h>

#include <algorithm>

#include "gft_internal.h"
#include "traverse.cuh"

namespace gft {
namespace dev {

constexpr uint32_t kThreadDegree = 32;  // bottom-up: larger vertices are scanned by the whole warp

// A row of WP words of source bits.
template <int WP>
struct Bits {
    uint32_t w[WP];
    __device__ __forceinline__ void clear()
    {
#pragma unroll
        for (int i = 0; i < WP; i++) w[i] = 0;
    }
    __device__ __forceinline__ bool any() const
    {
        uint32_t a = 0;
#pragma unroll
        for (int i = 0; i < WP; i++) a |= w[i];
        return a != 0;
    }
    __device__ __forceinline__ bool covers(const Bits &need) const
    {
        bool c = true;
#pragma unroll
        for (int i = 0; i < WP; i++) c &= (w[i] & need.w[i]) == need.w[i];
        return c;
    }
};

// Row loads and stores as aligned vectors (the row of v starts at v * WP
// words; the arrays are 16-byte aligned).
template <int WP>
__device__ __forceinline__ Bits<WP> ld_row(const uint32_t *base, uint32_t v)
{
    Bits<WP> b;
    const uint32_t *p = base + (size_t)v * WP;
    if constexpr (WP == 8) {
        const uint4 a = __ldcg(reinterpret_cast<const uint4 *>(p)), c = __ldcg(reinterpret_cast<const uint4 *>(p) + 1);
        b.w[0] = a.x, b.w[1] = a.y, b.w[2] = a.z, b.w[3] = a.w, b.w[4] = c.x, b.w[5] = c.y, b.w[6] = c.z, b.w[7] = c.w;
    } else if constexpr (WP == 4) {
        const uint4 a = __ldcg(reinterpret_cast<const uint4 *>(p));
        b.w[0] = a.x, b.w[1] = a.y, b.w[2] = a.z, b.w[3] = a.w;
    } else if constexpr (WP == 2) {
        const uint2 a = __ldcg(reinterpret_cast<const uint2 *>(p));
        b.w[0] = a.x, b.w[1] = a.y;
    } else {
        b.w[0] = __ldcg(p);
    }
    return b;
}

template <int WP>
__device__ __forceinline__ void st_row(uint32_t *base, uint32_t v, const Bits<WP> &b)
{
    uint32_t *p = base + (size_t)v * WP;
    if constexpr (WP == 8) {
        reinterpret_cast<uint4 *>(p)[0] = make_uint4(b.w[0], b.w[1], b.w[2], b.w[3]);
        reinterpret_cast<uint4 *>(p)[1] = make_uint4(b.w[4], b.w[5], b.w[6], b.w[7]);
    } else if constexpr (WP == 4) {
        reinterpret_cast<uint4 *>(p)[0] = make_uint4(b.w[0], b.w[1], b.w[2], b.w[3]);
    } else if constexpr (WP == 2) {
        reinterpret_cast<uint2 *>(p)[0] = make_uint2(b.w[0], b.w[1]);
    } else {
        p[0] = b.w[0];
    }
}

struct MsParams {
    const uint32_t *__restrict__ row_start;
    const uint32_t *__restrict__ edge_dst;
    uint32_t nnodes, nedges;
    uint32_t k;                // sources
    const uint32_t *sources;   // device copy, k entries
    uint32_t *planes;          // (max_levels) x nnodes x WP words
    uint32_t max_levels;
    uint32_t *seen, *next;     // nnodes x WP words each (next zeroed)
    uint32_t *queue[2];        // frontier vertices per level
    uint32_t *touched;         // top-down: vertices given new bits
    uint32_t *tstamp;          // top-down: level + 1 at which v was last touched
    uint32_t symmetric;
    uint32_t alpha;            // bottom-up when m_f * alpha > nedges
    TraversalCtl *ctl;
    unsigned long long timeout_ns;
};

// Bits of all k sources.
template <int WP>
__device__ __forceinline__ Bits<WP> all_sources(uint32_t k)
{
    Bits<WP> b;
#pragma unroll
    for (int i = 0; i < WP; i++)
        b.w[i] = 32u * (i + 1) <= k ? ~0u : (32u * i >= k ? 0u : (1u << (k % 32)) - 1u);
    return b;
}

template <int WP>
__global__ void __launch_bounds__(512, 2) msbfs_kernel(MsParams p)
{
    constexpr int BLOCK = 512;
    constexpr int kStep = WP >= 8 ? 2 : 4;  // edges a thread checks at once in bottom-up levels
    TraversalCtl *ctl = p.ctl;
    const unsigned lane = threadIdx.x & 31;
    const unsigned tid = blockIdx.x * BLOCK + threadIdx.x, nthreads = gridDim.x * BLOCK;
    const unsigned gwarp = tid / 32, nwarps = nthreads / 32;
    GridSync gs{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, gridDim.x, 0, p.timeout_ns};
    const uint32_t n = p.nnodes;
    const size_t plane_words = (size_t)n * WP;
    // Warp-aggregated appends (one reservation per flush) for the next
    // frontier and the top-down touched list.
    __shared__ uint32_t s_next[BLOCK / 32][kQueueBuf];
    __shared__ uint32_t s_touch[BLOCK / 32][kQueueBuf];
    WarpQueue nq{s_next[threadIdx.x >> 5], 0, nullptr, nullptr, n, &ctl->error, &ctl->error_where};
    WarpQueue tq{s_touch[threadIdx.x >> 5], 0, p.touched, nullptr, n, &ctl->error, &ctl->error_where};
    const Bits<WP> all = all_sources<WP>(p.k);
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
            p.seen[(size_t)s * WP + i / 32] |= 1u << (i % 32);
            p.planes[(size_t)s * WP + i / 32] |= 1u << (i % 32);
        }
        uint32_t nq0 = 0;
        unsigned long long mf = 0;
        for (uint32_t i = 0; i < p.k; i++) {
            const uint32_t s = p.sources[i];
            bool dup = false;
            for (uint32_t j = 0; j < i; j++) dup |= p.sources[j] == s;
            if (dup) continue;
            p.queue[0][nq0++] = s;
            mf += p.row_start[s + 1] - p.row_start[s];
        }
        *u32_of(ctl->qlen[0]) = nq0;
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
        nq.queue = ((L + 1) & 1) ? p.queue[1] : p.queue[0];  // no dynamic index: keeps p out of local memory
        nq.len = u32_of(ctl->qlen[nslot]);
        tq.len = u32_of(ctl->claim[slot]);
        unsigned long long my_mf = 0;
        const bool bottom_up = p.symmetric && mf * p.alpha > p.nedges;
        if (bottom_up) {
            // Dense pass over 32-vertex blocks: every vertex's next plane row
            // is written (0 when nothing new), so the plane needs no clearing.
            for (uint32_t b0 = gwarp * 32; b0 < n; b0 += nwarps * 32) {  // warp-uniform trip count
                const uint32_t v = b0 + lane;
                Bits<WP> need, acc;
                need.clear();
                acc.clear();
                uint32_t s = 0, e = 0;
                if (v < n) {
                    const Bits<WP> sv = ld_row<WP>(p.seen, v);
#pragma unroll
                    for (int i = 0; i < WP; i++) need.w[i] = all.w[i] & ~sv.w[i];
                    if (need.any()) {
                        s = __ldg(p.row_start + v);
                        e = __ldg(p.row_start + v + 1);
                    }
                }
                const bool heavy = e - s > kThreadDegree;
                if (!heavy) {  // this thread's own vertex, kStep edges at a time
                    for (uint32_t i = s; i < e; i += kStep) {
                        uint32_t u[kStep];
#pragma unroll
                        for (int k = 0; k < kStep; k++) u[k] = i + k < e ? __ldcs(p.edge_dst + i + k) : 0xFFFFFFFFu;
#pragma unroll
                        for (int k = 0; k < kStep; k++)
                            if (u[k] != 0xFFFFFFFFu) {
                                const Bits<WP> f = ld_row<WP>(F, u[k]);
#pragma unroll
                                for (int w = 0; w < WP; w++) acc.w[w] |= f.w[w] & need.w[w];
                            }
                        if (acc.covers(need)) break;
                    }
                }
                // The whole warp scans each heavy vertex of the block in turn.
                unsigned hm = __ballot_sync(kFull, heavy);
                while (hm) {
                    const int j = __ffs(hm) - 1;
                    hm &= hm - 1;
                    const uint32_t sj = __shfl_sync(kFull, s, j), ej = __shfl_sync(kFull, e, j);
                    Bits<WP> nj, a;
#pragma unroll
                    for (int w = 0; w < WP; w++) nj.w[w] = __shfl_sync(kFull, need.w[w], j);
                    a.clear();
                    for (uint32_t b = sj; b < ej; b += 32) {
                        if (b + lane < ej) {
                            const Bits<WP> f = ld_row<WP>(F, __ldcs(p.edge_dst + b + lane));
#pragma unroll
                            for (int w = 0; w < WP; w++) a.w[w] |= f.w[w] & nj.w[w];
                        }
#pragma unroll
                        for (int w = 0; w < WP; w++)
#pragma unroll
                            for (int o = 16; o > 0; o >>= 1) a.w[w] |= __shfl_xor_sync(kFull, a.w[w], o);
                        if (a.covers(nj)) break;  // warp uniform after the reduction
                    }
                    if ((int)lane == j) acc = a;
                }
                const bool got = acc.any();
                if (v < n) {
                    st_row<WP>(Fn, v, acc);
                    if (got) {
                        Bits<WP> s2;
#pragma unroll
                        for (int i = 0; i < WP; i++) s2.w[i] = (all.w[i] & ~need.w[i]) | acc.w[i];
                        st_row<WP>(p.seen, v, s2);
                        my_mf += e - s;
                    }
                }
                nq.push(got, v, lane);
            }
        } else {
            // Top-down: clear the next plane, expand, commit.
            for (size_t i = tid; i < plane_words; i += nthreads) Fn[i] = 0;
            if (!gs.sync()) return;
            const uint32_t *q = (L & 1) ? p.queue[1] : p.queue[0];
            for (uint32_t qi = gwarp; qi < nf; qi += nwarps) {
                const uint32_t u = __ldcg(q + qi);
                const Bits<WP> fu = ld_row<WP>(F, u);
                const uint32_t s = __ldg(p.row_start + u), e = __ldg(p.row_start + u + 1);
                for (uint32_t eb = s; eb < e; eb += 32) {  // warp-uniform trip count
                    const uint32_t ei = eb + lane;
                    bool touched = false;
                    uint32_t v = 0;
                    if (ei < e) {
                        v = __ldcs(p.edge_dst + ei);
                        const Bits<WP> sv = ld_row<WP>(p.seen, v);
#pragma unroll
                        for (int w = 0; w < WP; w++) {
                            const uint32_t b = fu.w[w] & ~sv.w[w];
                            if (b) {
                                atomicOr(p.next + (size_t)v * WP + w, b);
                                touched = true;
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
                    Bits<WP> nb = ld_row<WP>(p.next, v);
                    const Bits<WP> sv = ld_row<WP>(p.seen, v);
#pragma unroll
                    for (int w = 0; w < WP; w++) nb.w[w] &= ~sv.w[w];
                    Bits<WP> z;
                    z.clear();
                    st_row<WP>(p.next, v, z);
                    if (nb.any()) {
                        st_row<WP>(Fn, v, nb);
                        Bits<WP> s2;
#pragma unroll
                        for (int w = 0; w < WP; w++) s2.w[w] = sv.w[w] | nb.w[w];
                        st_row<WP>(p.seen, v, s2);
                        got = true;
                        my_mf += p.row_start[v + 1] - p.row_start[v];
                    }
                }
                nq.push(got, v, lane);
            }
        }
        nq.flush(lane);
        warp_add_u64(&ctl->hub[nslot].v, my_mf, lane);
        if (!gs.sync()) return;
        L++;
    }
    if (tid == 0) {
        ctl->levels = L;  // planes 0..L-1 hold the levels
        ctl->iterations = gs.epoch;
    }
}

// Level of source i at every vertex, from the planes (rows of wp words).
__global__ void msbfs_levels_kernel(const uint32_t *__restrict__ planes, uint32_t nnodes, uint32_t wp,
                                    uint32_t levels, uint32_t i, int32_t *out)
{
    const uint32_t w = i / 32, bit = 1u << (i % 32);
    const size_t plane_words = (size_t)nnodes * wp;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nnodes; v += gridDim.x * blockDim.x) {
        int32_t lv = 0x7FFFFFFF;
        for (uint32_t L = 0; L < levels; L++)
            if (planes[(size_t)L * plane_words + (size_t)v * wp + w] & bit) {
                lv = (int32_t)L;
                break;
            }
        out[v] = lv;
    }
}

}  // namespace dev
}  // namespace gft

using namespace gft;

namespace {

// Words per vertex row for k sources: ceil(k / 32) rounded up to a power of
// two, so every row is one aligned vector.
uint32_t row_words(uint32_t k)
{
    const uint32_t w = (k + 31) / 32;
    return w <= 1 ? 1 : w <= 2 ? 2 : w <= 4 ? 4 : 8;
}

const void *msbfs_kernel_for(uint32_t wp)
{
    switch (wp) {
    case 1: return (const void *)dev::msbfs_kernel<1>;
    case 2: return (const void *)dev::msbfs_kernel<2>;
    case 4: return (const void *)dev::msbfs_kernel<4>;
    case 8: return (const void *)dev::msbfs_kernel<8>;
    }
    return nullptr;
}

}  // namespace

extern "C" {

size_t gft_msbfs_plane_bytes(uint32_t nnodes, uint32_t k)
{
    return (size_t)nnodes * row_words(k) * 4;
}

gft_status gft_msbfs(gft_engine *e, const gft_graph *g, const uint32_t *h_sources, uint32_t k, uint32_t *d_planes,
                     uint32_t max_levels, uint32_t flags, void *stream_, gft_stats *stats)
{
    if (!e || !g || !h_sources || !d_planes) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs: null argument");
    if (k == 0 || k > 256) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs: k must be 1..256 (got %u)", k);
    if (max_levels < 2) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs: max_levels must be >= 2");
    if ((uintptr_t)d_planes % 16 != 0) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs: d_planes must be 16-byte aligned");
    std::lock_guard<std::mutex> lk(e->mu);
    GFT_TRY(check_engine_graph(e, g));
    const DeviceGraph &G = g->g;
    for (uint32_t i = 0; i < k; i++)
        if (h_sources[i] >= G.nnodes) return fail(GFT_ERR_INVALID_ARG, "gft_msbfs: source %u out of range", i);
    cudaStream_t stream = (cudaStream_t)stream_;
    DeviceScope device_scope(e->device);
    GFT_CUDA_TRY(device_scope.err);
    const uint32_t WP = row_words(k);
    const size_t vwords = (size_t)G.nnodes * WP;
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
    const void *kern = msbfs_kernel_for(WP);
    LaunchShape shape;
    GFT_TRY(resolve_shape(e, kern, 512, 2, 0, &shape));
    dev::MsParams p{};
    p.row_start = G.row_start;
    p.edge_dst = G.edge_dst;
    p.nnodes = G.nnodes;
    p.nedges = G.nedges;
    p.k = k;
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
    // Bottom-up once the frontier's edges exceed 1/64 of the graph's: a
    // bottom-up level checks a vertex's rows only until its sources are
    // covered, a top-down one pays atomics per edge for every source row.
    // 256 sources: RMAT-24 44.3 -> 42.8 ms and road 512^2 2.47 -> 2.28 ms
    // against 1/16 (Beamer et al.'s single-source value).
    p.alpha = 64;
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
    // Launch on the device that holds the planes, whatever device is current.
    cudaPointerAttributes attr;
    GFT_CUDA_TRY(cudaPointerGetAttributes(&attr, d_planes));
    if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
        return fail(GFT_ERR_INVALID_ARG, "gft_msbfs_levels: d_planes is not device memory");
    DeviceScope device_scope(attr.device);
    GFT_CUDA_TRY(device_scope.err);
    dev::msbfs_levels_kernel<<<1184, 256, 0, (cudaStream_t)stream>>>(d_planes, nnodes, row_words(k), levels, i, d_out);
    GFT_CUDA_TRY(cudaGetLastError());
    return GFT_OK;
}

}  // extern "C"
