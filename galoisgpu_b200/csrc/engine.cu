// engine.cu -- device graphs, engines (per-device traversal scratch) and
// persistent-grid sizing.
//
// Graph upload replaces CSRGraph::allocOnDevice / copy_to_gpu
// (rt/src/csr_graph.cu:222-261): one allocation per array, copies on the
// caller's stream, and edge_data only when the graph is weighted.  Grid
// sizing replaces maximum_residency / ggc_get_nSM
// (rt/include/cuda_launch_config.hpp:205-265, rt/src/ggc_rt.cu:23-28):
// the CUDA occupancy API gives the true per-SM residency on sm_100, and the
// launch is cooperative so an over-sized grid is refused, never run.
#include <string.h>

#include <algorithm>

#include "gft_internal.h"

namespace gft {

gft_status Scratch::ensure(size_t want)
{
    if (want <= bytes && ptr) return GFT_OK;
    if (ptr) {
        cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    size_t grow = std::max(want, (size_t)1 << 16);
    cudaError_t e = cudaMalloc(&ptr, grow);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return fail(GFT_ERR_OOM, "scratch allocation of %zu bytes failed: %s", grow, cudaGetErrorString(e));
    }
    bytes = grow;
    return GFT_OK;
}

void Scratch::release()
{
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

namespace dev {
__global__ void max_degree_kernel(const uint32_t *__restrict__ row_start, uint32_t n, unsigned *out)
{
    unsigned m = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        m = max(m, row_start[v + 1] - row_start[v]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// Lowest index of an edge whose destination is >= n, into *first.
__global__ void first_bad_edge(const uint32_t *__restrict__ dst, uint32_t m, uint32_t n, unsigned long long *first)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x)
        if (__ldcs(dst + e) >= n) {
            atomicMin(first, (unsigned long long)e);
            return;
        }
}

// One 16-byte slot per vertex: its destinations, or kBfsSlotWide for a
// vertex of more than 4 edges or of an edge leaving the graph.
__global__ void build_bfs_slots(const uint32_t *__restrict__ row_start, const uint32_t *__restrict__ dst, uint32_t n,
                                uint4 *__restrict__ slots)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t s = row_start[v], d = row_start[v + 1] - s;
        uint4 x = make_uint4(kBfsSlotNone, kBfsSlotNone, kBfsSlotNone, kBfsSlotNone);
        if (d > 4) x.x = kBfsSlotWide;
        else {
            if (d > 0) x.x = dst[s];
            if (d > 1) x.y = dst[s + 1];
            if (d > 2) x.z = dst[s + 2];
            if (d > 3) x.w = dst[s + 3];
            // A destination outside the graph sends the vertex through the
            // CSR, whose reader reports it; slot destinations are in range.
            if ((d > 0 && x.x >= n) || (d > 1 && x.y >= n) || (d > 2 && x.z >= n) || (d > 3 && x.w >= n))
                x = make_uint4(kBfsSlotWide, kBfsSlotNone, kBfsSlotNone, kBfsSlotNone);
        }
        slots[v] = x;
    }
}

__global__ void interleave_edges(const uint32_t *__restrict__ dst, const int32_t *__restrict__ w, uint32_t m,
                                 uint2 *__restrict__ out)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x)
        out[e] = make_uint2(dst[e], (uint32_t)w[e]);
}
}  // namespace dev

gft_status ensure_edge_pairs(gft_graph *g, cudaStream_t stream)
{
    std::lock_guard<std::mutex> lk(g->pair_mu);
    DeviceGraph &G = g->g;
    if (G.edge_dw || !G.edge_data || !G.nedges) return GFT_OK;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return GFT_OK;
    DeviceScope device_scope(G.device);
    GFT_CUDA_TRY(device_scope.err);
    uint2 *p = nullptr;
    if (cudaMalloc(&p, (size_t)G.nedges * sizeof(uint2)) != cudaSuccess) {
        cudaGetLastError();  // no room: queries keep reading the separate arrays
        return GFT_OK;
    }
    dev::interleave_edges<<<148 * 8, 256, 0, stream>>>(G.edge_dst, G.edge_data, G.nedges, p);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) {
        cudaFree(p);
        return fail(GFT_ERR_CUDA, "interleaving edges: %s", cudaGetErrorString(err));
    }
    G.edge_dw = p;  // complete before any query can see it
    return GFT_OK;
}

gft_status ensure_bfs_slots(gft_graph *g, cudaStream_t stream)
{
    std::lock_guard<std::mutex> lk(g->pair_mu);
    DeviceGraph &G = g->g;
    if (G.bfs_slots || !G.nnodes) return GFT_OK;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return GFT_OK;
    DeviceScope device_scope(G.device);
    GFT_CUDA_TRY(device_scope.err);
    uint4 *p = nullptr;
    if (cudaMalloc(&p, (size_t)G.nnodes * sizeof(uint4)) != cudaSuccess) {
        cudaGetLastError();  // no room: the BFS reads the CSR
        return GFT_OK;
    }
    dev::build_bfs_slots<<<148 * 4, 256, 0, stream>>>(G.row_start, G.edge_dst, G.nnodes, p);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) {
        cudaFree(p);
        return fail(GFT_ERR_CUDA, "building BFS slots: %s", cudaGetErrorString(err));
    }
    G.bfs_slots = p;  // complete before any query can see it
    return GFT_OK;
}

gft_status graph_degree_stats(DeviceGraph &G, cudaStream_t stream)
{
    unsigned *d = nullptr, h = 0;
    GFT_CUDA_TRY(cudaMallocAsync(&d, sizeof(unsigned), stream));
    cudaError_t err = cudaMemsetAsync(d, 0, sizeof(unsigned), stream);
    if (err == cudaSuccess && G.nnodes) {
        dev::max_degree_kernel<<<592, 256, 0, stream>>>(G.row_start, G.nnodes, d);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpyAsync(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost, stream);
    cudaFreeAsync(d, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    GFT_CUDA_TRY(err);
    G.max_degree = h;
    return GFT_OK;
}

gft_status check_edges_device(const DeviceGraph &G, cudaStream_t stream, uint64_t *first_bad)
{
    unsigned long long *d = nullptr, h = ~0ull;
    *first_bad = ~0ull;
    if (!G.nedges) return GFT_OK;
    GFT_CUDA_TRY(cudaMallocAsync(&d, sizeof h, stream));
    cudaError_t err = cudaMemcpyAsync(d, &h, sizeof h, cudaMemcpyHostToDevice, stream);
    if (err == cudaSuccess) {
        dev::first_bad_edge<<<148 * 8, 256, 0, stream>>>(G.edge_dst, G.nedges, G.nnodes, d);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, stream);
    cudaFreeAsync(d, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    GFT_CUDA_TRY(err);
    *first_bad = h;
    return GFT_OK;
}

gft_status resolve_shape(gft_engine *e, const void *kernel, int block_threads, int blocks_per_sm, size_t dyn_smem,
                         LaunchShape *out)
{
    int occ = 0;
    GFT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, block_threads, dyn_smem));
    if (occ <= 0) return fail(GFT_ERR_NOT_SUPPORTED, "kernel cannot run with %d threads per block", block_threads);
    out->block_threads = block_threads;
    out->blocks_per_sm = std::max(1, std::min(occ, blocks_per_sm));
    out->sms = e->sms;
    out->blocks = out->blocks_per_sm * e->sms;
    return GFT_OK;
}

gft_status check_engine_graph(gft_engine *e, const gft_graph *g)
{
    if (!e) return fail(GFT_ERR_INVALID_ARG, "engine is NULL");
    if (!g) return fail(GFT_ERR_INVALID_ARG, "graph is NULL");
    if (g->g.device != e->device)
        return fail(GFT_ERR_INVALID_ARG, "graph lives on device %d, engine on device %d", g->g.device, e->device);
    return GFT_OK;
}

static gft_status device_ok(int device, int *sms, int *major, int *minor)
{
    int n = 0;
    GFT_CUDA_TRY(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(GFT_ERR_INVALID_ARG, "device %d out of range (%d devices)", device, n);
    cudaDeviceProp prop;
    GFT_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return fail(GFT_ERR_NOT_SUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a only", device,
                    prop.major, prop.minor);
    if (!prop.cooperativeLaunch)
        return fail(GFT_ERR_NOT_SUPPORTED, "device %d does not support cooperative launches", device);
    if (sms) *sms = prop.multiProcessorCount;
    if (major) *major = prop.major;
    if (minor) *minor = prop.minor;
    return GFT_OK;
}

}  // namespace gft

using namespace gft;

extern "C" {

gft_status gft_engine_create(int device, gft_engine **out)
{
    if (!out) return fail(GFT_ERR_INVALID_ARG, "gft_engine_create: out is NULL");
    *out = nullptr;
    int sms = 0, major = 0, minor = 0;
    GFT_TRY(device_ok(device, &sms, &major, &minor));
    DeviceScope device_scope(device);
    GFT_CUDA_TRY(device_scope.err);
    gft_engine *e = new gft_engine();
    e->device = device;
    e->sms = sms;
    e->cc_major = major;
    e->cc_minor = minor;
    gft_status s = e->ctl.ensure(sizeof(TraversalCtl));
    if (s == GFT_OK && cudaMallocHost(&e->host_ctl, sizeof(TraversalCtl)) != cudaSuccess)
        s = fail(GFT_ERR_OOM, "gft_engine_create: pinned allocation failed");
    if (s == GFT_OK && (cudaEventCreate(&e->ev0) != cudaSuccess || cudaEventCreate(&e->ev1) != cudaSuccess))
        s = fail(GFT_ERR_CUDA, "gft_engine_create: event creation failed");
    if (s != GFT_OK) {
        gft_engine_destroy(e);
        return s;
    }
    *out = e;
    return GFT_OK;
}

void gft_engine_destroy(gft_engine *e)
{
    if (!e) return;
    DeviceScope device_scope(e->device);
    e->scratch.release();
    e->ctl.release();
    e->aux.release();
    if (e->host_ctl) cudaFreeHost(e->host_ctl);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->copy_stream) cudaStreamSynchronize(e->copy_stream), cudaStreamDestroy(e->copy_stream);
    for (int i = 0; i < 2; i++) {
        if (e->result_ready[i]) cudaEventDestroy(e->result_ready[i]);
        if (e->copy_done[i]) cudaEventDestroy(e->copy_done[i]);
    }
    delete e;
}

size_t gft_engine_scratch_bytes(const gft_engine *e)
{
    return e ? e->scratch.bytes + e->ctl.bytes + e->aux.bytes : 0;
}

gft_status gft_graph_upload(int device, const gft_csr *h, void *stream_, gft_graph **out)
{
    if (!h || !out || !h->row_start || (h->nedges && !h->edge_dst))
        return fail(GFT_ERR_INVALID_ARG, "gft_graph_upload: null argument");
    if (h->row_start[h->nnodes] != h->nedges)
        return fail(GFT_ERR_INVALID_ARG, "gft_graph_upload: row_start[nnodes] != nedges");
    *out = nullptr;
    GFT_TRY(device_ok(device, nullptr, nullptr, nullptr));
    DeviceScope device_scope(device);
    GFT_CUDA_TRY(device_scope.err);
    cudaStream_t stream = (cudaStream_t)stream_;
    gft_graph *g = new gft_graph();
    DeviceGraph &G = g->g;
    G.device = device;
    G.nnodes = h->nnodes;
    G.nedges = h->nedges;
    cudaError_t err = cudaMalloc(&G.row_start, ((size_t)h->nnodes + 1) * 4);
    if (err == cudaSuccess) err = cudaMalloc(&G.edge_dst, std::max<size_t>(h->nedges, 1) * 4);
    if (err == cudaSuccess && h->edge_data) err = cudaMalloc(&G.edge_data, std::max<size_t>(h->nedges, 1) * 4);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(G.row_start, h->row_start, ((size_t)h->nnodes + 1) * 4, cudaMemcpyHostToDevice, stream);
    if (err == cudaSuccess && h->nedges)
        err = cudaMemcpyAsync(G.edge_dst, h->edge_dst, (size_t)h->nedges * 4, cudaMemcpyHostToDevice, stream);
    if (err == cudaSuccess && h->edge_data && h->nedges)
        err = cudaMemcpyAsync(G.edge_data, h->edge_data, (size_t)h->nedges * 4, cudaMemcpyHostToDevice, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) {
        gft_graph_free(g);
        return fail(err == cudaErrorMemoryAllocation ? GFT_ERR_OOM : GFT_ERR_CUDA, "gft_graph_upload: %s",
                    cudaGetErrorString(err));
    }
    for (uint32_t v = 0; v < h->nnodes; v++) G.max_degree = std::max(G.max_degree, h->row_start[v + 1] - h->row_start[v]);
    *out = g;
    return GFT_OK;
}

gft_status gft_graph_wrap(int device, uint32_t nnodes, uint32_t nedges, const uint32_t *d_row_start,
                          const uint32_t *d_edge_dst, const int32_t *d_edge_data, gft_graph **out)
{
    if (!out || !d_row_start || (nedges && !d_edge_dst))
        return fail(GFT_ERR_INVALID_ARG, "gft_graph_wrap: null argument");
    GFT_TRY(device_ok(device, nullptr, nullptr, nullptr));
    gft_graph *g = new gft_graph();
    g->g.device = device;
    g->g.nnodes = nnodes;
    g->g.nedges = nedges;
    g->g.row_start = const_cast<uint32_t *>(d_row_start);
    g->g.edge_dst = const_cast<uint32_t *>(d_edge_dst);
    g->g.edge_data = const_cast<int32_t *>(d_edge_data);
    g->g.wrapped = true;
    DeviceScope device_scope(device);
    gft_status st = device_scope.err == cudaSuccess ? graph_degree_stats(g->g, nullptr)
                                                    : fail(GFT_ERR_CUDA, "gft_graph_wrap: cudaSetDevice failed");
    if (st != GFT_OK) {
        delete g;
        return st;
    }
    *out = g;
    return GFT_OK;
}

gft_status gft_graph_set_symmetric(gft_graph *g, int symmetric)
{
    if (!g) return fail(GFT_ERR_INVALID_ARG, "gft_graph_set_symmetric: graph is NULL");
    g->g.symmetric = symmetric != 0;
    return GFT_OK;
}

gft_status gft_graph_is_symmetric(const gft_graph *g, int *symmetric)
{
    if (!g || !symmetric) return fail(GFT_ERR_INVALID_ARG, "gft_graph_is_symmetric: null argument");
    *symmetric = g->g.symmetric ? 1 : 0;
    return GFT_OK;
}

gft_status gft_graph_info(const gft_graph *g, uint32_t *nnodes, uint32_t *nedges, int *weighted)
{
    if (!g) return fail(GFT_ERR_INVALID_ARG, "gft_graph_info: graph is NULL");
    if (nnodes) *nnodes = g->g.nnodes;
    if (nedges) *nedges = g->g.nedges;
    if (weighted) *weighted = g->g.edge_data != nullptr;
    return GFT_OK;
}

gft_status gft_graph_arrays(const gft_graph *g, const uint32_t **d_row_start, const uint32_t **d_edge_dst,
                            const int32_t **d_edge_data)
{
    if (!g) return fail(GFT_ERR_INVALID_ARG, "gft_graph_arrays: graph is NULL");
    if (d_row_start) *d_row_start = g->g.row_start;
    if (d_edge_dst) *d_edge_dst = g->g.edge_dst;
    if (d_edge_data) *d_edge_data = g->g.edge_data;
    return GFT_OK;
}

gft_status gft_graph_download(const gft_graph *g, gft_csr *out)
{
    if (!g || !out) return fail(GFT_ERR_INVALID_ARG, "gft_graph_download: null argument");
    memset(out, 0, sizeof *out);
    const DeviceGraph &G = g->g;
    DeviceScope device_scope(G.device);
    GFT_CUDA_TRY(device_scope.err);
    out->nnodes = G.nnodes;
    out->nedges = G.nedges;
    out->row_start = (uint32_t *)malloc(((size_t)G.nnodes + 1) * 4);
    out->edge_dst = (uint32_t *)malloc(std::max<size_t>(G.nedges, 1) * 4);
    if (G.edge_data) out->edge_data = (int32_t *)malloc(std::max<size_t>(G.nedges, 1) * 4);
    if (!out->row_start || !out->edge_dst || (G.edge_data && !out->edge_data)) {
        gft_csr_free(out);
        return fail(GFT_ERR_OOM, "gft_graph_download: host allocation failed");
    }
    cudaError_t err = cudaMemcpy(out->row_start, G.row_start, ((size_t)G.nnodes + 1) * 4, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess && G.nedges)
        err = cudaMemcpy(out->edge_dst, G.edge_dst, (size_t)G.nedges * 4, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess && G.edge_data && G.nedges)
        err = cudaMemcpy(out->edge_data, G.edge_data, (size_t)G.nedges * 4, cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) {
        gft_csr_free(out);
        return fail(GFT_ERR_CUDA, "gft_graph_download: %s", cudaGetErrorString(err));
    }
    return GFT_OK;
}

gft_status gft_graph_pick_sources(const gft_graph *g, uint64_t seed, uint32_t k, uint32_t *out_sources)
{
    if (!g || (k && !out_sources)) return fail(GFT_ERR_INVALID_ARG, "gft_graph_pick_sources: null argument");
    std::vector<uint32_t> rs((size_t)g->g.nnodes + 1);
    DeviceScope device_scope(g->g.device);
    GFT_CUDA_TRY(device_scope.err);
    GFT_CUDA_TRY(cudaMemcpy(rs.data(), g->g.row_start, rs.size() * 4, cudaMemcpyDeviceToHost));
    return pick_sources_rs(g->g.nnodes, rs.data(), seed, k, out_sources);
}

void gft_graph_free(gft_graph *g)
{
    if (!g) return;
    if (!g->g.wrapped) {
        DeviceScope device_scope(g->g.device);
        if (g->g.row_start) cudaFree(g->g.row_start);
        if (g->g.edge_dst) cudaFree(g->g.edge_dst);
        if (g->g.edge_data) cudaFree(g->g.edge_data);
    }
    if (g->g.edge_dw || g->g.bfs_slots) {
        DeviceScope device_scope(g->g.device);
        if (g->g.edge_dw) cudaFree(g->g.edge_dw);
        if (g->g.bfs_slots) cudaFree(g->g.bfs_slots);
    }
    delete g;
}

}  // extern "C"
