// gen_device.cu -- builds the seeded synthetic graphs of gen_common.h
// directly in device memory (gft_graph_generate).  Produces the same CSR as
// the host builders in gen_host.cpp: every undirected pair becomes two keys
// (u << b) | v, the keys are radix sorted, duplicates and self loops dropped,
// and rows delimited by binary search.  This is graph construction, not the
// traversal hot path; the sort and the unique selection use CUB from the
// CUDA toolkit.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include "gen_common.h"
#include "gft_internal.h"

namespace gft {
namespace dev {

struct GenSpec {
    uint32_t kind;  // 0 grid, 1 road, 2 rmat
    uint32_t rows, cols, nnodes;
    uint64_t n_grid;       // undirected grid edges (grid / road)
    uint32_t delete_ppm;
    uint64_t dkey, skey, rkey, wkey;
    uint32_t scale;
    RmatThresholds t;
    Perm perm;
    uint32_t bits;         // key = (u << bits) | v
};

__device__ __forceinline__ bool gen_pair(const GenSpec &s, uint64_t i, uint32_t *u, uint32_t *v)
{
    if (s.kind == 0) {
        if (s.rows == 1 || s.cols == 1) {
            *u = (uint32_t)i;
            *v = (uint32_t)i + 1;
            return true;
        }
        grid_edge_endpoints(s.rows, s.cols, i, u, v);
        return true;
    }
    if (s.kind == 1) {
        if (i < s.n_grid) {
            if (!road_keep(s.dkey, i, s.delete_ppm)) return false;
            grid_edge_endpoints(s.rows, s.rows, i, u, v);
            return true;
        }
        road_shortcut(s.skey, i - s.n_grid, s.nnodes, u, v);
        return true;
    }
    uint32_t a, b;
    rmat_sample(s.rkey, i, s.scale, s.t.ta, s.t.tab, s.t.tabc, &a, &b);
    *u = perm_apply(s.perm, a);
    *v = perm_apply(s.perm, b);
    return true;
}

__global__ void gen_keys(GenSpec s, uint64_t npairs, unsigned long long *keys)
{
    const unsigned long long sentinel = (unsigned long long)s.nnodes << s.bits;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npairs;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t u, v;
        bool ok = gen_pair(s, i, &u, &v) && u != v;
        keys[2 * i] = ok ? (((unsigned long long)u << s.bits) | v) : sentinel;
        keys[2 * i + 1] = ok ? (((unsigned long long)v << s.bits) | u) : sentinel;
    }
}

// Unique sorted keys -> edge_dst, edge_data, row_start.
__global__ void keys_to_csr(GenSpec s, const unsigned long long *keys, uint64_t ne, uint32_t *row_start,
                            uint32_t *edge_dst, int32_t *edge_data, uint32_t max_weight)
{
    const unsigned long long vmask = (1ull << s.bits) - 1;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < ne; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t u = (uint32_t)(keys[j] >> s.bits), v = (uint32_t)(keys[j] & vmask);
        edge_dst[j] = v;
        if (edge_data) edge_data[j] = (int32_t)pair_weight(s.wkey, u, v, max_weight);
        const uint32_t prev = j ? (uint32_t)(keys[j - 1] >> s.bits) : 0xFFFFFFFFu;
        // Rows (prev, u] start here (prev = -1 for the first edge).
        for (uint32_t x = prev + 1; x <= u; x++) row_start[x] = (uint32_t)j;
        if (j == ne - 1)
            for (uint32_t x = u + 1; x <= s.nnodes; x++) row_start[x] = (uint32_t)ne;
    }
}

__global__ void fill_row_start(uint32_t *row_start, uint32_t n, uint32_t value)
{
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x <= n; x += gridDim.x * blockDim.x) row_start[x] = value;
}

}  // namespace dev
}  // namespace gft

using namespace gft;

static uint32_t bits_for(uint32_t x)
{
    uint32_t b = 0;
    while (b < 32 && (1ull << b) <= x) b++;
    return b;
}

extern "C" gft_status gft_graph_generate(int device, const gft_gen_params *p, void *stream_, gft_graph **out)
{
    if (!p || !out) return fail(GFT_ERR_INVALID_ARG, "gft_graph_generate: null argument");
    *out = nullptr;
    cudaStream_t stream = (cudaStream_t)stream_;
    dev::GenSpec s{};
    s.kind = p->kind;
    uint64_t npairs = 0;
    uint32_t max_weight = p->max_weight;
    if (p->kind == 0) {
        if (!p->rows || !p->cols || (uint64_t)p->rows * p->cols >= 0xFFFFFFFFull)
            return fail(GFT_ERR_INVALID_ARG, "gft_graph_generate: bad grid size");
        s.rows = p->rows;
        s.cols = p->cols;
        s.nnodes = p->rows * p->cols;
        npairs = (p->rows == 1 || p->cols == 1) ? (uint64_t)s.nnodes - 1 : grid_undirected_edges(p->rows, p->cols);
    } else if (p->kind == 1) {
        if (p->rows < 2 || (uint64_t)p->rows * p->rows >= 0xFFFFFFFFull || p->delete_ppm > 1000000)
            return fail(GFT_ERR_INVALID_ARG, "gft_graph_generate: bad road parameters");
        s.rows = s.cols = p->rows;
        s.nnodes = p->rows * p->rows;
        s.n_grid = grid_undirected_edges(p->rows, p->rows);
        s.delete_ppm = p->delete_ppm;
        s.dkey = stream_key(p->seed, kStreamDelete);
        s.skey = stream_key(p->seed, kStreamShortcut);
        npairs = s.n_grid + road_shortcuts(p->rows, p->shortcut_ppm);
    } else if (p->kind == 2) {
        if (!p->scale || p->scale > 31 || !p->edge_factor || (uint64_t)p->a_q32 + p->b_q32 + p->c_q32 > 0xFFFFFFFFull)
            return fail(GFT_ERR_INVALID_ARG, "gft_graph_generate: bad rmat parameters");
        s.scale = p->scale;
        s.nnodes = 1u << p->scale;
        s.rkey = stream_key(p->seed, kStreamRmat);
        s.t = rmat_thresholds(p->a_q32, p->b_q32, p->c_q32);
        s.perm = make_perm(p->seed, p->scale);
        npairs = (uint64_t)p->edge_factor << p->scale;
    } else {
        return fail(GFT_ERR_INVALID_ARG, "gft_graph_generate: unknown kind %u", p->kind);
    }
    s.wkey = stream_key(p->seed, kStreamWeight);
    s.bits = bits_for(s.nnodes);
    if (2 * s.bits > 64) return fail(GFT_ERR_INVALID_ARG, "gft_graph_generate: graph too large");
    const uint64_t nkeys = 2 * npairs;
    if (nkeys >= 0x7FFFFFFFull) return fail(GFT_ERR_INVALID_ARG, "gft_graph_generate: too many edges for one sort");

    DeviceScope device_scope(device);
    GFT_CUDA_TRY(device_scope.err);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned long long *k0 = nullptr, *k1 = nullptr;
    int *d_nsel = nullptr;
    void *tmp = nullptr;
    size_t tmp_sort = 0, tmp_sel = 0;
    gft_graph *g = nullptr;
    gft_status st = GFT_OK;
    int nsel = 0;
    const int end_bit = (int)(2 * s.bits);
    cudaError_t err = cudaMalloc(&k0, std::max<uint64_t>(nkeys, 1) * 8);
    if (err == cudaSuccess) err = cudaMalloc(&k1, std::max<uint64_t>(nkeys, 1) * 8);
    if (err == cudaSuccess) err = cudaMalloc(&d_nsel, sizeof(int));
    if (err == cudaSuccess)
        err = cub::DeviceRadixSort::SortKeys(nullptr, tmp_sort, k0, k1, (int)nkeys, 0, end_bit, stream);
    if (err == cudaSuccess) err = cub::DeviceSelect::Unique(nullptr, tmp_sel, k1, k0, d_nsel, (int)nkeys, stream);
    if (err == cudaSuccess) err = cudaMalloc(&tmp, std::max(tmp_sort, tmp_sel));
    if (err == cudaSuccess && nkeys) {
        dev::gen_keys<<<sms * 8, 256, 0, stream>>>(s, npairs, k0);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess && nkeys)
        err = cub::DeviceRadixSort::SortKeys(tmp, tmp_sort, k0, k1, (int)nkeys, 0, end_bit, stream);
    if (err == cudaSuccess && nkeys)
        err = cub::DeviceSelect::Unique(tmp, tmp_sel, k1, k0, d_nsel, (int)nkeys, stream);
    if (err == cudaSuccess && nkeys) err = cudaMemcpyAsync(&nsel, d_nsel, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err == cudaSuccess) {
        // The sentinel (u == nnodes) sorts last; it is present iff some pair was dropped.
        uint64_t ne = (uint64_t)nsel;
        if (ne) {
            unsigned long long last = 0;
            err = cudaMemcpy(&last, k0 + ne - 1, 8, cudaMemcpyDeviceToHost);
            if (err == cudaSuccess && (last >> s.bits) == s.nnodes) ne--;
        }
        if (err == cudaSuccess) {
            g = new gft_graph();
            g->g.device = device;
            g->g.symmetric = true;  // every generator emits both directions of each edge
            g->g.nnodes = s.nnodes;
            g->g.nedges = (uint32_t)ne;
            err = cudaMalloc(&g->g.row_start, ((size_t)s.nnodes + 1) * 4);
            if (err == cudaSuccess) err = cudaMalloc(&g->g.edge_dst, std::max<uint64_t>(ne, 1) * 4);
            if (err == cudaSuccess && max_weight) err = cudaMalloc(&g->g.edge_data, std::max<uint64_t>(ne, 1) * 4);
            if (err == cudaSuccess) {
                if (ne) {
                    dev::keys_to_csr<<<sms * 8, 256, 0, stream>>>(s, k0, ne, g->g.row_start, g->g.edge_dst,
                                                                    g->g.edge_data, max_weight);
                } else {
                    dev::fill_row_start<<<sms, 256, 0, stream>>>(g->g.row_start, s.nnodes, 0);
                }
                err = cudaGetLastError();
            }
            if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
        }
    }
    if (err != cudaSuccess)
        st = fail(err == cudaErrorMemoryAllocation ? GFT_ERR_OOM : GFT_ERR_CUDA, "gft_graph_generate: %s",
                  cudaGetErrorString(err));
    if (st == GFT_OK && g) st = graph_degree_stats(g->g, stream);
    cudaFree(k0);
    cudaFree(k1);
    cudaFree(d_nsel);
    cudaFree(tmp);
    if (st != GFT_OK) {
        gft_graph_free(g);
        return st;
    }
    *out = g;
    return GFT_OK;
}
