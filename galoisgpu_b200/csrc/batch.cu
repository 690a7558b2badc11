// batch.cu -- many BFS / SSSP queries in one persistent launch, replayed as
// a captured CUDA graph (gft_batch_*).
//
// The reference runs one query per process and one persistent grid per
// query (skelapp/skel.cu:139-151, apps/sssp/kernel.cu:426-454).  Most queries
// of a mixed batch are small or high-diameter and cannot keep 148 SMs busy,
// so one launch runs them side by side in two phases:
//   phase 1: queries on graphs of at least `group_min_nodes` vertices run on
//            groups of `group` consecutive CTAs (GridMode over the group,
//            control block in global memory, one per group); the launch is
//            cooperative whenever there are such queries, so a group is
//            co-resident and its bounded barrier cannot wait on a CTA that
//            never starts;
//   phase 2: the rest run on ONE CTA each (CtaMode: control block in shared
//            memory, __syncthreads as the barrier, no grid-wide atomics).
// Both phases take queries from a device job table, largest first (longest
// processing time first keeps the tail short), and a CTA whose group finds
// no large query left moves on to phase 2 at once.
//
// The job table is copied from pinned host memory by the first node of the
// captured graph, so changing a query's source between replays needs no
// re-capture.
#include <string.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "frontier.cuh"
#include "gft_internal.h"
#include "job.cuh"

namespace gft {
namespace dev {

// jobs[0, nbig) are large queries, run in phase 1 by groups of `group`
// CTAs (consecutive blockIdx; the launch is cooperative whenever nbig > 0,
// so a group is co-resident); jobs[nbig, njobs) run in phase 2, one CTA
// each.  A CTA joins phase 2 as soon as its group finds no large job left,
// so large and small queries overlap.  cursors[0] / cursors[1] hand out
// small / large jobs; gctl holds one zeroed control block per group.
// Per-warp push buffers: 256 entries up to 512 threads per CTA (32 KB of
// the CTA's static shared memory), 128 at 1024 threads.
template <int BLOCK>
constexpr unsigned kBatchQueueBuf = BLOCK <= 512 ? 256 : kQueueBuf;

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)
    batch_kernel(BatchJob *jobs, unsigned njobs, unsigned nbig, unsigned group, unsigned *cursors, char *scratch,
                 uint32_t hub_degree, TraversalCtl *gctl, unsigned long long timeout_ns)
{
    __shared__ TraversalCtl s_ctl;
    constexpr unsigned QB = kBatchQueueBuf<BLOCK>;
    __shared__ uint32_t s_near[BLOCK / 32][QB];
    __shared__ uint32_t s_far[BLOCK / 32][QB];
    __shared__ unsigned s_job;
    // The running job's parameters live in shared memory: the traversal
    // bodies read them by reference, which keeps them out of registers.
    __shared__ TravParams s_p;
    __shared__ unsigned s_app;
    __shared__ unsigned long long s_t0;
    const unsigned w = threadIdx.x >> 5;

    // Phase 1: large jobs on CTA groups.
    const unsigned ngroups = (nbig > 0 && group > 1) ? gridDim.x / group : 0;
    const unsigned g = blockIdx.x / max(group, 1u), rank = blockIdx.x % max(group, 1u);
    if (g < ngroups) {
        TraversalCtl *ctl = gctl + g;
        GridSync gs{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, group, 0, timeout_ns};
        for (;;) {
            if (rank == 0 && threadIdx.x == 0) *u32_of(ctl->job) = atomicAdd(&cursors[1], 1u);
            if (!gs.sync()) break;
            const unsigned j = ld_relaxed_u32(u32_of(ctl->job));
            if (j >= nbig) break;
            if (rank == 0) {  // per-job state; the barrier lines and the job line persist
                for (int k = 0; k < 3; k++) {
                    if (threadIdx.x == 32 * k + 0) ctl->qlen[k].v = 0;
                    if (threadIdx.x == 32 * k + 1) ctl->claim[k].v = 0;
                    if (threadIdx.x == 32 * k + 2) ctl->hub[k].v = 0;
                    if (threadIdx.x == 32 * k + 3) ctl->hub_claim[k].v = 0;
                    if (threadIdx.x == 32 * k + 4) ctl->far_len[k].v = 0;
                    if (threadIdx.x == 32 * k + 5) ctl->far_min[k].v = 0;
                }
                if (threadIdx.x == 128) {
                    ctl->levels = 0;
                    ctl->iterations = 0;
                    ctl->threshold = 0;
                    ctl->edges = 0;
                    ctl->pushes = 0;
                    ctl->reached = 0;
                }
            }
            if (!gs.sync()) break;
            if (threadIdx.x == 0) {
                const BatchJob jb = jobs[j];
                s_p = job_params(jb, scratch, hub_degree, ctl);
                s_app = jb.app;
                s_t0 = globaltimer_ns();
            }
            __syncthreads();
            const unsigned long long t0 = s_t0;
            const unsigned tid = rank * BLOCK + threadIdx.x;
            GridMode m{gs, ctl, tid, group * BLOCK, tid / 32, group * BLOCK / 32};
            if (s_app == 1) sssp_body<GridMode, false, QB>(s_p, m, s_near[w], s_far[w]);
            else bfs_body<GridMode, false, QB>(s_p, m, s_near[w]);
            gs.epoch = m.gs.epoch;
            const bool ok = gs.sync();
            if (rank == 0 && threadIdx.x == 0) {
                TraversalCtl c;
                c.error = ld_relaxed_u32(&ctl->error);
                c.error_where = ctl->error_where;
                c.levels = ctl->levels;
                c.iterations = ctl->iterations;
                c.edges = ctl->edges;
                write_result(jobs[j], c, t0);
            }
            if (!ok) break;  // an error aborts this group's phase 1
        }
    }

    // Phase 2: small jobs, one CTA each (control block in shared memory).
    for (;;) {
        if (threadIdx.x == 0) s_job = nbig + atomicAdd(&cursors[0], 1u);
        for (unsigned i = threadIdx.x; i < sizeof(TraversalCtl) / 4; i += BLOCK)
            reinterpret_cast<unsigned *>(&s_ctl)[i] = 0;
        __syncthreads();
        const unsigned j = s_job;
        if (j >= njobs) return;
        if (threadIdx.x == 0) {
            const BatchJob jb = jobs[j];
            s_p = job_params(jb, scratch, hub_degree, &s_ctl);
            s_app = jb.app;
            s_t0 = globaltimer_ns();
        }
        __syncthreads();
        const unsigned long long t0 = s_t0;
        CtaMode m{&s_ctl, threadIdx.x, BLOCK, w, BLOCK / 32, 0};
        if (s_app == 1) sssp_body<CtaMode, false, QB>(s_p, m, s_near[w], s_far[w]);
        else bfs_body<CtaMode, false, QB>(s_p, m, s_near[w]);
        __syncthreads();
        if (threadIdx.x == 0) write_result(jobs[j], s_ctl, t0);
        __syncthreads();
    }
}

}  // namespace dev

static const void *batch_kernel_ptr(int block)
{
    switch (block) {
    case 128: return (const void *)dev::batch_kernel<128>;
    case 256: return (const void *)dev::batch_kernel<256>;
    case 512: return (const void *)dev::batch_kernel<512>;
    case 1024: return (const void *)dev::batch_kernel<1024>;
    }
    return nullptr;
}

gft_status launch_batch_jobs(const BatchJob *d_jobs, unsigned njobs, unsigned nbig, unsigned group,
                             unsigned *d_cursors, char *d_scratch, uint32_t hub_degree, TraversalCtl *d_gctl,
                             int block, int blocks, cudaStream_t stream)
{
    const void *kern = batch_kernel_ptr(block);
    if (!kern) return fail(GFT_ERR_INVALID_ARG, "batch: block_threads must be 128, 256, 512 or 1024");
    BatchJob *dj = const_cast<BatchJob *>(d_jobs);
    unsigned nj = njobs, nb = nbig, grp = group;
    unsigned *cur = d_cursors;
    char *scr = d_scratch;
    uint32_t hub = hub_degree;
    TraversalCtl *gc = d_gctl;
    unsigned long long timeout = 20000ull * 1000000ull;
    void *args[] = {&dj, &nj, &nb, &grp, &cur, &scr, &hub, &gc, &timeout};
    GFT_CUDA_TRY(cudaMemsetAsync(d_cursors, 0, 2 * sizeof(unsigned), stream));
    cudaLaunchConfig_t lc;
    memset(&lc, 0, sizeof lc);
    lc.gridDim = dim3(blocks);
    lc.blockDim = dim3(block);
    lc.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = nbig > 0 && group > 1 ? 1 : 0;
    lc.attrs = attr;
    lc.numAttrs = 1;
    GFT_CUDA_TRY(cudaLaunchKernelExC(&lc, kern, args));
    return GFT_OK;
}

int batch_occupancy(int block)
{
    const void *kern = batch_kernel_ptr(block);
    if (!kern) return 0;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, block, 0) != cudaSuccess) return 0;
    return occ;
}

// Fills a job record for one query (scratch offset left to the caller).
void fill_batch_job(BatchJob &j, const gft_query &x, uint32_t hub_degree)
{
    const DeviceGraph &G = x.graph->g;
    memset(&j, 0, sizeof j);
    j.row_start = G.row_start;
    j.edge_dst = G.edge_dst;
    j.edge_data = G.edge_data;
    j.out = x.d_out;
    j.parent = x.app == 0 ? x.d_parent : nullptr;
    j.nnodes = G.nnodes;
    j.nedges = G.nedges;
    j.src = x.src;
    j.delta = x.app == 1 ? (uint32_t)x.delta : 0;
    j.app = x.app;
    j.hub_cap = (uint32_t)std::min<uint64_t>(G.nnodes, (uint64_t)G.nedges / hub_degree + 1);
    j.vec_ok = ((uintptr_t)G.edge_dst % 16 == 0) && (!G.edge_data || (uintptr_t)G.edge_data % 16 == 0);
    j.uniform = G.max_degree <= kUniformDegree;
    j.dir_opt = x.app == 0 && G.symmetric;
}

// Bytes of scratch one CTA-mode job needs (layout of batch_kernel).
size_t batch_job_scratch(uint32_t app, uint32_t nnodes, uint32_t hub_cap)
{
    const size_t qbytes = ((size_t)nnodes * 4 + 255) & ~(size_t)255;
    const size_t hbytes = ((size_t)hub_cap * 8 + 255) & ~(size_t)255;
    if (app == 1) return 5 * qbytes + hbytes;  // 4 queues, pile stamps (distances in place in `out`)
    const size_t vbytes = ((size_t)((nnodes + 31) / 32) * 4 + 255) & ~(size_t)255;
    return 2 * qbytes + vbytes + hbytes;
}

}  // namespace gft

struct gft_batch {
    gft_engine *engine = nullptr;
    uint32_t n = 0;
    uint32_t nbig = 0;
    uint32_t group = 8;
    uint32_t group_min_nodes = 1u << 18;
    int block = 512;
    int blocks = 0;
    uint32_t hub_degree = 256;
    gft::TraversalCtl *d_gctl = nullptr;
    size_t gctl_bytes = 0;
    std::vector<uint32_t> order;      // job slot -> caller's query index
    gft::BatchJob *h_jobs = nullptr;  // pinned, caller-owned inputs: the graph's first node uploads it
    gft::BatchJob *h_res = nullptr;   // pinned, the job table as the last launch left it
    gft::BatchJob *d_jobs = nullptr;
    bool in_flight = false;           // submitted and not yet waited for
    unsigned *d_cursor = nullptr;
    char *d_scratch = nullptr;
    size_t scratch_bytes = 0;
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t last_stream = nullptr;
};

using namespace gft;


extern "C" {

void gft_batch_destroy(gft_batch *b)
{
    if (!b) return;
    DeviceScope device_scope(b->engine ? b->engine->device : 0);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->h_jobs) cudaFreeHost(b->h_jobs);
    if (b->h_res) cudaFreeHost(b->h_res);
    if (b->d_jobs) cudaFree(b->d_jobs);
    if (b->d_cursor) cudaFree(b->d_cursor);
    if (b->d_scratch) cudaFree(b->d_scratch);
    if (b->d_gctl) cudaFree(b->d_gctl);
    delete b;
}

gft_status gft_batch_create(gft_engine *e, const gft_query *q, uint32_t n, const gft_tuning *tune, gft_batch **out)
{
    if (!e || !out || (n && !q)) return fail(GFT_ERR_INVALID_ARG, "gft_batch_create: null argument");
    *out = nullptr;
    if (n == 0) return fail(GFT_ERR_INVALID_ARG, "gft_batch_create: empty batch");
    gft_batch *b = new gft_batch();
    b->engine = e;
    b->n = n;
    if (tune && tune->block_threads) b->block = (int)tune->block_threads;
    if (tune && tune->hub_degree) b->hub_degree = std::max<uint32_t>(32, tune->hub_degree);
    if (tune && tune->group_blocks) b->group = tune->group_blocks;
    if (tune && tune->group_min_nodes) b->group_min_nodes = tune->group_min_nodes;
    const void *kern = batch_kernel_ptr(b->block);
    if (!kern) {
        delete b;
        return fail(GFT_ERR_INVALID_ARG, "gft_batch_create: block_threads must be 128, 256, 512 or 1024");
    }
    // Validate and order: largest estimated work first.
    b->order.resize(n);
    std::iota(b->order.begin(), b->order.end(), 0u);
    for (uint32_t i = 0; i < n; i++) {
        const gft_query &x = q[i];
        if (!x.graph || !x.d_out || x.app > 1 || (x.app == 1 && x.delta <= 0) || x.src >= x.graph->g.nnodes ||
            x.graph->g.device != e->device) {
            gft_batch_destroy(b);
            return fail(GFT_ERR_INVALID_ARG, "gft_batch_create: query %u is invalid", i);
        }
    }
    // Large queries (run on CTA groups) first, then the rest; each class
    // largest first.
    auto big = [&](uint32_t i) { return b->group > 1 && q[i].graph->g.nnodes >= b->group_min_nodes; };
    std::stable_sort(b->order.begin(), b->order.end(), [&](uint32_t a, uint32_t c) {
        if (big(a) != big(c)) return big(a);
        const DeviceGraph &ga = q[a].graph->g, &gc = q[c].graph->g;
        return (uint64_t)ga.nedges + ga.nnodes > (uint64_t)gc.nedges + gc.nnodes;
    });
    b->nbig = 0;
    for (uint32_t i = 0; i < n; i++) b->nbig += big(i);
    DeviceScope device_scope(e->device);
    cudaError_t err = device_scope.err;
    if (err == cudaSuccess) err = cudaMallocHost(&b->h_jobs, sizeof(BatchJob) * n);
    if (err == cudaSuccess) err = cudaMallocHost(&b->h_res, sizeof(BatchJob) * n);
    if (err != cudaSuccess) {
        gft_batch_destroy(b);
        return fail(GFT_ERR_OOM, "gft_batch_create: %s", cudaGetErrorString(err));
    }
    size_t off = 0;
    for (uint32_t s = 0; s < n; s++) {
        BatchJob &j = b->h_jobs[s];
        fill_batch_job(j, q[b->order[s]], b->hub_degree);
        j.scratch = off;
        off += batch_job_scratch(j.app, j.nnodes, j.hub_cap);
    }
    b->scratch_bytes = off;
    int occ = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, b->block, 0);
    if (err == cudaSuccess && occ <= 0) err = cudaErrorInvalidConfiguration;
    uint32_t bps = (tune && tune->blocks_per_sm) ? tune->blocks_per_sm : (uint32_t)occ;
    b->blocks = std::max(1, std::min<int>(occ, (int)bps)) * e->sms;
    if (b->nbig && (int)b->group > b->blocks) b->group = (uint32_t)b->blocks;
    const uint32_t ngroups = b->nbig ? (uint32_t)b->blocks / std::max(1u, b->group) : 0;
    b->gctl_bytes = std::max<size_t>(1, ngroups) * sizeof(TraversalCtl);
    if (err == cudaSuccess) err = cudaMalloc(&b->d_jobs, sizeof(BatchJob) * n);
    if (err == cudaSuccess) err = cudaMalloc(&b->d_cursor, 2 * sizeof(unsigned));
    if (err == cudaSuccess) err = cudaMalloc(&b->d_gctl, b->gctl_bytes);
    if (err == cudaSuccess) err = cudaMalloc(&b->d_scratch, std::max<size_t>(off, 256));
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreate(&b->ev0);
    if (err == cudaSuccess) err = cudaEventCreate(&b->ev1);
    if (err != cudaSuccess) {
        gft_status s = fail(err == cudaErrorMemoryAllocation ? GFT_ERR_OOM : GFT_ERR_CUDA,
                            "gft_batch_create: %s (scratch %zu bytes)", cudaGetErrorString(err), off);
        gft_batch_destroy(b);
        return s;
    }
    // Capture: job table upload, cursor reset, persistent batch kernel.
    cudaStream_t cs = b->capture_stream;
    err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
        cudaMemcpyAsync(b->d_jobs, b->h_jobs, sizeof(BatchJob) * n, cudaMemcpyHostToDevice, cs);
        cudaMemsetAsync(b->d_gctl, 0, b->gctl_bytes, cs);
        gft_status ls = launch_batch_jobs(b->d_jobs, n, b->nbig, b->group, b->d_cursor, b->d_scratch, b->hub_degree,
                                          b->d_gctl, b->block, b->blocks, cs);
        cudaGraph_t gph = nullptr;
        err = cudaStreamEndCapture(cs, &gph);
        b->graph = gph;
        if (err == cudaSuccess && ls != GFT_OK) err = cudaErrorInvalidValue;
    }
    if (err == cudaSuccess) err = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (err != cudaSuccess) {
        gft_status s = fail(GFT_ERR_CUDA, "gft_batch_create: graph capture failed: %s", cudaGetErrorString(err));
        gft_batch_destroy(b);
        return s;
    }
    *out = b;
    return GFT_OK;
}

gft_status gft_batch_set_source(gft_batch *b, uint32_t query, uint32_t src)
{
    if (!b || query >= b->n) return fail(GFT_ERR_INVALID_ARG, "gft_batch_set_source: bad batch or index");
    // The replay uploads h_jobs when its first node runs, which may be after
    // submit returns: changing it before the wait could reach the running batch.
    if (b->in_flight) return fail(GFT_ERR_BUSY, "gft_batch_set_source: a submit is in flight; call gft_batch_wait first");
    for (uint32_t s = 0; s < b->n; s++)
        if (b->order[s] == query) {
            if (src >= b->h_jobs[s].nnodes) return fail(GFT_ERR_INVALID_ARG, "gft_batch_set_source: source out of range");
            b->h_jobs[s].src = src;
            return GFT_OK;
        }
    return fail(GFT_ERR_INVALID_ARG, "gft_batch_set_source: query not found");
}

gft_status gft_batch_submit(gft_batch *b, void *stream)
{
    if (!b) return fail(GFT_ERR_INVALID_ARG, "gft_batch_submit: batch is NULL");
    DeviceScope device_scope(b->engine->device);
    GFT_CUDA_TRY(device_scope.err);
    cudaStream_t s = (cudaStream_t)stream;
    GFT_CUDA_TRY(cudaEventRecord(b->ev0, s));
    GFT_CUDA_TRY(cudaGraphLaunch(b->exec, s));
    b->in_flight = true;
    GFT_CUDA_TRY(cudaEventRecord(b->ev1, s));
    b->last_stream = s;
    return GFT_OK;
}

gft_status gft_batch_wait(gft_batch *b, gft_query *q, gft_batch_stats *st)
{
    if (!b) return fail(GFT_ERR_INVALID_ARG, "gft_batch_wait: batch is NULL");
    DeviceScope device_scope(b->engine->device);
    GFT_CUDA_TRY(device_scope.err);
    cudaStream_t s = b->last_stream;
    GFT_CUDA_TRY(cudaMemcpyAsync(b->h_res, b->d_jobs, sizeof(BatchJob) * b->n, cudaMemcpyDeviceToHost, s));
    GFT_CUDA_TRY(cudaStreamSynchronize(s));
    b->in_flight = false;
    gft_status worst = GFT_OK;
    unsigned long long t_first = ~0ull, t_last = 0;
    uint64_t edges = 0;
    for (uint32_t k = 0; k < b->n; k++) {
        const BatchJob &j = b->h_res[k];
        if (j.status && worst == GFT_OK) worst = (gft_status)j.status;
        t_first = std::min(t_first, j.t_start);
        t_last = std::max(t_last, j.t_end);
        edges += j.edges;
        if (q) {
            gft_query &x = q[b->order[k]];
            x.status = (gft_status)j.status;
            x.levels = j.levels;
            x.iterations = j.iterations;
            x.edges_scanned = j.edges;
            x.device_ms = (float)((j.t_end - j.t_start) * 1e-6);
        }
    }
    if (st) {
        float ms = 0;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        st->queries = b->n;
        st->launch_ms = ms;
        st->busy_ms = (float)((t_last - t_first) * 1e-6);
        st->edges_scanned = edges;
        st->grid_blocks = (uint32_t)b->blocks;
        st->block_threads = (uint32_t)b->block;
        st->scratch_bytes = b->scratch_bytes;
    }
    if (worst != GFT_OK) return fail(worst, "gft_batch_wait: a query reported %s", gft_status_string(worst));
    return GFT_OK;
}

}  // extern "C"
