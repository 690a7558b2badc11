// gft_internal.h -- shared definitions of the libgft implementation files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <mutex>
#include <string>
#include <vector>

#include "gft.h"

namespace gft {

// Thread-local message of the last failure (gft_last_error).
void set_error(const char *fmt, ...);
void clear_error();

// Returns `s` after recording a formatted message.
gft_status fail(gft_status s, const char *fmt, ...);

#define GFT_CUDA_TRY(call)                                                                             \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return ::gft::fail(e_ == cudaErrorMemoryAllocation ? GFT_ERR_OOM : GFT_ERR_CUDA,           \
                               "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,       \
                               __LINE__);                                                              \
    } while (0)

#define GFT_TRY(call)                        \
    do {                                     \
        gft_status s_ = (call);              \
        if (s_ != GFT_OK) return s_;         \
    } while (0)

// Device-resident graph.  The arrays are owned unless `wrapped`.
struct DeviceGraph {
    int device = 0;
    uint32_t nnodes = 0, nedges = 0;
    uint32_t *row_start = nullptr;
    uint32_t *edge_dst = nullptr;
    int32_t *edge_data = nullptr;
    bool wrapped = false;
    bool symmetric = false;  // every out-edge is also an in-edge: BFS may run bottom-up
    uint32_t max_degree = 0;  // largest out-degree (set when the graph is created)
    // (edge_dst[e], edge_data[e]) interleaved, built on the first weighted
    // SSSP query and owned by the graph even when the arrays above are
    // wrapped; NULL until then.
    uint2 *edge_dw = nullptr;
    // Small low-degree graphs (the one-CTA thread-per-vertex BFS): one
    // 16-byte slot per vertex with its up to 4 destinations (kBfsSlotNone
    // after them), or kBfsSlotWide first for a vertex of more edges or of
    // a destination outside the graph (read through the CSR).  Built
    // on the first such BFS, owned by the graph; NULL until then.
    uint4 *bfs_slots = nullptr;
};

constexpr uint32_t kBfsSlotNone = 0xFFFFFFFFu;  // never a destination: ids are < nnodes <= 2^32 - 2
constexpr uint32_t kBfsSlotWide = 0xFFFFFFFEu;

// Lazily grown device allocation owned by an engine.
struct Scratch {
    void *ptr = nullptr;
    size_t bytes = 0;
    gft_status ensure(size_t want);
    void release();
};

// Control block of one persistent traversal, zeroed before every launch.
// Counters are triple buffered by iteration (slot = iteration % 3): a slot is
// read during its own iteration, written by the iteration before it and
// cleared by the iteration after it, so no extra grid barrier is needed to
// recycle them.
// Every counter that is hit by atomics sits alone in a 128-byte line.
struct alignas(128) CtlLine {
    unsigned long long v;
    unsigned long long pad[15];
};

struct TraversalCtl {
    CtlLine barrier;       // grid barrier arrival counter (u64)
    CtlLine release;       // grid barrier release flag: last completed episode (u32)
    CtlLine qlen[3];       // frontier (SSSP: near pile) length per iteration slot (u32)
    CtlLine claim[3];      // work-claim cursor per iteration slot (u32)
    CtlLine hub[3];        // (hubs << 32) | hub chunks per iteration slot (u64)
    CtlLine hub_claim[3];  // hub chunk cursor per iteration slot (u32)
    CtlLine far_len[3];    // SSSP far pile length per phase slot (u32)
    CtlLine far_min[3];    // SSSP least distance sent to the far pile per phase slot (u32)
    CtlLine job;           // batch kernel: job claimed by a CTA group (u32)
    CtlLine handoff[3];    // SSSP: loop state left by the CTA that ran small iterations alone
                           // ([0] threshold; [1] done << 63 | phase << 32 | iteration;
                           // [2] the iteration that started the phase)
    // Cold fields, written once per launch.
    unsigned error;        // gft_status recorded by the device (0 = none)
    unsigned error_where;  // barrier episode or queue index of the failure
    unsigned levels;       // BFS levels / SSSP phases
    unsigned iterations;   // grid-synchronous iterations
    unsigned threshold;    // SSSP final bucket threshold
    unsigned pad0;
    unsigned long long edges;    // edges scanned
    unsigned long long pushes;   // frontier pushes
    unsigned long long reached;  // vertices reached (BFS)
};

__host__ __device__ inline unsigned *u32_of(CtlLine &l) { return reinterpret_cast<unsigned *>(&l.v); }

// One query of a batched / served launch (device job table entry).  The
// CTA that runs the job writes the result fields.
struct BatchJob {
    const uint32_t *row_start;
    const uint32_t *edge_dst;
    const int32_t *edge_data;
    int32_t *out;
    uint32_t *parent;
    unsigned long long scratch;  // byte offset of this job's scratch
    uint32_t nnodes, nedges, src, delta;
    uint32_t app;  // 0 BFS, 1 SSSP
    uint32_t hub_cap;
    uint32_t vec_ok;
    uint32_t uniform;  // max degree <= kUniformDegree: static chunks
    uint32_t dir_opt;  // BFS on a graph marked symmetric: direction-optimising
    uint32_t min_lanes;  // resident serving: lanes the job asks for at least (0 or 1: no minimum)
    uint32_t status, error_where, levels, iterations;
    unsigned long long edges;
    unsigned long long t_start, t_end;  // %globaltimer, ns
};

struct LaunchShape {
    int block_threads = 512;
    int blocks = 0;
    int blocks_per_sm = 0;
    int sms = 0;
};

}  // namespace gft

struct gft_graph {
    gft::DeviceGraph g;
    std::mutex pair_mu;  // guards the lazy build of g.edge_dw
};

struct gft_engine {
    int device = 0;
    int sms = 0;
    int cc_major = 0, cc_minor = 0;
    gft::Scratch scratch;    // traversal state (queues, bitmaps, stamps)
    gft::Scratch ctl;        // TraversalCtl
    gft::Scratch aux;        // per-call small buffers (e.g. the source id)
    void *host_ctl = nullptr;  // pinned copy of the TraversalCtl read back after a launch
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Many-query host calls: results go back to the host on this stream while
    // the next query runs; created on first use.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t result_ready[2] = {nullptr, nullptr}, copy_done[2] = {nullptr, nullptr};
    std::mutex mu;
};

namespace gft {
// Resolves tuning defaults and the cooperative grid for a kernel.
gft_status resolve_shape(gft_engine *e, const void *kernel, int block_threads, int blocks_per_sm,
                         size_t dyn_smem, LaunchShape *out);
// Makes `device` current for one entry point and gives the caller's current
// device back when the scope ends, so no call leaves the calling thread on
// another device.
struct DeviceScope {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int device)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        err = cudaSetDevice(device);
    }
    ~DeviceScope()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceScope(const DeviceScope &) = delete;
    DeviceScope &operator=(const DeviceScope &) = delete;
};

// Largest out-degree of a device graph, stored in G.max_degree (one small
// reduction kernel on `stream`, then a wait).
// Builds g->g.edge_dw on `stream` if the graph is weighted and it is not
// there yet, and waits for it; on an allocation failure, or while `stream`
// is being captured, the graph keeps the separate arrays only.
gft_status ensure_edge_pairs(gft_graph *g, cudaStream_t stream);
// Builds g->g.bfs_slots on `stream` (not under stream capture; no room:
// left NULL, and the BFS reads the CSR).
gft_status ensure_bfs_slots(gft_graph *g, cudaStream_t stream);
gft_status graph_degree_stats(DeviceGraph &G, cudaStream_t stream);
// Resident-kernel serving (resident.cu), behind gft_serve_* when
// gft_serve_config.resident is set.
struct ResidentServer;
gft_status resident_open(gft_engine *e, const gft_serve_config &cfg, ResidentServer **out);
const gft_serve_config &resident_config(const ResidentServer *s);
gft_status resident_enqueue(ResidentServer *s, const gft_query &q, size_t scratch_bytes, uint64_t *ticket);
gft_status resident_poll(ResidentServer *s, gft_completion *out, uint32_t max, uint32_t *n, uint32_t wait_us);
void resident_stats(ResidentServer *s, uint64_t *in_flight, uint64_t *launches, uint64_t *queries);
void resident_close(ResidentServer *s);

// Index of the first edge whose destination is >= nnodes (~0 if none).
gft_status check_edges_device(const DeviceGraph &G, cudaStream_t stream, uint64_t *first_bad);
// Graphs whose out-degrees are all at most this many edges have near-equal
// work per frontier vertex, so a frontier is split into one static chunk
// per warp (no shared claim cursor); others are claimed dynamically.
constexpr uint32_t kUniformDegree = 32;
gft_status check_engine_graph(gft_engine *e, const gft_graph *g);
// Runs one BFS (is_sssp false) or SSSP query; caller holds e->mu.
gft_status run_traversal(bool is_sssp, gft_engine *e, const gft_graph *g, uint32_t src, int32_t delta, int32_t *d_out,
                         uint32_t *d_parent, const gft_tuning *tune, cudaStream_t stream, gft_stats *stats);
gft_status reach_stats(const gft_graph *g, const int32_t *d_val, cudaStream_t stream, uint64_t *v_r, uint64_t *e_r);
gft_status pick_sources_rs(uint32_t nnodes, const uint32_t *row_start, uint64_t seed, uint32_t k, uint32_t *out);
// CTA-mode batch kernel plumbing shared by gft_batch_* and the server.
// jobs[0, nbig) run on groups of `group` CTAs (cooperative launch, one
// zeroed TraversalCtl per group in d_gctl), the rest on one CTA each;
// d_cursors holds 2 counters.
gft_status launch_batch_jobs(const BatchJob *d_jobs, unsigned njobs, unsigned nbig, unsigned group,
                             unsigned *d_cursors, char *d_scratch, uint32_t hub_degree, TraversalCtl *d_gctl,
                             int block, int blocks, cudaStream_t stream);
int batch_occupancy(int block);
void fill_batch_job(BatchJob &j, const gft_query &x, uint32_t hub_degree);
size_t batch_job_scratch(uint32_t app, uint32_t nnodes, uint32_t hub_cap);
}  // namespace gft
