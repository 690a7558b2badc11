// serve.cpp -- request loop over resident graphs with continuous batching
// (gft_serve_*).  No counterpart in the reference, which runs one query per
// process (skelapp/skel.cu:139-151).
//
// The device's resident CTAs are split into lanes of `lane_blocks` CTAs,
// each with its own stream, job table and scratch arena; launches on
// different lanes fit side by side, so their work overlaps on the device.
// A dispatcher thread hands work to free lanes in arrival order:
//   * a heavy request (a graph of at least `group_min_nodes` vertices,
//     except BFS on a graph whose average degree is below `sparse_degree`
//     when that is non-zero) runs alone as ONE CTA group spanning w free
//     lanes, w = free lanes / heavy requests waiting (at least 1): an idle
//     server gives a request the whole device, so its latency is that of
//     the query run alone, and under load requests share the device lane by
//     lane, which overlaps the latency-bound levels of many traversals;
//   * light requests are packed into one micro-batch on one lane, one CTA
//     each.
// A request that arrives while others run starts as soon as a lane and
// arena space are free, and a long request never holds up a launch of short
// ones.  Admission is against memory: a request is taken only if its scratch
// fits in a lane's arena, and refused at enqueue if it could never fit.
// Latency is measured from enqueue to the moment the dispatcher sees the
// request's launch complete.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

#include "gft_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double now_ms()
{
    return std::chrono::duration<double, std::milli>(Clock::now().time_since_epoch()).count();
}

struct Req {
    gft_query q;
    double t_arrive = 0, t_start = 0;
    uint32_t lane = 0, batch = 0, width = 1;
};

struct Lane {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    gft::BatchJob *h_jobs = nullptr;  // pinned
    gft::BatchJob *d_jobs = nullptr;
    unsigned *d_cursor = nullptr;     // 2 counters
    char *d_arena = nullptr;
    gft::TraversalCtl *d_gctl = nullptr;  // one per CTA group
    std::vector<uint64_t> tickets;        // in job-table order
    bool busy = false;
    int owner = -1;  // lent to the launch on lane `owner`
};

}  // namespace

struct gft_server {
    gft_engine *engine = nullptr;
    gft_serve_config cfg{};
    int occ = 0;
    std::vector<Lane> lanes;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> pending;       // requests for the shared lanes
    std::deque<uint64_t> wide_pending;  // requests for the wide pool
    std::unordered_map<uint64_t, Req> reqs;
    std::deque<gft_completion> done;
    uint64_t next_ticket = 1;
    uint64_t in_flight = 0;
    std::atomic<bool> stop{false};
    std::thread dispatcher;
    uint64_t launched_batches = 0, launched_queries = 0;
    gft::ResidentServer *rs = nullptr;  // resident mode: everything below is its job
};

using namespace gft;

static size_t req_scratch(const gft_query &q, uint32_t hub)
{
    const DeviceGraph &G = q.graph->g;
    uint32_t hub_cap = (uint32_t)std::min<uint64_t>(G.nnodes, (uint64_t)G.nedges / hub + 1);
    return (batch_job_scratch(q.app, G.nnodes, hub_cap) + 255) & ~(size_t)255;
}

static bool runs_on_group(const gft_server *s, const gft_query &q)
{
    const DeviceGraph &G = q.graph->g;
    if (s->cfg.group_blocks <= 1 || G.nnodes < s->cfg.group_min_nodes) return false;
    const bool sparse = (uint64_t)G.nedges < (uint64_t)s->cfg.sparse_degree * G.nnodes;
    return !(q.app == 0 && sparse);
}

// SSSP on a large skewed-degree graph (R-MAT-like): such a query moves so
// much memory that it runs no faster side by side than alone, and it takes
// many times longer on a narrow group.  It runs on the wide pool: lanes
// [0, wide_lanes), one request at a time.
static bool is_wide(const gft_server *s, const gft_query &q)
{
    const DeviceGraph &G = q.graph->g;
    return s->cfg.wide_lanes > 0 && q.app == 1 && G.max_degree > kUniformDegree && G.nedges >= s->cfg.wide_min_edges;
}

static void complete(gft_server *s, uint64_t t, gft_status st, uint32_t levels, uint64_t edges, double t_done)
{
    auto it = s->reqs.find(t);
    if (it == s->reqs.end()) return;
    gft_completion c;
    memset(&c, 0, sizeof c);
    c.ticket = t;
    c.status = st;
    c.latency_ms = t_done - it->second.t_arrive;
    c.queue_ms = it->second.t_start - it->second.t_arrive;
    c.lane = it->second.lane;
    c.batch_size = it->second.batch;
    c.width = it->second.width;
    c.levels = levels;
    c.edges_scanned = edges;
    s->done.push_back(c);
    s->reqs.erase(it);
    s->in_flight--;
}

// Launches one micro-batch on lane `li`: group queries first in the job table.
// A heavy request (big, one entry) runs as one group over `width` lanes:
// lane `li` and the lanes in `lent`, which stay busy until `li` completes.
static void launch_lane(gft_server *s, uint32_t li, std::vector<uint64_t> &big, std::vector<uint64_t> &small,
                        const std::vector<uint32_t> &lent)
{
    Lane &l = s->lanes[li];
    const uint32_t n = (uint32_t)(big.size() + small.size());
    const uint32_t width = 1 + (uint32_t)lent.size();
    const uint32_t G = big.empty() ? s->cfg.group_blocks : width * s->cfg.lane_blocks;
    const double t = now_ms();
    size_t off = 0;
    l.tickets.clear();
    for (auto *cls : {&big, &small})
        for (auto tk : *cls) {
            Req &r = s->reqs[tk];
            BatchJob &j = l.h_jobs[l.tickets.size()];
            fill_batch_job(j, r.q, s->cfg.hub_degree);
            j.scratch = off;
            off += req_scratch(r.q, s->cfg.hub_degree);
            r.t_start = t;
            r.lane = li + 1;
            r.batch = n;
            r.width = width;
            l.tickets.push_back(tk);
        }
    const uint32_t nbig = (uint32_t)big.size();
    const int blocks = nbig ? (int)G : std::min((int)s->cfg.lane_blocks, (int)small.size());
    cudaError_t e = cudaMemcpyAsync(l.d_jobs, l.h_jobs, sizeof(BatchJob) * n, cudaMemcpyHostToDevice, l.stream);
    if (e == cudaSuccess && nbig) e = cudaMemsetAsync(l.d_gctl, 0, sizeof(TraversalCtl), l.stream);
    gft_status st = e == cudaSuccess ? launch_batch_jobs(l.d_jobs, n, nbig, G, l.d_cursor, l.d_arena,
                                                         s->cfg.hub_degree, l.d_gctl, (int)s->cfg.block_threads,
                                                         blocks, l.stream)
                                     : GFT_ERR_CUDA;
    if (st == GFT_OK)
        e = cudaMemcpyAsync(l.h_jobs, l.d_jobs, sizeof(BatchJob) * n, cudaMemcpyDeviceToHost, l.stream);
    if (st == GFT_OK && e == cudaSuccess) e = cudaEventRecord(l.done, l.stream);
    if (st != GFT_OK || e != cudaSuccess) {
        for (auto tk : l.tickets) complete(s, tk, st != GFT_OK ? st : GFT_ERR_CUDA, 0, 0, now_ms());
        l.tickets.clear();
        return;
    }
    l.busy = true;
    for (uint32_t b : lent) {
        s->lanes[b].busy = true;
        s->lanes[b].owner = (int)li;
    }
    s->launched_batches++;
    s->launched_queries += n;
}

static void dispatcher_loop(gft_server *s)
{
    cudaSetDevice(s->engine->device);
    while (true) {
        bool idle = true;
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->stop && s->pending.empty() && s->wide_pending.empty()) {
            bool any_busy = false;
            for (auto &l : s->lanes) any_busy |= l.busy;
            if (!any_busy) break;
        }
        // Completions; a finished launch also returns the lanes lent to it.
        for (uint32_t li = 0; li < s->lanes.size(); li++) {
            Lane &l = s->lanes[li];
            if (!l.busy || l.owner >= 0) continue;
            cudaError_t q = cudaEventQuery(l.done);
            if (q == cudaErrorNotReady) continue;
            const double t = now_ms();
            for (size_t k = 0; k < l.tickets.size(); k++) {
                const BatchJob &j = l.h_jobs[k];
                gft_status st = q != cudaSuccess ? GFT_ERR_CUDA : (gft_status)j.status;
                complete(s, l.tickets[k], st, j.levels, j.edges, t);
            }
            l.tickets.clear();
            l.busy = false;
            for (auto &b : s->lanes)
                if (b.owner == (int)li) {
                    b.owner = -1;
                    b.busy = false;
                }
            idle = false;
        }
        if (!s->done.empty()) s->cv_done.notify_all();
        // Dispatch, in arrival order: a heavy request runs alone on a fair
        // share of the free lanes; a run of light requests shares one lane.
        // The wide pool takes the oldest wide request once all its lanes are
        // free, plus every free shared lane when no other request waits.
        const uint32_t W = s->cfg.wide_lanes;
        if (!s->wide_pending.empty()) {
            bool pool_free = true;
            for (uint32_t li = 0; li < W; li++) pool_free &= !s->lanes[li].busy;
            if (pool_free) {
                std::vector<uint64_t> big{s->wide_pending.front()}, none;
                s->wide_pending.pop_front();
                std::vector<uint32_t> lent;
                for (uint32_t li = 1; li < W; li++) lent.push_back(li);
                if (s->pending.empty())
                    for (uint32_t li = W; li < s->lanes.size(); li++)
                        if (!s->lanes[li].busy) lent.push_back(li);
                launch_lane(s, 0, big, none, lent);
                idle = false;
            }
        }
        std::vector<uint32_t> free_lanes;
        for (uint32_t li = W; li < s->lanes.size(); li++)
            if (!s->lanes[li].busy) free_lanes.push_back(li);
        size_t fi = 0;
        while (fi < free_lanes.size() && !s->pending.empty()) {
            std::vector<uint64_t> big, small;
            std::vector<uint32_t> lent;
            const uint32_t li = free_lanes[fi++];
            if (runs_on_group(s, s->reqs[s->pending.front()].q)) {
                // Heavy requests waiting, counted over a bounded window.
                size_t heavy = 0, seen = 0;
                for (auto it = s->pending.begin(); it != s->pending.end() && seen < 4 * s->lanes.size(); ++it, ++seen)
                    heavy += runs_on_group(s, s->reqs[*it].q);
                const size_t avail = free_lanes.size() - (fi - 1);
                size_t w = std::max<size_t>(1, avail / std::max<size_t>(1, heavy));
                w = std::min<size_t>(w, s->cfg.max_lanes_per_request);
                while (lent.size() + 1 < w) lent.push_back(free_lanes[fi++]);
                big.push_back(s->pending.front());
                s->pending.pop_front();
            } else {
                size_t used = 0;
                while (!s->pending.empty() && small.size() < s->cfg.max_batch) {
                    const uint64_t tk = s->pending.front();
                    const Req &r = s->reqs[tk];
                    if (runs_on_group(s, r.q)) break;
                    const size_t need = req_scratch(r.q, s->cfg.hub_degree);
                    if (used + need > s->cfg.lane_arena_bytes) break;  // wait for arena space
                    used += need;
                    small.push_back(tk);
                    s->pending.pop_front();
                }
            }
            if (big.empty() && small.empty()) break;
            launch_lane(s, li, big, small, lent);
            idle = false;
        }
        if (idle) s->cv_work.wait_for(lk, std::chrono::microseconds(20));
    }
}

extern "C" {

gft_status gft_serve_config_default(gft_serve_config *cfg)
{
    if (!cfg) return fail(GFT_ERR_INVALID_ARG, "gft_serve_config_default: null argument");
    memset(cfg, 0, sizeof *cfg);
    cfg->lanes = 0;  // resident CTAs / group_blocks at open
    cfg->max_batch = 256;
    cfg->lane_arena_bytes = (size_t)768 << 20;
    cfg->block_threads = 512;
    cfg->hub_degree = 256;
    cfg->lane_blocks = 0;  // group_blocks
    cfg->group_blocks = 16;
    cfg->group_min_nodes = 1u << 18;
    cfg->sparse_degree = 0;
    cfg->queue_capacity = 1u << 20;
    cfg->max_lanes_per_request = 0;  // all lanes
    cfg->wide_lanes = GFT_SERVE_AUTO;  // 4/9 of the lanes when there are at least 4
    cfg->wide_min_edges = 1u << 25;
    return GFT_OK;
}

gft_status gft_serve_open(gft_engine *e, const gft_serve_config *cfg_in, gft_server **out)
{
    if (!e || !out) return fail(GFT_ERR_INVALID_ARG, "gft_serve_open: null argument");
    *out = nullptr;
    gft_serve_config cfg;
    gft_serve_config_default(&cfg);
    if (cfg_in) cfg = *cfg_in;
    if (cfg.max_batch == 0 || cfg.lane_arena_bytes == 0 || cfg.queue_capacity == 0)
        return fail(GFT_ERR_INVALID_ARG, "gft_serve_open: arena, batch and queue sizes must be > 0");
    if (cfg.hub_degree < 32) cfg.hub_degree = 32;
    if (cfg.resident) {
        gft::ResidentServer *rs = nullptr;
        GFT_TRY(gft::resident_open(e, cfg, &rs));
        gft_server *s = new gft_server();
        s->engine = e;
        s->rs = rs;
        s->cfg = gft::resident_config(rs);
        *out = s;
        return GFT_OK;
    }
    gft_server *s = new gft_server();
    s->engine = e;
    s->cfg = cfg;
    s->occ = batch_occupancy((int)cfg.block_threads);
    if (s->occ <= 0) {
        delete s;
        return fail(GFT_ERR_INVALID_ARG, "gft_serve_open: block_threads must be 128, 256, 512 or 1024");
    }
    const int resident = s->occ * e->sms;
    s->cfg.group_blocks = std::max(1u, std::min<uint32_t>(s->cfg.group_blocks, (uint32_t)resident));
    if (s->cfg.lane_blocks == 0) s->cfg.lane_blocks = s->cfg.group_blocks;
    s->cfg.lane_blocks = std::max(s->cfg.group_blocks, std::min<uint32_t>(s->cfg.lane_blocks, (uint32_t)resident));
    if (s->cfg.lanes == 0) s->cfg.lanes = std::max(1u, (uint32_t)resident / s->cfg.lane_blocks);
    if (s->cfg.lanes * s->cfg.lane_blocks > (uint32_t)resident)
        s->cfg.lanes = std::max(1u, (uint32_t)resident / s->cfg.lane_blocks);
    if (s->cfg.max_lanes_per_request == 0 || s->cfg.max_lanes_per_request > s->cfg.lanes)
        s->cfg.max_lanes_per_request = s->cfg.lanes;
    if (s->cfg.wide_lanes == GFT_SERVE_AUTO) s->cfg.wide_lanes = s->cfg.lanes >= 4 ? (s->cfg.lanes * 4 + 8) / 9 : 0;
    if (s->cfg.wide_lanes >= s->cfg.lanes) s->cfg.wide_lanes = s->cfg.lanes - 1;
    DeviceScope device_scope(e->device);
    cudaError_t err = device_scope.err;
    s->lanes.resize(s->cfg.lanes);
    for (auto &l : s->lanes) {
        if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming);
        if (err == cudaSuccess) err = cudaMallocHost(&l.h_jobs, sizeof(BatchJob) * s->cfg.max_batch);
        if (err == cudaSuccess) err = cudaMalloc(&l.d_jobs, sizeof(BatchJob) * s->cfg.max_batch);
        if (err == cudaSuccess) err = cudaMalloc(&l.d_cursor, 2 * sizeof(unsigned));
        if (err == cudaSuccess) err = cudaMalloc(&l.d_arena, s->cfg.lane_arena_bytes);
        if (err == cudaSuccess) err = cudaMalloc(&l.d_gctl, sizeof(TraversalCtl));
    }
    if (err != cudaSuccess) {
        gft_status st = fail(err == cudaErrorMemoryAllocation ? GFT_ERR_OOM : GFT_ERR_CUDA, "gft_serve_open: %s",
                             cudaGetErrorString(err));
        gft_serve_close(s);
        return st;
    }
    s->dispatcher = std::thread(dispatcher_loop, s);
    *out = s;
    return GFT_OK;
}

gft_status gft_serve_enqueue(gft_server *s, const gft_query *q, uint64_t *ticket)
{
    if (!s || !q || !ticket) return fail(GFT_ERR_INVALID_ARG, "gft_serve_enqueue: null argument");
    if (!q->graph || !q->d_out || q->app > 1 || (q->app == 1 && q->delta <= 0) || q->src >= q->graph->g.nnodes ||
        q->graph->g.device != s->engine->device)
        return fail(GFT_ERR_INVALID_ARG, "gft_serve_enqueue: invalid query");
    if (s->rs) return resident_enqueue(s->rs, *q, req_scratch(*q, s->cfg.hub_degree), ticket);
    if (req_scratch(*q, s->cfg.hub_degree) > s->cfg.lane_arena_bytes)
        return fail(GFT_ERR_OOM, "gft_serve_enqueue: the query's scratch exceeds a lane arena (%zu bytes)",
                    s->cfg.lane_arena_bytes);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(GFT_ERR_INVALID_ARG, "gft_serve_enqueue: server is closing");
    if (s->in_flight >= s->cfg.queue_capacity) return fail(GFT_ERR_BUSY, "gft_serve_enqueue: queue full");
    const uint64_t t = s->next_ticket++;
    Req r;
    r.q = *q;
    r.t_arrive = now_ms();
    s->reqs.emplace(t, r);
    s->in_flight++;
    (is_wide(s, *q) ? s->wide_pending : s->pending).push_back(t);
    s->cv_work.notify_one();
    *ticket = t;
    return GFT_OK;
}

gft_status gft_serve_poll(gft_server *s, gft_completion *out, uint32_t max, uint32_t *n, uint32_t wait_us)
{
    if (!s || !n || (max && !out)) return fail(GFT_ERR_INVALID_ARG, "gft_serve_poll: null argument");
    if (s->rs) return resident_poll(s->rs, out, max, n, wait_us);
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_us)
        s->cv_done.wait_for(lk, std::chrono::microseconds(wait_us), [&] { return !s->done.empty(); });
    uint32_t k = 0;
    while (k < max && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    *n = k;
    return GFT_OK;
}

gft_status gft_serve_stats(gft_server *s, uint64_t *in_flight, uint64_t *batches, uint64_t *queries)
{
    if (!s) return fail(GFT_ERR_INVALID_ARG, "gft_serve_stats: server is NULL");
    if (s->rs) {
        resident_stats(s->rs, in_flight, batches, queries);
        return GFT_OK;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (in_flight) *in_flight = s->in_flight;
    if (batches) *batches = s->launched_batches;
    if (queries) *queries = s->launched_queries;
    return GFT_OK;
}

gft_status gft_serve_close(gft_server *s)
{
    if (!s) return GFT_OK;
    if (s->rs) {
        resident_close(s->rs);
        delete s;
        return GFT_OK;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    DeviceScope device_scope(s->engine->device);
    for (auto &l : s->lanes) {
        if (l.stream) cudaStreamSynchronize(l.stream);
        if (l.stream) cudaStreamDestroy(l.stream);
        if (l.done) cudaEventDestroy(l.done);
        if (l.h_jobs) cudaFreeHost(l.h_jobs);
        if (l.d_jobs) cudaFree(l.d_jobs);
        if (l.d_cursor) cudaFree(l.d_cursor);
        if (l.d_arena) cudaFree(l.d_arena);
        if (l.d_gctl) cudaFree(l.d_gctl);
    }
    delete s;
    return GFT_OK;
}

}  // extern "C"
