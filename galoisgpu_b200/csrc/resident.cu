// resident.cu -- serving through one resident persistent kernel
// (gft_serve_* with gft_serve_config.resident = 1).  No counterpart in the
// reference, which runs one query per process (skelapp/skel.cu:139-151).
//
// One cooperative launch keeps every resident CTA on the device.  The CTAs
// are split into lanes of `lane_blocks` consecutive CTAs.  Requests reach
// the kernel through a ring in pinned, device-mapped host memory: the host
// writes a job (BatchJob) into the next ring slot and then publishes the
// ring's tail; nothing is launched per request.
//
// Teams.  The first CTA of an idle lane polls the tail.  When it sees an
// unclaimed job it takes itself out of the idle set (one atomicAnd on a
// bitmask of idle lanes) and claims the job (atomicCAS on the device head
// counter).  It then drafts more idle lanes for the job, as many as are
// idle divided by the jobs still waiting (so an idle server gives a request
// the whole device and a loaded one spreads its lanes over the waiting
// requests), capped by max_lanes_per_request.  Drafting is one atomicAnd on
// the idle mask: a lane is only ever taken by one leader.  The leader
// resets its team control block, copies the job into device memory and
// posts a command in each team lane's mailbox (release store of a sequence
// number).  Every CTA of a drafted lane polls its mailbox, joins, and the
// team runs the traversal as one grid (GridMode over the team's CTAs, the
// team's own bounded barrier), on the leader lane's scratch arena.
// Requests that arrive while others run therefore start as soon as lanes
// are free, their work overlaps on the device, and each runs the same
// traversal bodies as gft_bfs / gft_sssp on a group of CTAs, so every
// result equals the query run alone.
//
// Completion.  After the team's last barrier its first CTA writes the
// result record into the ring's completion slot in mapped host memory and
// publishes it with a system-scope fence and a sequence number; a host
// thread polls those slots.  Each CTA then counts itself out of the team's
// control block (the block is reused only once every member has left it),
// and each lane's first CTA puts its lane back into the idle set.
//
// Ordering.  A request goes through no CUDA stream, so nothing orders it
// with other work: whatever writes its buffers (say, a fill kernel on another
// stream) must have finished before it is enqueued, and its results are
// ready once its completion is polled.  Kernels launched on other streams
// while the resident kernel holds the SMs wait until it ends (it leaves
// after idle_exit_us without work).
//
// Waits.  Every device wait is bounded.  Team barriers time out after the
// engine's barrier limit.  The kernel closes as a whole once every lane has
// been idle for idle_exit_us (or the host asked it to stop and no job
// waits): each lane then takes its own bit out of the idle set, so it is
// never drafted after leaving, and posts its own exit command, which ends
// the lane's waiting CTAs.  The host launches the kernel again when a job
// is published and no kernel is running.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <vector>

#include "frontier.cuh"
#include "gft_internal.h"
#include "job.cuh"

namespace gft {

constexpr unsigned kResMaxLanes = 64;  // one bit per lane in the idle mask
constexpr unsigned long long kGatherNs = 3000000;       // a large job's gather with other claims held back
constexpr unsigned long long kGatherLongNs = 12000000;  // its longest gather while it has under half its width
constexpr unsigned kCmdRun = 1, kCmdExit = 2;

struct alignas(128) ResLaneBox {
    unsigned seq;         // bumped with a release store when the lane gets a command
    unsigned cmd;         // kCmdRun or kCmdExit
    unsigned job;         // ring index of the job (kCmdRun)
    unsigned team_lane;   // the team's first lane: its control block and arena
    unsigned team_lanes;  // lanes in the team
    unsigned rank;        // this lane's place in the team
};

struct alignas(128) ResTeam {
    TraversalCtl ctl;               // barrier and counters of the team's current job
    BatchJob job;                   // device copy of the job
    unsigned long long t_claim;     // %globaltimer when the leader claimed the job
    unsigned index;                 // ring index of the job
    unsigned left;                  // CTAs of the current job that have finished with this block
    unsigned members;               // CTAs of the current job
};

// Device memory.
struct ResDev {
    unsigned long long idle;       // bit per lane that is idle and may be drafted
    unsigned long long last_busy;  // %globaltimer of the last claim or completion (0 at launch)
    unsigned head;                 // next ring index to claim (persists across launches)
    unsigned closing;              // set once: every lane leaves as soon as it is idle
    unsigned gathering;            // leaders gathering lanes for a large job: idle lanes claim nothing meanwhile
    unsigned pad[25];
    ResLaneBox box[kResMaxLanes];
    ResTeam team[kResMaxLanes];
};

// One completion record in mapped host memory.
struct ResDone {
    unsigned long long edges;
    unsigned long long t_claim, t_start, t_end;  // %globaltimer
    unsigned status, levels, iterations, lane, width;
    unsigned seq;  // ring index + 1 once the record is complete
};

// Pinned, device-mapped host memory.
struct ResHost {
    unsigned long long tail;     // jobs [0, tail) are published (host writes)
    unsigned stop;               // host: leave when idle (set by close)
    unsigned pad[29];
    // followed by BatchJob ring[R] and ResDone done[R]
};

namespace dev {

__device__ __forceinline__ unsigned long long ld_acquire_sys_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_acquire_sys_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_sys_u32(unsigned *p, unsigned v)
{
    asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bumps a mailbox sequence number with release semantics.  An atomic, so
// that the writer never works from a stale copy of the number (a plain load
// could hit this SM's L1 while another SM's leader has bumped it since).
__device__ __forceinline__ void bump_release_u32(unsigned *p)
{
    unsigned old;
    asm volatile("atom.release.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(p) : "memory");
}

// Copies a job out of the mapped ring with system-scope loads, so that no
// line this SM cached earlier (a neighbouring slot shares it) is used.
__device__ __forceinline__ void load_ring_job(BatchJob *dst, const BatchJob *src)
{
    static_assert(sizeof(BatchJob) % 8 == 0, "BatchJob is copied in 8-byte words");
    const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
    unsigned long long *d = reinterpret_cast<unsigned long long *>(dst);
#pragma unroll
    for (unsigned i = 0; i < sizeof(BatchJob) / 8; i++) {
        unsigned long long v;
        asm volatile("ld.relaxed.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(s + i) : "memory");
        d[i] = v;
    }
}

// Copies a job from device memory with L2 (coherent) loads: the team's CTAs
// run on SMs whose L1 may still hold an earlier job of the same control
// block.
__device__ __forceinline__ void load_job_cg(BatchJob *dst, const BatchJob *src)
{
    const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
    unsigned long long *d = reinterpret_cast<unsigned long long *>(dst);
#pragma unroll
    for (unsigned i = 0; i < sizeof(BatchJob) / 8; i++) d[i] = __ldcg(s + i);
}

#ifdef GFT_RESIDENT_TRACE
// Diagnostic builds only: (time, lane << 48 | event << 40 | value) records.
__device__ unsigned long long g_rtrace[2 * 65536];
__device__ unsigned g_rtrace_n;
__device__ __forceinline__ void rtrace(unsigned lane, unsigned ev, unsigned long long v)
{
    const unsigned i = atomicAdd(&g_rtrace_n, 1u);
    if (i < 65536) {
        g_rtrace[2 * i] = globaltimer_ns();
        g_rtrace[2 * i + 1] = ((unsigned long long)lane << 48) | ((unsigned long long)ev << 40) | (v & 0xFFFFFFFFFFull);
    }
}
#else
__device__ __forceinline__ void rtrace(unsigned, unsigned, unsigned long long) {}
#endif

struct ResArgs {
    ResDev *S;
    ResHost *H;
    BatchJob *ring;
    ResDone *done;
    unsigned ring_size;
    unsigned lane_ctas;
    unsigned nlanes;
    unsigned max_team_lanes;
    char *arenas;
    unsigned long long arena_bytes;
    uint32_t hub_degree;
    unsigned long long all_lanes;  // the idle mask with every lane in it
    unsigned long long idle_ns;
    unsigned long long timeout_ns;
};

// Resets the fields of a team control block that a traversal reads
// before writing (what batch_kernel resets between the jobs of a group,
// plus the barrier, whose episodes restart at 0 for the new team).
__device__ __forceinline__ void reset_team_ctl(TraversalCtl *c)
{
    c->barrier.v = 0;
    c->release.v = 0;
    for (int k = 0; k < 3; k++) {
        c->qlen[k].v = 0;
        c->claim[k].v = 0;
        c->hub[k].v = 0;
        c->hub_claim[k].v = 0;
        c->far_len[k].v = 0;
        c->far_min[k].v = 0;
        c->handoff[k].v = 0;
    }
    c->job.v = 0;
    c->error = 0;
    c->error_where = 0;
    c->levels = 0;
    c->iterations = 0;
    c->threshold = 0;
    c->edges = 0;
    c->pushes = 0;
    c->reached = 0;
}

// The leader lane has claimed ring index h: draft a team, prepare the
// team's control block and post the commands.  Thread 0 of the lane's
// first CTA.  Returns false when the previous job on this control block
// did not drain in time (the caller then gives up: a fault elsewhere).
__device__ bool lead_team(const ResArgs &a, unsigned lane, unsigned long long h, unsigned long long tail)
{
    ResDev *S = a.S;
    const unsigned long long mine = 1ull << lane;
    ResTeam &T = S->team[lane];
    // The control block is free once every CTA of its last job left it.
    const unsigned long long t0 = globaltimer_ns();
    while (ld_acquire_u32(&T.left) != __ldcg(&T.members)) {
        if (globaltimer_ns() - t0 > a.timeout_ns) {
            // The job cannot run here: report it.
            ResDone &d = a.done[h % a.ring_size];
            d.status = GFT_ERR_TIMEOUT;
            d.t_claim = d.t_start = d.t_end = globaltimer_ns();
            d.lane = lane;
            d.width = 0;
            __threadfence_system();
            st_release_sys_u32(&d.seq, (unsigned)h + 1);
            return false;
        }
    }
    load_ring_job(&T.job, a.ring + h % a.ring_size);  // from mapped host memory
    // Width: the idle lanes shared among the jobs still waiting, but at least
    // the job's own minimum (a large graph runs several times slower per
    // query on a narrow team than alone), as far as idle lanes allow.
    const unsigned long long snap = ld_relaxed_u64(&S->idle) & ~mine;
    const unsigned long long waiting = tail > h + 1 ? tail - (h + 1) : 0;
    const unsigned long long idle_lanes = (unsigned long long)__popcll(snap) + 1;  // with this lane
    unsigned want = (unsigned)(idle_lanes / (waiting + 1));
    want = max(want, T.job.min_lanes);
    want = max(1u, min(want, a.max_team_lanes));
    unsigned long long pick = 0, rest = snap;
    for (unsigned k = 1; k < want && rest; k++) {
        const unsigned long long low = rest & (~rest + 1);
        pick |= low;
        rest &= rest - 1;
    }
    unsigned long long got = 0;
    if (pick) got = atomicAnd(&S->idle, ~pick) & pick;
    // A large job that found too few idle lanes gathers more as other teams
    // finish: on one or two lanes it would run 30-40 times longer than
    // alone.  For up to kGatherNs idle lanes claim no new job meanwhile, so
    // the lanes that other teams free come to it; after that it competes
    // with new claims, and it keeps gathering only while it has fewer than
    // half of its lanes, up to kGatherLongNs.  (Holding claims back for the
    // whole gather cost a quarter of the saturated throughput.)
    const unsigned need = min(max(T.job.min_lanes, 1u), a.max_team_lanes);
    if ((unsigned)__popcll(got) + 1 < need) {
        atomicAdd(&S->gathering, 1u);
        bool holding = true;
        const unsigned long long tg = globaltimer_ns();
        unsigned sleep_ns = 64;
        for (;;) {
            const unsigned have = (unsigned)__popcll(got) + 1;
            const unsigned long long waited = globaltimer_ns() - tg;
            if (holding && (have >= need || waited >= kGatherNs)) {
                atomicSub(&S->gathering, 1u);
                holding = false;
            }
            if (have >= need || (!holding && (2 * have >= need || waited >= kGatherLongNs))) break;
            unsigned long long more = ld_relaxed_u64(&S->idle) & ~mine & ~got;
            unsigned long long take = 0;
            for (unsigned k = __popcll(got) + 1; k < need && more; k++) {
                const unsigned long long low = more & (~more + 1);
                take |= low;
                more &= more - 1;
            }
            if (take) got |= atomicAnd(&S->idle, ~take) & take;
            else {
                __nanosleep(sleep_ns);
                sleep_ns = min(sleep_ns * 2, 1024u);
            }
        }
    }
    const unsigned team_lanes = 1 + __popcll(got);

    reset_team_ctl(&T.ctl);
    T.left = 0;
    T.members = team_lanes * a.lane_ctas;
    T.index = (unsigned)h;
    T.t_claim = globaltimer_ns();
    __threadfence();
    // Commands: this lane is rank 0, the drafted lanes follow in lane order.
    unsigned rank = 0;
    for (unsigned long long m = mine | got; m; m &= m - 1) {
        const unsigned l = __ffsll((long long)m) - 1;
        ResLaneBox &b = S->box[l];
        b.cmd = kCmdRun;
        b.job = (unsigned)h;
        b.team_lane = lane;
        b.team_lanes = team_lanes;
        b.rank = l == lane ? 0u : ++rank;
        bump_release_u32(&b.seq);
    }
    rtrace(lane, 1, (h << 8) | team_lanes);
    return true;
}

// Thread 0 of a lane's first CTA while its lane is idle: claims jobs and
// leads teams until the lane has a command of its own (which it returns
// through the mailbox).  The kernel closes as a whole: once every lane has
// been idle for `idle_ns` (or the host asked to stop and no job waits), the
// first lane to see it sets `closing`, and from then on every lane leaves
// the idle set and posts kCmdExit for itself as soon as it is idle.  (A lane
// leaving on its own would take its share of the device away until the
// whole kernel ended.)
__device__ void lane_leader_idle(const ResArgs &a, unsigned lane, unsigned seen, unsigned long long t_start)
{
    ResDev *S = a.S;
    const unsigned long long mine = 1ull << lane;
    unsigned sleep_ns = 32;
    unsigned long long t_drafted = 0;  // when the lane was first found drafted without its command yet
    for (;;) {
        if (ld_acquire_u32(&S->box[lane].seq) != seen) return;
        if (t_drafted && globaltimer_ns() - t_drafted > a.timeout_ns) {
            // A drafter took this lane but its command never came: leave, so
            // that the wait is bounded (the team's own barrier times out).
            ResLaneBox &b = S->box[lane];
            b.cmd = kCmdExit;
            bump_release_u32(&b.seq);
            rtrace(lane, 6, 0);
            return;
        }
        if (!ld_relaxed_u32(&S->closing)) {
            const unsigned long long tail = ld_acquire_sys_u64(&a.H->tail);
            const unsigned head = ld_relaxed_u32(&S->head);
            if (head < tail && ld_relaxed_u32(&S->gathering) != 0) {
                // A leader gathers lanes for a large job: stay idle to be
                // drafted (bounded: a gather lasts at most kGatherNs).
                __nanosleep(sleep_ns);
                sleep_ns = min(sleep_ns * 2, 256u);
                continue;
            }
            if (head < tail) {
                const unsigned long long old = atomicAnd(&S->idle, ~mine);
                if (!(old & mine)) {  // drafted meanwhile: the mailbox gets the command
                    if (!t_drafted) t_drafted = globaltimer_ns();
                    continue;
                }
                if (atomicCAS(&S->head, head, head + 1) == head) {
                    atomicMax(&S->last_busy, globaltimer_ns());
                    if (!lead_team(a, lane, head, tail)) atomicOr(&S->idle, mine);
                } else {
                    atomicOr(&S->idle, mine);  // another lane claimed it first
                }
                sleep_ns = 32;
                continue;
            }
            const unsigned long long now = globaltimer_ns();
            const unsigned long long last = max(ld_relaxed_u64(&S->last_busy), t_start);
            const bool all_idle = ld_relaxed_u64(&S->idle) == a.all_lanes;
            if (!ld_acquire_sys_u32(&a.H->stop) && !(all_idle && now - last > a.idle_ns)) {
                __nanosleep(sleep_ns);
                sleep_ns = min(sleep_ns * 2, 1024u);
                continue;
            }
            atomicExch(&S->closing, 1u);
        }
        {
            const unsigned long long old = atomicAnd(&S->idle, ~mine);
            if (old & mine) {  // out of the idle set: nobody can draft this lane now
                ResLaneBox &b = S->box[lane];
                b.cmd = kCmdExit;
                bump_release_u32(&b.seq);
                rtrace(lane, 5, 0);
                return;
            }
            if (!t_drafted) t_drafted = globaltimer_ns();
            continue;  // drafted before the kernel began to close: run that job first
        }
    }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) serve_resident(ResArgs a)
{
    constexpr unsigned QB = BLOCK <= 512 ? 256 : kQueueBuf;
    __shared__ uint32_t s_near[BLOCK / 32][QB];
    __shared__ uint32_t s_far[BLOCK / 32][QB];
    __shared__ TravParams s_p;
    __shared__ BatchJob s_jb;
    __shared__ unsigned s_app, s_cmd, s_job, s_team_lane, s_team_lanes, s_rank;
    __shared__ unsigned long long s_t0;
    const unsigned lane = blockIdx.x / a.lane_ctas, r = blockIdx.x % a.lane_ctas;
    if (lane >= a.nlanes) return;
    const unsigned w = threadIdx.x >> 5;
    ResDev *S = a.S;
    // Mailboxes start at 0 in every launch (the host clears them), so a
    // command posted before this CTA started is still seen.
    unsigned seen = 0;
    unsigned long long t_start = 0;
    if (threadIdx.x == 0) t_start = globaltimer_ns();
    for (;;) {
        if (threadIdx.x == 0) {
            if (r == 0) lane_leader_idle(a, lane, seen, t_start);
            // Wait for the lane's command.  Bounded: while the device is
            // busy anywhere, or within idle_ns after, the lane's first CTA
            // posts a command (a job or kCmdExit).
            const unsigned long long t0 = globaltimer_ns();
            unsigned sleep_ns = 32;
            unsigned s = ld_acquire_u32(&S->box[lane].seq);
            while (s == seen) {
                const unsigned long long ref = max(t0, ld_relaxed_u64(&S->last_busy));
                if (globaltimer_ns() - ref > a.idle_ns + a.timeout_ns) break;
                __nanosleep(sleep_ns);
                sleep_ns = min(sleep_ns * 2, 512u);
                s = ld_acquire_u32(&S->box[lane].seq);
            }
            // The mailbox fields through L2 (see load_job_cg).
            ResLaneBox *b = &S->box[lane];
            s_cmd = s == seen ? kCmdExit : __ldcg(&b->cmd);
            if (s == seen) rtrace(lane, 7, r);
            seen = s;
            s_job = __ldcg(&b->job);
            s_team_lane = __ldcg(&b->team_lane);
            s_team_lanes = __ldcg(&b->team_lanes);
            s_rank = __ldcg(&b->rank);
            if (r == 0) rtrace(lane, 2, ((unsigned long long)s_job << 16) | (s_rank << 8) | s_cmd);
        }
        __syncthreads();
        if (s_cmd != kCmdRun) return;
        ResTeam &T = S->team[s_team_lane];
        const unsigned team_ctas = s_team_lanes * a.lane_ctas;
        const unsigned rank_cta = s_rank * a.lane_ctas + r;
        if (threadIdx.x == 0) {
            load_job_cg(&s_jb, &T.job);
            s_p = job_params(s_jb, a.arenas + (size_t)s_team_lane * a.arena_bytes, a.hub_degree, &T.ctl);
            s_app = s_jb.app;
            s_t0 = globaltimer_ns();
        }
        __syncthreads();
        TraversalCtl *ctl = &T.ctl;
        GridSync gs{&ctl->barrier.v, u32_of(ctl->release), &ctl->error, &ctl->error_where, team_ctas, 0,
                    a.timeout_ns};
        const unsigned tid = rank_cta * BLOCK + threadIdx.x;
        GridMode m{gs, ctl, tid, team_ctas * BLOCK, tid / 32, team_ctas * BLOCK / 32};
        if (s_app == 1) sssp_body<GridMode, false, QB>(s_p, m, s_near[w], s_far[w]);
        else bfs_body<GridMode, false, QB>(s_p, m, s_near[w]);
        gs.epoch = m.gs.epoch;
        gs.sync();  // the whole team is done with the traversal
        if (threadIdx.x == 0) {
            if (rank_cta == 0) {
                const unsigned index = __ldcg(&T.index);
                ResDone &d = a.done[index % a.ring_size];
                d.status = ld_relaxed_u32(&ctl->error);
                d.levels = __ldcg(&ctl->levels);
                d.iterations = __ldcg(&ctl->iterations);
                d.edges = __ldcg(&ctl->edges);
                d.t_claim = __ldcg(&T.t_claim);
                d.t_start = s_t0;
                d.t_end = globaltimer_ns();
                d.lane = s_team_lane;
                d.width = s_team_lanes;
                __threadfence_system();  // the record and the results before the sequence number
                st_release_sys_u32(&d.seq, index + 1);
                rtrace(lane, 3, ((unsigned long long)index << 8) | d.status);
            }
            atomicAdd(&T.left, 1u);  // after this the block may be reset for the next job
            if (r == 0) {
                atomicMax(&S->last_busy, globaltimer_ns());
                atomicOr(&S->idle, 1ull << lane);
            }
        }
        __syncthreads();
    }
}

const void *resident_kernel_ptr(int block)
{
    switch (block) {
    case 256: return (const void *)serve_resident<256>;
    case 512: return (const void *)serve_resident<512>;
    case 1024: return (const void *)serve_resident<1024>;
    }
    return nullptr;
}

}  // namespace dev

#ifdef GFT_RESIDENT_TRACE
extern "C" GFT_API int gft_debug_resident_trace(unsigned long long *host, int max_records)
{
    unsigned n = 0;
    if (cudaMemcpyFromSymbol(&n, dev::g_rtrace_n, sizeof n) != cudaSuccess) return -1;
    n = std::min<unsigned>(n, 65536u);
    n = std::min<unsigned>(n, (unsigned)max_records);
    if (n && cudaMemcpyFromSymbol(host, dev::g_rtrace, sizeof(unsigned long long) * 2 * n) != cudaSuccess) return -1;
    return (int)n;
}
#endif

namespace {

// Edges per lane of 8 CTAs up to which a team of that many lanes served a
// query about as efficiently as the whole device did (serving graphs on a
// B200: 2-11x more queries side by side up to 16 M edges, 0.5-0.7x on
// 64 M-edge graphs run on one or two lanes).
constexpr uint64_t kLaneEdges = 8ull << 20;

using Clock = std::chrono::steady_clock;
double now_ms() { return std::chrono::duration<double, std::milli>(Clock::now().time_since_epoch()).count(); }

struct Slot {
    uint64_t ticket = 0;
    double t_arrive = 0;
    bool busy = false;
};

}  // namespace

struct ResidentServer {
    gft_engine *engine = nullptr;
    gft_serve_config cfg{};
    int device = 0;
    unsigned lane_ctas = 0, nlanes = 0, ring = 0;
    ResHost *H = nullptr;        // mapped pinned
    BatchJob *h_ring = nullptr;  // inside H's allocation
    ResDone *h_done = nullptr;
    ResHost *dH = nullptr;       // device views of the same memory
    BatchJob *d_ring = nullptr;
    ResDone *d_done = nullptr;
    ResDev *D = nullptr;
    char *arenas = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    const void *kern = nullptr;
    unsigned long long all_lanes = 0;  // source of the launch's idle-mask copy
    bool running = false;
    uint64_t launches = 0;

    std::mutex mu;
    std::condition_variable cv_done;
    std::vector<Slot> slots;
    std::deque<uint64_t> inflight;  // ring indices in publication order
    std::deque<gft_completion> done;
    uint64_t tail = 0;              // published
    uint64_t claimed = 0;           // the device head when the kernel last ended
    uint64_t next_ticket = 1;
    std::atomic<bool> stop{false};
    std::thread poller;
    gft_status fatal = GFT_OK;
};

namespace {

// Launches the resident kernel (mu held).  All lanes start idle.
gft_status launch_locked(ResidentServer *s)
{
    // idle = every lane, last_busy = 0, closing = gathering = 0; head persists.
    static const unsigned long long zero = 0;
    const unsigned long long all = s->nlanes >= 64 ? ~0ull : ((1ull << s->nlanes) - 1);
    s->all_lanes = all;
    GFT_CUDA_TRY(cudaMemcpyAsync(&s->D->idle, &s->all_lanes, sizeof all, cudaMemcpyHostToDevice, s->stream));
    GFT_CUDA_TRY(cudaMemcpyAsync(&s->D->last_busy, &zero, sizeof zero, cudaMemcpyHostToDevice, s->stream));
    GFT_CUDA_TRY(cudaMemsetAsync(&s->D->closing, 0, 2 * sizeof(unsigned), s->stream));  // closing, gathering
    // Mailboxes and control blocks: nothing of an earlier launch is left in them.
    GFT_CUDA_TRY(cudaMemsetAsync(s->D->box, 0, sizeof(s->D->box), s->stream));
    GFT_CUDA_TRY(cudaMemsetAsync(s->D->team, 0, sizeof(s->D->team), s->stream));
    dev::ResArgs a;
    a.S = s->D;
    a.H = s->dH;
    a.ring = s->d_ring;
    a.done = s->d_done;
    a.ring_size = s->ring;
    a.lane_ctas = s->lane_ctas;
    a.nlanes = s->nlanes;
    a.max_team_lanes = std::max(1u, std::min(s->cfg.max_lanes_per_request, s->nlanes));
    a.arenas = s->arenas;
    a.arena_bytes = s->cfg.lane_arena_bytes;
    a.hub_degree = s->cfg.hub_degree;
    a.all_lanes = all;
    a.idle_ns = (unsigned long long)s->cfg.idle_exit_us * 1000ull;
    a.timeout_ns = 20000ull * 1000000ull;
    void *args[] = {&a};
    GFT_CUDA_TRY(cudaLaunchCooperativeKernel(s->kern, dim3(s->nlanes * s->lane_ctas), dim3(s->cfg.block_threads), args,
                                             0, s->stream));
    GFT_CUDA_TRY(cudaEventRecord(s->ev, s->stream));
    s->running = true;
    s->launches++;
    return GFT_OK;
}

void poll_loop(ResidentServer *s)
{
    cudaSetDevice(s->device);
    unsigned idle_spins = 0;
    for (;;) {
        bool progress = false;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            // Completions, in any order.
            for (auto it = s->inflight.begin(); it != s->inflight.end();) {
                const uint64_t idx = *it;
                volatile ResDone *d = &s->h_done[idx % s->ring];
                if (d->seq != (unsigned)(idx + 1)) {
                    ++it;
                    continue;
                }
                std::atomic_thread_fence(std::memory_order_acquire);
                Slot &sl = s->slots[idx % s->ring];
                gft_completion c;
                memset(&c, 0, sizeof c);
                c.ticket = sl.ticket;
                c.status = (gft_status)d->status;
                c.latency_ms = now_ms() - sl.t_arrive;
                const double dev_ms = (double)(d->t_end - d->t_start) * 1e-6;
                c.queue_ms = std::max(0.0, c.latency_ms - dev_ms);
                c.lane = d->lane + 1;
                c.batch_size = 1;
                c.width = d->width;
                c.levels = d->levels;
                c.edges_scanned = d->edges;
                s->done.push_back(c);
                sl.busy = false;
                it = s->inflight.erase(it);
                progress = true;
            }
            if (progress) s->cv_done.notify_all();
            // The kernel leaves when idle; launch it again for work it has
            // not claimed (its head counter is exact once it has ended).
            if (s->running) {
                const cudaError_t e = cudaEventQuery(s->ev);
                if (e != cudaErrorNotReady) {
                    s->running = false;
                    if (e != cudaSuccess && s->fatal == GFT_OK) s->fatal = GFT_ERR_CUDA;
                    unsigned head = 0;
                    if (e == cudaSuccess &&
                        (cudaMemcpyAsync(&head, &s->D->head, sizeof head, cudaMemcpyDeviceToHost, s->stream) !=
                             cudaSuccess ||
                         cudaStreamSynchronize(s->stream) != cudaSuccess))
                        s->fatal = GFT_ERR_CUDA;
                    s->claimed = head;
                }
            }
            if (!s->running && s->fatal == GFT_OK && s->claimed < s->tail) {
                if (launch_locked(s) != GFT_OK) s->fatal = GFT_ERR_CUDA;
                progress = true;
            }
            if (s->stop && s->inflight.empty() && !s->running) break;
            if (s->fatal != GFT_OK && !s->running) {
                // Nothing will complete the rest: report them.
                for (uint64_t idx : s->inflight) {
                    Slot &sl = s->slots[idx % s->ring];
                    gft_completion c;
                    memset(&c, 0, sizeof c);
                    c.ticket = sl.ticket;
                    c.status = s->fatal;
                    c.latency_ms = now_ms() - sl.t_arrive;
                    s->done.push_back(c);
                    sl.busy = false;
                }
                s->inflight.clear();
                s->cv_done.notify_all();
                if (s->stop) break;
            }
        }
        if (progress) {
            idle_spins = 0;
        } else if (++idle_spins > 64) {
            std::this_thread::sleep_for(std::chrono::microseconds(5));
        }
    }
}

}  // namespace

gft_status resident_open(gft_engine *e, const gft_serve_config &cfg, ResidentServer **out)
{
    *out = nullptr;
    const void *kern = dev::resident_kernel_ptr((int)cfg.block_threads);
    if (!kern) return fail(GFT_ERR_INVALID_ARG, "gft_serve_open: resident mode needs block_threads 256, 512 or 1024");
    DeviceScope device_scope(e->device);
    GFT_CUDA_TRY(device_scope.err);
    int occ = 0;
    GFT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, (int)cfg.block_threads, 0));
    if (occ <= 0) return fail(GFT_ERR_NOT_SUPPORTED, "gft_serve_open: the resident kernel cannot be resident");
    ResidentServer *s = new ResidentServer();
    s->engine = e;
    s->cfg = cfg;
    s->device = e->device;
    s->kern = kern;
    const unsigned resident = (unsigned)(occ * e->sms);
    s->lane_ctas = std::max(1u, std::min(cfg.lane_blocks ? cfg.lane_blocks : 8u, resident));
    s->nlanes = std::min(kResMaxLanes, resident / s->lane_ctas);
    if (cfg.lanes) s->nlanes = std::min(s->nlanes, cfg.lanes);
    s->cfg.lanes = s->nlanes;
    s->cfg.lane_blocks = s->lane_ctas;
    if (s->cfg.max_lanes_per_request == 0 || s->cfg.max_lanes_per_request > s->nlanes)
        s->cfg.max_lanes_per_request = s->nlanes;
    if (s->cfg.idle_exit_us == 0) s->cfg.idle_exit_us = 2000;
    s->ring = std::max(16u, std::min(cfg.queue_capacity, 1u << 16));
    const size_t hbytes = sizeof(ResHost) + sizeof(BatchJob) * s->ring + sizeof(ResDone) * s->ring;
    cudaError_t err = cudaHostAlloc((void **)&s->H, hbytes, cudaHostAllocMapped | cudaHostAllocPortable);
    if (err == cudaSuccess) {
        memset(s->H, 0, hbytes);
        s->h_ring = reinterpret_cast<BatchJob *>(s->H + 1);
        s->h_done = reinterpret_cast<ResDone *>(s->h_ring + s->ring);
        err = cudaHostGetDevicePointer((void **)&s->dH, s->H, 0);
    }
    if (err == cudaSuccess) {
        s->d_ring = reinterpret_cast<BatchJob *>(s->dH + 1);
        s->d_done = reinterpret_cast<ResDone *>(s->d_ring + s->ring);
        err = cudaMalloc(&s->D, sizeof(ResDev));
    }
    if (err == cudaSuccess) err = cudaMemset(s->D, 0, sizeof(ResDev));
    if (err == cudaSuccess) err = cudaMalloc(&s->arenas, (size_t)s->nlanes * cfg.lane_arena_bytes);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming);
    if (err != cudaSuccess) {
        gft_status st = fail(err == cudaErrorMemoryAllocation ? GFT_ERR_OOM : GFT_ERR_CUDA, "gft_serve_open: %s",
                             cudaGetErrorString(err));
        resident_close(s);
        return st;
    }
    s->slots.resize(s->ring);
    s->poller = std::thread(poll_loop, s);
    *out = s;
    return GFT_OK;
}

const gft_serve_config &resident_config(const ResidentServer *s) { return s->cfg; }

gft_status resident_enqueue(ResidentServer *s, const gft_query &q, size_t scratch_bytes, uint64_t *ticket)
{
    if (scratch_bytes > s->cfg.lane_arena_bytes)
        return fail(GFT_ERR_OOM, "gft_serve_enqueue: the query's scratch exceeds a lane arena (%zu bytes)",
                    s->cfg.lane_arena_bytes);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(GFT_ERR_INVALID_ARG, "gft_serve_enqueue: server is closing");
    if (s->fatal != GFT_OK) return fail(s->fatal, "gft_serve_enqueue: the resident kernel failed");
    const uint64_t idx = s->tail;
    Slot &sl = s->slots[idx % s->ring];
    if (sl.busy) return fail(GFT_ERR_BUSY, "gft_serve_enqueue: queue full (%u requests in flight)", s->ring);
    BatchJob &j = s->h_ring[idx % s->ring];
    fill_batch_job(j, q, s->cfg.hub_degree);
    j.scratch = 0;  // at the start of the team leader's arena
    // About kLaneEdges edges per lane: below that a narrow team serves the
    // query as efficiently as the whole device; above, it slows down.
    const uint64_t e = q.graph->g.nedges;
    j.min_lanes = (uint32_t)std::min<uint64_t>(s->nlanes, std::max<uint64_t>(1, (e + kLaneEdges - 1) / kLaneEdges));
    sl.busy = true;
    sl.ticket = s->next_ticket++;
    sl.t_arrive = now_ms();
    s->inflight.push_back(idx);
    s->tail = idx + 1;
    std::atomic_thread_fence(std::memory_order_release);
    *(volatile unsigned long long *)&s->H->tail = s->tail;
    if (!s->running) {
        gft_status st = launch_locked(s);
        if (st != GFT_OK) s->fatal = st;
    }
    *ticket = sl.ticket;
    return GFT_OK;
}

gft_status resident_poll(ResidentServer *s, gft_completion *out, uint32_t max, uint32_t *n, uint32_t wait_us)
{
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

void resident_stats(ResidentServer *s, uint64_t *in_flight, uint64_t *launches, uint64_t *queries)
{
    std::lock_guard<std::mutex> lk(s->mu);
    if (in_flight) *in_flight = s->inflight.size();
    if (launches) *launches = s->launches;
    if (queries) *queries = s->tail;
}

void resident_close(ResidentServer *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        if (s->H) *(volatile unsigned *)&s->H->stop = 1u;
    }
    if (s->poller.joinable()) s->poller.join();
    DeviceScope device_scope(s->device);
    if (s->stream) {
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
    }
    if (s->ev) cudaEventDestroy(s->ev);
    if (s->arenas) cudaFree(s->arenas);
    if (s->D) cudaFree(s->D);
    if (s->H) cudaFreeHost(s->H);
    delete s;
}

}  // namespace gft
