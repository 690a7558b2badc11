// ingest.cpp -- .gr files read in parallel chunks, straight into device
// memory (gft_graph_load_gr) or into host arrays (gft_gr_read_chunked).
//
// The reference parses a .gr file with one serial per-edge loop over an
// mmap (CSRGraph::readFromGR, rt/src/csr_graph.cu:152-241) and then uploads
// four arrays with synchronous pageable cudaMemcpy (copy_to_gpu, :250-261),
// edge_data included even when the file has none.  Here the file's three
// sections (u64 end offsets, u32 destinations, u32 weights; layout in
// gft.h) are cut into fixed-size chunks that worker threads take in turn:
//   - a worker preads a chunk into one of its two pinned staging buffers;
//   - an end-offset chunk is narrowed to u32 row_start entries in place and
//     checked (monotone, at most numEdges; the u64 before the chunk is read
//     along with it so that chunk boundaries are checked too);
//   - the chunk goes to the device with cudaMemcpyAsync on the worker's own
//     stream, while the worker reads its next chunk into the other buffer.
// So the disk or page-cache reads of all workers overlap each other and the
// PCIe copies.  Destinations are checked on the device after the copies
// (one pass over edge_dst at HBM speed) instead of on the host, and the
// maximum degree comes from the device row_start.  The host sink runs the
// same chunking and checks into pageable arrays, for tests on machines
// without a GPU.
//
// The pinned staging buffers (kWorkers x 2 x kChunk bytes) are allocated
// by the first device load and kept for later loads; gft_ingest_release
// frees them.
#include <errno.h>
#include <fcntl.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <thread>

#include "gft_internal.h"

namespace gft {
namespace {

constexpr size_t kChunk = (size_t)8 << 20;  // bytes per chunk (a multiple of 8)
constexpr unsigned kWorkers = 8;

enum Section { kIdx = 0, kDst = 1, kW = 2 };

struct Task {
    Section sec;
    uint64_t first;  // first element of the section in this chunk
    uint64_t count;  // elements
};

struct Layout {
    uint64_t nn = 0, ne = 0, size_edge_ty = 0;
    uint64_t off_idx = 32, off_dst = 0, off_w = 0, end = 0;
};

gft_status read_layout(int fd, const char *path, Layout *L)
{
    uint64_t hdr[4];
    if (pread(fd, hdr, sizeof hdr, 0) != (ssize_t)sizeof hdr)
        return fail(GFT_ERR_FORMAT, "%s: truncated header", path);
    if (hdr[0] != 1)
        return fail(GFT_ERR_FORMAT, "%s: version %llu, expected 1", path, (unsigned long long)hdr[0]);
    if (hdr[1] != 0 && hdr[1] != 4)
        return fail(GFT_ERR_FORMAT, "%s: sizeEdgeTy %llu unsupported (0 or 4)", path, (unsigned long long)hdr[1]);
    if (hdr[2] >= 0xFFFFFFFFull || hdr[3] >= 0xFFFFFFFFull)
        return fail(GFT_ERR_FORMAT, "%s: %llu nodes / %llu edges exceed 32-bit ids", path,
                    (unsigned long long)hdr[2], (unsigned long long)hdr[3]);
    L->size_edge_ty = hdr[1];
    L->nn = hdr[2];
    L->ne = hdr[3];
    L->off_dst = L->off_idx + L->nn * 8;
    L->off_w = L->off_dst + L->ne * 4 + ((L->ne & 1) ? 4 : 0);
    L->end = L->size_edge_ty ? L->off_w + L->ne * 4 : L->off_dst + L->ne * 4;
    struct stat st;
    if (fstat(fd, &st) != 0) return fail(GFT_ERR_IO, "%s: fstat failed: %s", path, strerror(errno));
    if ((uint64_t)st.st_size < L->end) return fail(GFT_ERR_FORMAT, "%s: truncated file", path);
    if (!L->nn && L->ne) return fail(GFT_ERR_FORMAT, "%s: edges without nodes", path);
    return GFT_OK;
}

std::vector<Task> make_tasks(const Layout &L)
{
    std::vector<Task> t;
    const uint64_t per_idx = kChunk / 8 - 1, per_u32 = kChunk / 4;  // one u64 of a chunk is the previous offset
    for (uint64_t i = 0; i < L.nn; i += per_idx) t.push_back({kIdx, i, std::min(per_idx, L.nn - i)});
    for (uint64_t i = 0; i < L.ne; i += per_u32) t.push_back({kDst, i, std::min(per_u32, L.ne - i)});
    if (L.size_edge_ty)
        for (uint64_t i = 0; i < L.ne; i += per_u32) t.push_back({kW, i, std::min(per_u32, L.ne - i)});
    return t;
}

bool pread_all(int fd, void *dst, size_t bytes, uint64_t off)
{
    char *p = (char *)dst;
    while (bytes) {
        ssize_t got = pread(fd, p, bytes, (off_t)off);
        if (got <= 0) {
            if (got < 0 && errno == EINTR) continue;
            return false;
        }
        p += got;
        bytes -= (size_t)got;
        off += (uint64_t)got;
    }
    return true;
}

// Reads task t into buf and returns the bytes to deliver (u32 elements),
// narrowing and checking end offsets in place.  buf holds kChunk bytes.
gft_status load_task(int fd, const char *path, const Layout &L, const Task &t, char *buf, size_t *bytes)
{
    if (t.sec == kIdx) {
        // u64 offsets [first - 1, first + count): the one before is the
        // previous chunk's last (0 before the first node).
        uint64_t *w = reinterpret_cast<uint64_t *>(buf);
        const bool head = t.first == 0;
        uint64_t *vals = head ? w + 1 : w;
        if (head) w[0] = 0;
        const uint64_t from = L.off_idx + (t.first - (head ? 0 : 1)) * 8;
        const uint64_t n = t.count + (head ? 0 : 1);
        if (!pread_all(fd, vals, n * 8, from)) return fail(GFT_ERR_FORMAT, "%s: truncated file", path);
        uint32_t *out = reinterpret_cast<uint32_t *>(buf);
        uint64_t prev = w[0];
        for (uint64_t i = 0; i < t.count; i++) {  // out[i] (byte 4i) never passes w[i + 1] (byte 8i + 8)
            const uint64_t x = w[i + 1];
            if (x < prev || x > L.ne)
                return fail(GFT_ERR_FORMAT, "%s: outIdx is not a monotone end-offset array ending at numEdges",
                            path);
            out[i] = (uint32_t)x;
            prev = x;
        }
        if (t.first + t.count == L.nn && prev != L.ne)
            return fail(GFT_ERR_FORMAT, "%s: outIdx is not a monotone end-offset array ending at numEdges", path);
        *bytes = t.count * 4;
        return GFT_OK;
    }
    const uint64_t from = (t.sec == kDst ? L.off_dst : L.off_w) + t.first * 4;
    if (!pread_all(fd, buf, t.count * 4, from)) return fail(GFT_ERR_FORMAT, "%s: truncated file", path);
    *bytes = t.count * 4;
    return GFT_OK;
}

// Destination of task t's delivered bytes in arrays (row_start, dst, w).
char *task_dest(const Task &t, uint32_t *row_start, uint32_t *dst, int32_t *w)
{
    if (t.sec == kIdx) return reinterpret_cast<char *>(row_start + 1 + t.first);
    if (t.sec == kDst) return reinterpret_cast<char *>(dst + t.first);
    return reinterpret_cast<char *>(w + t.first);
}

// Runs every task on up to kWorkers threads; worker(k, tasks) is given the
// tasks one at a time through a shared cursor.  Returns the first failure.
template <class Worker>
gft_status run_workers(const std::vector<Task> &tasks, unsigned nworkers, Worker worker)
{
    std::atomic<size_t> cursor{0};
    std::atomic<int> status{GFT_OK};
    std::vector<std::string> errs(nworkers);
    std::vector<std::thread> th;
    for (unsigned k = 0; k < nworkers; k++)
        th.emplace_back([&, k] {
            gft_status s = worker(k, cursor, status);
            if (s != GFT_OK) {
                errs[k] = gft_last_error();
                int expect = GFT_OK;
                status.compare_exchange_strong(expect, (int)s);
            }
        });
    for (auto &x : th) x.join();
    if (status.load() != GFT_OK) {
        for (auto &e : errs)
            if (!e.empty()) return fail((gft_status)status.load(), "%s", e.c_str());
        return fail((gft_status)status.load(), "ingest failed");
    }
    return GFT_OK;
}

// Pinned staging kept between device loads.
struct Staging {
    std::mutex mu;
    char *buf[kWorkers][2] = {};
    bool ready = false;
    gft_status ensure()
    {
        if (ready) return GFT_OK;
        for (unsigned k = 0; k < kWorkers; k++)
            for (int b = 0; b < 2; b++)
                if (cudaHostAlloc((void **)&buf[k][b], kChunk, cudaHostAllocPortable) != cudaSuccess) {
                    cudaGetLastError();
                    release();
                    return fail(GFT_ERR_OOM, "gft_graph_load_gr: pinned staging allocation failed");
                }
        ready = true;
        return GFT_OK;
    }
    void release()
    {
        for (unsigned k = 0; k < kWorkers; k++)
            for (int b = 0; b < 2; b++) {
                if (buf[k][b]) cudaFreeHost(buf[k][b]);
                buf[k][b] = nullptr;
            }
        ready = false;
    }
};
Staging g_staging;

unsigned workers_for(size_t ntasks)
{
    unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    return (unsigned)std::max<size_t>(1, std::min<size_t>({(size_t)kWorkers, (size_t)hw, ntasks}));
}

struct Fd {
    int fd = -1;
    ~Fd()
    {
        if (fd >= 0) close(fd);
    }
};

}  // namespace
}  // namespace gft

using namespace gft;

extern "C" {

gft_status gft_gr_read_chunked(const char *path, gft_csr *out)
{
    if (!path || !out) return fail(GFT_ERR_INVALID_ARG, "gft_gr_read_chunked: null argument");
    memset(out, 0, sizeof *out);
    Fd f;
    f.fd = open(path, O_RDONLY);
    if (f.fd < 0) return fail(GFT_ERR_IO, "gft_gr_read_chunked: cannot open %s: %s", path, strerror(errno));
    Layout L;
    GFT_TRY(read_layout(f.fd, path, &L));
    out->row_start = (uint32_t *)malloc((L.nn + 1) * 4);
    out->edge_dst = (uint32_t *)malloc(std::max<uint64_t>(L.ne, 1) * 4);
    if (L.size_edge_ty) out->edge_data = (int32_t *)malloc(std::max<uint64_t>(L.ne, 1) * 4);
    if (!out->row_start || !out->edge_dst || (L.size_edge_ty && !out->edge_data)) {
        gft_csr_free(out);
        return fail(GFT_ERR_OOM, "gft_gr_read_chunked: host allocation failed");
    }
    out->row_start[0] = 0;
    const std::vector<Task> tasks = make_tasks(L);
    const unsigned nw = workers_for(tasks.size());
    gft_status s = run_workers(tasks, nw, [&](unsigned, std::atomic<size_t> &cursor, std::atomic<int> &status) {
        std::vector<char> buf(kChunk);
        for (size_t i = cursor++; i < tasks.size() && status.load() == GFT_OK; i = cursor++) {
            size_t bytes = 0;
            GFT_TRY(load_task(f.fd, path, L, tasks[i], buf.data(), &bytes));
            memcpy(task_dest(tasks[i], out->row_start, out->edge_dst, out->edge_data), buf.data(), bytes);
        }
        return GFT_OK;
    });
    if (s == GFT_OK)
        for (uint64_t e = 0; e < L.ne; e++)
            if (out->edge_dst[e] >= L.nn) {
                s = fail(GFT_ERR_FORMAT, "gft_gr_read_chunked: %s: edge %llu has destination %u >= numNodes %llu",
                         path, (unsigned long long)e, out->edge_dst[e], (unsigned long long)L.nn);
                break;
            }
    if (s != GFT_OK) {
        gft_csr_free(out);
        return s;
    }
    out->nnodes = (uint32_t)L.nn;
    out->nedges = (uint32_t)L.ne;
    clear_error();
    return GFT_OK;
}

gft_status gft_graph_load_gr(int device, const char *path, void *stream_, gft_graph **out)
{
    if (!path || !out) return fail(GFT_ERR_INVALID_ARG, "gft_graph_load_gr: null argument");
    *out = nullptr;
    Fd f;
    f.fd = open(path, O_RDONLY);
    if (f.fd < 0) return fail(GFT_ERR_IO, "gft_graph_load_gr: cannot open %s: %s", path, strerror(errno));
    Layout L;
    GFT_TRY(read_layout(f.fd, path, &L));
    DeviceScope device_scope(device);
    GFT_CUDA_TRY(device_scope.err);
    cudaStream_t stream = (cudaStream_t)stream_;
    std::lock_guard<std::mutex> lk(g_staging.mu);
    GFT_TRY(g_staging.ensure());

    gft_graph *g = new gft_graph();
    DeviceGraph &G = g->g;
    G.device = device;
    G.nnodes = (uint32_t)L.nn;
    G.nedges = (uint32_t)L.ne;
    cudaError_t err = cudaMalloc(&G.row_start, (L.nn + 1) * 4);
    if (err == cudaSuccess) err = cudaMalloc(&G.edge_dst, std::max<uint64_t>(L.ne, 1) * 4);
    if (err == cudaSuccess && L.size_edge_ty) err = cudaMalloc(&G.edge_data, std::max<uint64_t>(L.ne, 1) * 4);
    if (err == cudaSuccess) err = cudaMemsetAsync(G.row_start, 0, 4, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) {
        gft_graph_free(g);
        return fail(err == cudaErrorMemoryAllocation ? GFT_ERR_OOM : GFT_ERR_CUDA, "gft_graph_load_gr: %s",
                    cudaGetErrorString(err));
    }
    const std::vector<Task> tasks = make_tasks(L);
    const unsigned nw = workers_for(tasks.size());
    gft_status s = run_workers(tasks, nw, [&](unsigned k, std::atomic<size_t> &cursor, std::atomic<int> &status) {
        DeviceScope ds(device);
        cudaStream_t ws = nullptr;
        cudaEvent_t done[2] = {nullptr, nullptr};
        cudaError_t e = ds.err;
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming);
        gft_status ws_status = GFT_OK;
        bool used[2] = {false, false};
        unsigned b = 0;
        for (size_t i = cursor++; e == cudaSuccess && i < tasks.size() && status.load() == GFT_OK; i = cursor++) {
            char *buf = g_staging.buf[k][b];
            if (used[b]) e = cudaEventSynchronize(done[b]);  // the copy out of this buffer has finished
            if (e != cudaSuccess) break;
            size_t bytes = 0;
            ws_status = load_task(f.fd, path, L, tasks[i], buf, &bytes);
            if (ws_status != GFT_OK) break;
            e = cudaMemcpyAsync(task_dest(tasks[i], G.row_start, G.edge_dst, G.edge_data), buf, bytes,
                                cudaMemcpyHostToDevice, ws);
            if (e == cudaSuccess) e = cudaEventRecord(done[b], ws);
            used[b] = true;
            b ^= 1;
        }
        if (ws) {
            cudaError_t e2 = cudaStreamSynchronize(ws);
            if (e == cudaSuccess) e = e2;
            cudaStreamDestroy(ws);
        }
        for (auto ev : done)
            if (ev) cudaEventDestroy(ev);
        if (ws_status != GFT_OK) return ws_status;
        if (e != cudaSuccess) return fail(GFT_ERR_CUDA, "gft_graph_load_gr: %s", cudaGetErrorString(e));
        return GFT_OK;
    });
    uint64_t bad = ~0ull;
    if (s == GFT_OK) s = check_edges_device(G, stream, &bad);
    if (s == GFT_OK && bad != ~0ull)
        s = fail(GFT_ERR_FORMAT, "gft_graph_load_gr: %s: edge %llu has a destination >= numNodes %llu", path,
                 (unsigned long long)bad, (unsigned long long)L.nn);
    if (s == GFT_OK) s = graph_degree_stats(G, stream);
    if (s != GFT_OK) {
        gft_graph_free(g);
        return s;
    }
    *out = g;
    clear_error();
    return GFT_OK;
}

void gft_ingest_release(void)
{
    std::lock_guard<std::mutex> lk(g_staging.mu);
    g_staging.release();
}

}  // extern "C"
