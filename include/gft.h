/*
 * gft.h -- C ABI of the B200 frontier-traversal engine (libgft.so).
 *
 * The engine replaces the data-driven worklist BFS and SSSP of LonestarGPU
 * v3 (apps/bfs, apps/sssp).  Every entry point below names the reference
 * interface it stands in for (file:line within the reference project).
 *
 * Conventions
 *   - Plain C types only: pointers, sizes, integers.  No exceptions cross
 *     this boundary and nothing calls exit(): every function returns a
 *     gft_status (0 = GFT_OK); gft_last_error() gives a message for the
 *     calling thread's last failure.
 *   - Vertex and edge ids are uint32 (the reference's index_type,
 *     rt/include/csr_graph.h:22); levels and distances are int32 with
 *     GFT_INF = INT_MAX for unreached vertices (apps/bfs/kernel.cu:16).
 *   - Output buffers are caller-owned.  Functions that take "d_" pointers
 *     want device memory; "h_" pointers are host memory (pinned host memory
 *     gives the fastest copies).
 *   - Work is enqueued on the caller's stream (NULL = legacy default
 *     stream).  Passing a gft_stats* makes the call wait for the stream and
 *     fill the statistics; passing NULL keeps the call asynchronous.
 *   - A gft_engine owns the traversal scratch (frontier queues, visited
 *     bitmaps, counters) for one device; calls on one engine must not
 *     overlap in time.  Use one engine per host thread / stream for
 *     concurrency.
 */
#ifndef GFT_H
#define GFT_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GFT_API __attribute__((visibility("default")))
#else
#define GFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GFT_VERSION 1
#define GFT_INF 0x7FFFFFFF
#define GFT_NO_PARENT 0xFFFFFFFFu

typedef enum gft_status {
    GFT_OK = 0,
    GFT_ERR_INVALID_ARG = 1,   /* bad pointer, size or option                     */
    GFT_ERR_IO = 2,            /* open/read/write failed                          */
    GFT_ERR_FORMAT = 3,        /* malformed .gr file                              */
    GFT_ERR_CUDA = 4,          /* a CUDA runtime call failed                      */
    GFT_ERR_OOM = 5,           /* device or host allocation failed / over budget  */
    GFT_ERR_TIMEOUT = 6,       /* a bounded device-side wait expired              */
    GFT_ERR_OVERFLOW = 7,      /* a queue capacity or distance range was exceeded */
    GFT_ERR_NOT_SUPPORTED = 8, /* device is not sm_100 or feature unavailable     */
    GFT_ERR_BUSY = 9           /* serving queue full                              */
} gft_status;

/* Host CSR graph; field meaning as CSRGraph (rt/include/csr_graph.h:96-100). */
typedef struct gft_csr {
    uint32_t nnodes;
    uint32_t nedges;
    uint32_t *row_start; /* nnodes + 1 entries, row_start[nnodes] == nedges */
    uint32_t *edge_dst;  /* nedges entries                                  */
    int32_t *edge_data;  /* nedges entries, or NULL for an unweighted graph  */
} gft_csr;

typedef struct gft_graph gft_graph;   /* device-resident graph            */
typedef struct gft_engine gft_engine; /* per-device traversal scratch     */

typedef struct gft_stats {
    uint32_t levels;            /* BFS: number of levels (max level + 1); SSSP: phases */
    uint32_t iterations;        /* grid-synchronous iterations run                     */
    uint64_t vertices_reached;  /* V_r                                                 */
    uint64_t edges_scanned;     /* edges read by the traversal (with re-relaxations)   */
    uint64_t pushes;            /* frontier pushes                                     */
    float kernel_ms;            /* device time of the traversal launch                 */
    uint32_t grid_blocks;       /* persistent grid size used                           */
    uint32_t block_threads;
} gft_stats;

/* Tunables of one traversal; zero fields take the engine defaults. */
typedef struct gft_tuning {
    uint32_t block_threads;   /* 256, 512 or 1024                                   */
    uint32_t blocks_per_sm;   /* persistent CTAs per SM (capped by occupancy)       */
    uint32_t hub_degree;      /* degree at which a vertex is split across the grid  */
    uint32_t timeout_ms;      /* bound on every device-side wait                    */
    int32_t test_skip_block;  /* test hook: CTA that never arrives (-1 = none)      */
    uint32_t max_blocks;      /* cap on the persistent grid; 0 = automatic (graphs
                                 of <= 2^17 vertices and <= 2^19 edges run on one
                                 CTA, larger ones on the whole grid); 1 = one CTA.
                                 One CTA has 1024 threads whatever block_threads
                                 says; BFS there on a graph of <= 2^17 vertices
                                 and out-degrees <= 32 gives each thread a
                                 frontier vertex and always runs top-down
                                 (levels are the same either way) */
    uint32_t group_blocks;    /* batches: CTAs that share one large query (0 = 8)   */
    uint32_t group_min_nodes; /* batches: queries on graphs with at least this many
                                 vertices run on a CTA group (0 = 262144; set it
                                 above every graph to run each query on one CTA) */
    uint32_t direction;       /* BFS: 0 = direction-optimising when the graph is
                                 marked symmetric, 1 = top-down only          */
    uint32_t cta_small;       /* SSSP on the grid: iterations of at most this
                                 many vertices run on one CTA while the others
                                 wait (0 = engine default: 256 on graphs of
                                 uniform degree, never on skewed ones;
                                 UINT32_MAX = never) */
    uint32_t fuse_budget;     /* SSSP: near vertices a warp may expand itself in
                                 the iteration that found them (0 = engine
                                 default: 256 on graphs of uniform degree,
                                 never on skewed ones; UINT32_MAX = never;
                                 near piles above 524288 vertices are never
                                 fused)                                       */
    uint32_t queue_tile;      /* grid-wide kernels: push-buffer entries per warp,
                                 64, 128 or 256 (0 = engine default: 256, and
                                 128 for SSSP at 1024 threads, whose two
                                 buffers then take at most 128)               */
    uint32_t warp_degree;     /* frontier vertices of at least this many edges
                                 are expanded by a whole warp, smaller ones
                                 flattened across the warp (0 = 32)           */
} gft_tuning;

/* ---------------------------------------------------------------------------
 * Library
 * ------------------------------------------------------------------------- */
GFT_API int gft_version(void);
/* Message of the calling thread's last failed call ("" if none). */
GFT_API const char *gft_last_error(void);
GFT_API const char *gft_status_string(gft_status s);

/* ---------------------------------------------------------------------------
 * .gr binary CSR files.
 * gft_gr_read replaces CSRGraph::read / readFromGR
 * (rt/src/csr_graph.cu:152-241).  Layout (little endian): u64 version (=1),
 * u64 sizeEdgeTy (0 or 4), u64 numNodes, u64 numEdges, u64 outIdx[numNodes]
 * (end offsets), u32 outs[numEdges], u32 pad if numEdges is odd, u32
 * edgeData[numEdges] if sizeEdgeTy != 0.  Unlike the reference (which only
 * prints a warning, csr_graph.cu:219), an edge whose destination is
 * >= numNodes, a non-monotone outIdx or a truncated file is rejected with
 * GFT_ERR_FORMAT.  Arrays are malloc'd; release with gft_csr_free.
 * ------------------------------------------------------------------------- */
GFT_API gft_status gft_gr_read(const char *path, gft_csr *out);
/* The same parse as gft_gr_read through the parallel chunked reader that
 * gft_graph_load_gr uses (pread of 8 MB chunks by up to 8 threads, end
 * offsets narrowed and checked per chunk), into host arrays: the host side
 * of that pipeline, for checking it without a GPU.  Same results and
 * errors as gft_gr_read. */
GFT_API gft_status gft_gr_read_chunked(const char *path, gft_csr *out);
GFT_API gft_status gft_gr_write(const char *path, const gft_csr *g);
GFT_API void gft_csr_free(gft_csr *g);

/* ---------------------------------------------------------------------------
 * Seeded synthetic graphs (host side).  Deterministic functions of their
 * arguments; the same graph is produced by the device generators.
 *   grid:  r x c 4-neighbour grid, ids r*cols+c, both directions; weights
 *          1 when unit_weights, else uniform [1, max_weight] per undirected
 *          edge.
 *   road:  side x side grid with each undirected edge deleted with
 *          probability delete_ppm/1e6, plus shortcut_ppm/1e6 * (grid edges)
 *          random undirected shortcuts; weights uniform [1, max_weight].
 *   rmat:  2^scale vertices, edge_factor * 2^scale samples with quadrant
 *          probabilities a,b,c (d = 1-a-b-c) in parts per 2^32, seeded
 *          vertex permutation, symmetrised, self loops and duplicates
 *          removed; weights uniform [1, max_weight] when max_weight > 0.
 * All graphs are symmetric with rows sorted by destination.
 * ------------------------------------------------------------------------- */
GFT_API gft_status gft_gen_grid(uint32_t rows, uint32_t cols, uint64_t seed, uint32_t max_weight, gft_csr *out);
GFT_API gft_status gft_gen_road(uint32_t side, uint64_t seed, uint32_t delete_ppm, uint32_t shortcut_ppm,
                        uint32_t max_weight, gft_csr *out);
GFT_API gft_status gft_gen_rmat(uint32_t scale, uint32_t edge_factor, uint32_t a_q32, uint32_t b_q32, uint32_t c_q32,
                        uint64_t seed, uint32_t max_weight, gft_csr *out);
/* Draws k distinct sources with out-degree > 0 (k <= nnodes) from seed. */
GFT_API gft_status gft_pick_sources(const gft_csr *g, uint64_t seed, uint32_t k, uint32_t *out_sources);

/* ---------------------------------------------------------------------------
 * Device graphs.
 * gft_graph_upload replaces CSRGraph::copy_to_gpu (rt/src/csr_graph.cu:250-261):
 * it allocates device arrays and copies row_start, edge_dst and edge_data
 * (edge_data only when present) on `stream`, then waits for the copies.
 * gft_graph_wrap adopts caller-owned device arrays without copying; the
 * caller keeps them alive until gft_graph_free.
 * ------------------------------------------------------------------------- */
GFT_API gft_status gft_graph_upload(int device, const gft_csr *g, void *stream, gft_graph **out);
/* .gr file straight to the device: replaces CSRGraph::read + copy_to_gpu
 * (rt/src/csr_graph.cu:152-261, a serial per-edge parse loop, then four
 * synchronous pageable copies).  Worker threads pread 8 MB chunks into
 * pinned staging buffers and copy each with cudaMemcpyAsync on their own
 * stream while reading the next, so file reads and PCIe transfers overlap;
 * end offsets are narrowed to u32 and checked on the host per chunk,
 * destinations are checked on the device.  No host copy of the graph is
 * made.  The pinned staging (128 MB) is allocated by the first call and kept
 * for later ones until gft_ingest_release.  Errors as gft_gr_read. */
GFT_API gft_status gft_graph_load_gr(int device, const char *path, void *stream, gft_graph **out);
GFT_API void gft_ingest_release(void);
GFT_API gft_status gft_graph_wrap(int device, uint32_t nnodes, uint32_t nedges, const uint32_t *d_row_start,
                          const uint32_t *d_edge_dst, const int32_t *d_edge_data, gft_graph **out);
/* Generates a synthetic graph directly in device memory (same result as the
 * host generators above; kind 0 = grid, 1 = road, 2 = rmat, with the
 * parameters of those functions in p[0..7] as listed in gft_gen_params). */
typedef struct gft_gen_params {
    uint32_t kind;          /* 0 grid, 1 road, 2 rmat                        */
    uint32_t rows, cols;    /* grid; road uses rows as the side              */
    uint32_t scale, edge_factor, a_q32, b_q32, c_q32; /* rmat              */
    uint32_t delete_ppm, shortcut_ppm;                  /* road              */
    uint32_t max_weight;    /* 0 = unweighted (grid: 1 = unit weights)       */
    uint64_t seed;
} gft_gen_params;
GFT_API gft_status gft_graph_generate(int device, const gft_gen_params *p, void *stream, gft_graph **out);
GFT_API gft_status gft_graph_info(const gft_graph *g, uint32_t *nnodes, uint32_t *nedges, int *weighted);
/* Symmetry mark (no counterpart in the reference, whose BFS is top-down
 * only).  A graph marked symmetric (every edge u->v has v->u) lets gft_bfs
 * run direction-optimising: levels with a large frontier run bottom-up,
 * each unvisited vertex looking for a parent among its own edges.
 * gft_graph_generate marks its graphs; uploaded and wrapped graphs start
 * unmarked, and the caller marks them only when the mark is true (a wrong
 * mark gives wrong levels).  Levels are the same in either direction. */
GFT_API gft_status gft_graph_set_symmetric(gft_graph *g, int symmetric);
GFT_API gft_status gft_graph_is_symmetric(const gft_graph *g, int *symmetric);
/* Device pointers of a graph (any may be NULL). */
GFT_API gft_status gft_graph_arrays(const gft_graph *g, const uint32_t **d_row_start, const uint32_t **d_edge_dst,
                            const int32_t **d_edge_data);
/* gft_pick_sources for a device graph (reads only its row_start). */
GFT_API gft_status gft_graph_pick_sources(const gft_graph *g, uint64_t seed, uint32_t k, uint32_t *out_sources);
/* Copies a device graph back to a host CSR (arrays malloc'd). */
GFT_API gft_status gft_graph_download(const gft_graph *g, gft_csr *out);
GFT_API void gft_graph_free(gft_graph *g);

/* ---------------------------------------------------------------------------
 * Engines
 * ------------------------------------------------------------------------- */
GFT_API gft_status gft_engine_create(int device, gft_engine **out);
GFT_API void gft_engine_destroy(gft_engine *e);
/* Bytes of device scratch the engine currently holds. */
GFT_API size_t gft_engine_scratch_bytes(const gft_engine *e);

/* ---------------------------------------------------------------------------
 * Single queries.
 *
 * gft_bfs replaces gg_main of apps/bfs (apps/bfs/kernel.cu:380-393) with its
 * persistent driver gg_main_pipe_1_gpu_gb (:312-334): d_level[v] = hop
 * distance from src, GFT_INF if unreached.  If d_parent is non-NULL it
 * receives a BFS tree: parent[src] = src, parent[v] = a vertex p with an
 * edge (p, v) and level[p] + 1 == level[v], GFT_NO_PARENT if unreached.
 *
 * gft_sssp replaces gg_main of apps/sssp (apps/sssp/kernel.cu:455-480) with
 * gg_main_pipe_1_gpu_gb (:355-391): d_dist[v] = shortest-path distance from
 * src under int32 edge weights (reference -d delta: `delta` is the bucket
 * width, > 0, and affects only the schedule), GFT_INF if unreached.  An
 * unweighted graph has weight 0 on every edge, as in the reference (whose
 * edge_data is calloc'd, rt/src/csr_graph.cu:211).  d_parent as for BFS with
 * dist[p] + w(p, v) == dist[v] (weights must be >= 1 for a tree).
 * Returns GFT_ERR_OVERFLOW if a distance would exceed INT_MAX - 1.
 * ------------------------------------------------------------------------- */
GFT_API gft_status gft_bfs(gft_engine *e, const gft_graph *g, uint32_t src, int32_t *d_level, uint32_t *d_parent,
                   const gft_tuning *tune, void *stream, gft_stats *stats);
GFT_API gft_status gft_sssp(gft_engine *e, const gft_graph *g, uint32_t src, int32_t delta, int32_t *d_dist,
                    uint32_t *d_parent, const gft_tuning *tune, void *stream, gft_stats *stats);

/* Host-buffer variants (the end-to-end path of the reference's skel driver,
 * skelapp/skel.cu:159-174: traversal, then copy of node_data to the host).
 * The source goes to the device and the nnodes results come back inside the
 * call; h_out (and h_parent if non-NULL) are host arrays of nnodes entries.
 * The call returns when the results are in host memory. */
GFT_API gft_status gft_bfs_host(gft_engine *e, const gft_graph *g, uint32_t src, int32_t *h_level, uint32_t *h_parent,
                        const gft_tuning *tune, void *stream, gft_stats *stats);
GFT_API gft_status gft_sssp_host(gft_engine *e, const gft_graph *g, uint32_t src, int32_t delta, int32_t *h_dist,
                         uint32_t *h_parent, const gft_tuning *tune, void *stream, gft_stats *stats);

/* Many single-source queries on one graph, results to host memory.  The
 * reference runs one source per process and copies node_data back after
 * each traversal (skelapp/skel.cu:139-174); these calls run the k sources
 * one after another on `stream`, each exactly as gft_bfs_host /
 * gft_sssp_host would, but copy a query's results back on an engine-owned
 * stream while the next query runs (two device result buffers), so the
 * device->host transfer overlaps the traversal.  h_out holds k rows of
 * nnodes int32 (row i: levels / distances from sources[i]); it should be
 * pinned memory, or the copies cannot overlap.  stats: NULL or k entries.
 * All sources are checked before anything runs.  On an error no copy is
 * left in flight and the rows of the queries before the failing one are
 * complete. */
GFT_API gft_status gft_bfs_host_many(gft_engine *e, const gft_graph *g, const uint32_t *sources, uint32_t k,
                             int32_t *h_out, const gft_tuning *tune, void *stream, gft_stats *stats);
GFT_API gft_status gft_sssp_host_many(gft_engine *e, const gft_graph *g, const uint32_t *sources, uint32_t k,
                              int32_t delta, int32_t *h_out, const gft_tuning *tune, void *stream,
                              gft_stats *stats);

/* Allocation-free BFS.  No counterpart in the reference: gg_main allocates
 * its worklists on every call (apps/bfs/kernel.cu:389, rt/include/worklist.h:
 * 73-118).  For callers that cannot call cudaMalloc -- code running while
 * another component owns the device memory, or paths where an allocation's
 * implicit synchronisation is not allowed -- this variant neither allocates
 * nor frees anything: no engine, no cudaMalloc/cudaFree, no allocating
 * library routine.  Its scratch is one fixed file-scope device array
 * (about 16.2 MB, held by every GPU that loads libgft until exit), so the
 * graph may have at most 1,048,576 vertices; larger graphs are rejected with
 * GFT_ERR_INVALID_ARG.  The caller passes the graph and the output buffers
 * (d_level, optional d_parent) as for gft_bfs; results are identical, and
 * the schedule is gft_bfs's too (bottom-up levels on a graph marked
 * symmetric unless tune->direction says otherwise).
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress with that device current); make that first call
 * before any stream capture.  Every call reuses the same array (the control
 * block is cleared on `stream` before each launch), so calls whose work
 * overlaps on the GPU race: serialise them.  Waits for `stream`; stats as
 * for gft_bfs except kernel_ms (0: no events are created). */
GFT_API gft_status gft_bfs_noalloc(const gft_graph *g, uint32_t src, int32_t *d_level, uint32_t *d_parent,
                                   const gft_tuning *tune, void *stream, gft_stats *stats);

/* ---------------------------------------------------------------------------
 * Batched queries (no counterpart in the reference, which runs one query per
 * process: skelapp/skel.cu:139-151).  Many BFS / SSSP queries, on one or many
 * resident graphs, run in one persistent launch: each query runs on one CTA
 * (control block in shared memory, block-level barriers), the largest
 * queries first.  The launch (job-table upload, cursor reset, kernel) is
 * captured once as a CUDA graph by gft_batch_create and replayed by every
 * gft_batch_submit.  Results are identical to gft_bfs / gft_sssp.
 * ------------------------------------------------------------------------- */
#define GFT_APP_BFS 0u
#define GFT_APP_SSSP 1u

typedef struct gft_query {
    const gft_graph *graph;
    uint32_t app;        /* GFT_APP_BFS or GFT_APP_SSSP                        */
    uint32_t src;
    int32_t delta;       /* SSSP bucket width (> 0)                            */
    int32_t *d_out;      /* device, nnodes int32: levels / distances           */
    uint32_t *d_parent;  /* device, nnodes, or NULL (BFS only in batches)      */
    /* filled by gft_batch_wait */
    gft_status status;
    uint32_t levels, iterations;
    uint64_t edges_scanned;
    float device_ms;     /* time the query occupied its CTA                    */
} gft_query;

typedef struct gft_batch_stats {
    uint32_t queries;
    float launch_ms;        /* device time of the whole launch (events)      */
    float busy_ms;          /* first query start to last query end (device)  */
    uint64_t edges_scanned;
    uint32_t grid_blocks, block_threads;
    size_t scratch_bytes;   /* device scratch held by the batch               */
} gft_batch_stats;

typedef struct gft_batch gft_batch;

/* Validates the n queries, allocates the batch's scratch (per query: 2 or 6
 * x nnodes x 4 bytes plus its hub list), uploads nothing yet and captures the
 * launch.  tune: block_threads (256/512/1024), blocks_per_sm, hub_degree. */
GFT_API gft_status gft_batch_create(gft_engine *e, const gft_query *q, uint32_t n, const gft_tuning *tune,
                                    gft_batch **out);
/* Changes query `query`'s source for the next submit (no re-capture).
 * Returns GFT_ERR_BUSY between a submit and its gft_batch_wait: the replay
 * reads the job table when it starts on the device. */
GFT_API gft_status gft_batch_set_source(gft_batch *b, uint32_t query, uint32_t src);
/* Replays the captured launch on `stream` (asynchronous). */
GFT_API gft_status gft_batch_submit(gft_batch *b, void *stream);
/* Waits for the last submit and fills each query's status and statistics
 * (q may be NULL); returns the first failing query's status, if any. */
GFT_API gft_status gft_batch_wait(gft_batch *b, gft_query *q, gft_batch_stats *stats);
GFT_API void gft_batch_destroy(gft_batch *b);

/* ---------------------------------------------------------------------------
 * Serving (no counterpart in the reference, which runs one query per
 * process).  A request loop over resident graphs with continuous batching.
 * The device's resident CTAs are split into `lanes` of `lane_blocks` CTAs,
 * each with its own stream and scratch arena, so their launches overlap on
 * the device.  In arrival order, a heavy request (a graph of at least
 * `group_min_nodes` vertices; with sparse_degree > 0, BFS on a graph of
 * lower average degree counts as light) runs alone as one CTA group over
 * w free lanes, w = free lanes / heavy requests waiting, at least 1 and at
 * most `max_lanes_per_request`: on an idle server a request gets the whole
 * device, under load requests share it lane by lane.  SSSP on a large
 * skewed graph (see wide_lanes) instead runs on a reserved pool of lanes,
 * one request at a time, taking every free lane when nothing else waits:
 * such a query moves so much memory that it gains nothing side by side.  A run of light
 * requests shares one launch on one lane, one CTA each.  A request that
 * arrives while others run starts as soon as a lane and arena space are
 * free, and a long request never holds up a launch of short ones.  A
 * request is taken only when its scratch fits in the lane's arena
 * (`lane_arena_bytes`); one that could never fit is refused at enqueue with
 * GFT_ERR_OOM, and a full queue returns GFT_ERR_BUSY.  The caller owns each
 * request's output buffer (d_out) until its completion is polled.
 * ------------------------------------------------------------------------- */
typedef struct gft_serve_config {
    uint32_t lanes;             /* streams (0 = resident CTAs / lane_blocks)     */
    uint32_t max_batch;         /* light requests per launch (default 256)       */
    size_t lane_arena_bytes;    /* scratch arena per lane (default 768 MiB)      */
    uint32_t block_threads;     /* CTA size (default 512)                        */
    uint32_t hub_degree;        /* default 256                                   */
    uint32_t lane_blocks;       /* CTAs per lane (0 = group_blocks)              */
    uint32_t group_blocks;      /* default lane size in CTAs (default 16)        */
    uint32_t group_min_nodes;   /* default 2^18                                  */
    uint32_t sparse_degree;     /* default 0 (no exception)                      */
    uint32_t queue_capacity;    /* requests admitted but not completed           */
    uint32_t max_lanes_per_request; /* widest heavy launch (0 = all lanes)       */
    uint32_t wide_lanes;        /* lanes reserved for wide requests: SSSP on a
                                   graph with a vertex of degree > 32 and at
                                   least wide_min_edges edges.  They run one at
                                   a time on the whole pool (GFT_SERVE_AUTO =
                                   4/9 of the lanes when there are >= 4; 0 =
                                   no pool)                                   */
    uint32_t wide_min_edges;    /* default 2^25                                */
    uint32_t resident;          /* 1: one resident persistent kernel takes the
                                   requests from a ring in mapped host memory
                                   and runs each on a team of lanes drafted on
                                   the device (lane_blocks CTAs per lane,
                                   default 8; widths as idle lanes / waiting
                                   requests, at most max_lanes_per_request);
                                   0: one launch per lane micro-batch (default).
                                   A resident request is ordered with no
                                   stream: work that writes its buffers must
                                   be finished before gft_serve_enqueue, and
                                   kernels launched meanwhile on other
                                   streams wait until the resident kernel
                                   ends (idle_exit_us after its last work) */
    uint32_t idle_exit_us;      /* resident: the kernel ends after this long
                                   without work and is launched again by the
                                   next request (0 = 2000)                    */
} gft_serve_config;
#define GFT_SERVE_AUTO 0xFFFFFFFFu

typedef struct gft_completion {
    uint64_t ticket;
    gft_status status;
    double latency_ms;      /* enqueue -> completion observed                 */
    double queue_ms;        /* enqueue -> launch                              */
    uint32_t lane;          /* lane (1-based) that ran the request             */
    uint32_t batch_size;    /* requests in the same launch                    */
    uint32_t width;         /* lanes the launch spanned                       */
    uint32_t levels;
    uint64_t edges_scanned;
} gft_completion;

typedef struct gft_server gft_server;

GFT_API gft_status gft_serve_config_default(gft_serve_config *cfg);
GFT_API gft_status gft_serve_open(gft_engine *e, const gft_serve_config *cfg, gft_server **out);
/* Non-blocking; *ticket identifies the request's completion. */
GFT_API gft_status gft_serve_enqueue(gft_server *s, const gft_query *q, uint64_t *ticket);
/* Up to `max` completions; waits up to wait_us for the first one. */
GFT_API gft_status gft_serve_poll(gft_server *s, gft_completion *out, uint32_t max, uint32_t *n, uint32_t wait_us);
GFT_API gft_status gft_serve_stats(gft_server *s, uint64_t *in_flight, uint64_t *batches, uint64_t *queries);
/* Finishes the admitted requests, then releases the server. */
GFT_API gft_status gft_serve_close(gft_server *s);

/* ---------------------------------------------------------------------------
 * Multi-source BFS (no counterpart in the reference, which runs one source
 * per process).  k <= 256 BFS queries on one graph in one launch with
 * per-vertex bitsets (one bit per source).  The result is a stack of
 * frontier planes in caller memory (16-byte aligned): d_planes holds
 * max_levels planes of gft_msbfs_plane_bytes(nnodes, k) bytes each.  A plane
 * has one row of WP words per vertex, WP = ceil(k / 32) rounded up to 1, 2,
 * 4 or 8; in plane L, bit i % 32 of word i / 32 of vertex v's row is set iff
 * source i reaches v at level L.  stats->levels = planes used;
 * GFT_ERR_OVERFLOW if the traversal needs more than max_levels.  The last
 * level is only known to be last once its expansion found nothing new, which
 * needs room for one more plane: give max_levels >= levels + 1 (a graph whose
 * sources reach everything within D hops needs D + 2).
 * gft_msbfs_levels writes source i's int32 levels (as gft_bfs would) from
 * the planes.  flags: GFT_MSBFS_SYMMETRIC allows bottom-up levels (the
 * graph's out-edges must also be its in-edges); without it every level is
 * top-down.
 * ------------------------------------------------------------------------- */
#define GFT_MSBFS_SYMMETRIC 1u
GFT_API size_t gft_msbfs_plane_bytes(uint32_t nnodes, uint32_t k);
GFT_API gft_status gft_msbfs(gft_engine *e, const gft_graph *g, const uint32_t *h_sources, uint32_t k,
                             uint32_t *d_planes, uint32_t max_levels, uint32_t flags, void *stream, gft_stats *stats);
GFT_API gft_status gft_msbfs_levels(const uint32_t *d_planes, uint32_t nnodes, uint32_t k, uint32_t levels, uint32_t i,
                                    int32_t *d_out, void *stream);

/* ---------------------------------------------------------------------------
 * Connected components: replaces apps/cc gg_main (apps/cc/kernel.cu:630-723),
 * whose result is node_data.  d_label[v] (int32, nnodes entries) becomes the
 * smallest vertex id of v's weakly connected component: every edge joins its
 * endpoints, as the reference's hooks treat it (:249-330).  The reference's
 * own labels are whichever roots its racy hooks leave, so only its
 * partition and its count ("components: N", :449-462,719) are comparable;
 * these labels do not depend on the schedule.  *components receives the
 * number of components.  On a graph marked symmetric each undirected edge is
 * joined once.
 * ------------------------------------------------------------------------- */
GFT_API gft_status gft_cc(gft_engine *e, const gft_graph *g, int32_t *d_label, const gft_tuning *tune, void *stream,
                          gft_stats *stats, uint64_t *components);
GFT_API gft_status gft_cc_host(gft_engine *e, const gft_graph *g, int32_t *h_label, const gft_tuning *tune,
                               void *stream, gft_stats *stats, uint64_t *components);
/* Writes CC labels in the reference's output format (apps/cc/support.cu:
 * 16-36): per node "%d %d\n", then one "\te %d: %d %d %d\n" line per out-edge
 * (edge index, destination, edge_data or 0, destination's label).  The host
 * CSR supplies the edges.  path "-" writes to stdout. */
GFT_API gft_status gft_write_cc_output(const char *path, const gft_csr *g, const int32_t *h_label);

/* ---------------------------------------------------------------------------
 * PageRank by residual push: replaces apps/pr gg_main (apps/pr/kernel.cu:
 * 362-389) with its constants ALPHA = 0.85 and EPSILON = 1e-6 (:19-20).
 * d_rank (float, nnodes entries) receives the unnormalised ranks the
 * reference prints; max_iterations bounds the worklist rounds (its -x
 * option; UINT32_MAX = until converged); stats->levels = rounds run,
 * stats->edges_scanned = edges pushed along, stats->pushes = worklist
 * entries processed over all rounds.  Float
 * atomicAdd makes the summation order, and so the last bits of the ranks,
 * depend on the schedule, in the reference as here.
 * ------------------------------------------------------------------------- */
GFT_API gft_status gft_pr(gft_engine *e, const gft_graph *g, float *d_rank, uint32_t max_iterations,
                          const gft_tuning *tune, void *stream, gft_stats *stats);
GFT_API gft_status gft_pr_host(gft_engine *e, const gft_graph *g, float *h_rank, uint32_t max_iterations,
                               const gft_tuning *tune, void *stream, gft_stats *stats);
/* Writes ranks as the reference does: "%d %f\n" per node (apps/pr/support.cu:
 * 95-101).  path "-" writes to stdout. */
GFT_API gft_status gft_write_pr_output(const char *path, uint32_t nnodes, const float *h_rank);

/* ---------------------------------------------------------------------------
 * Maximal independent set: replaces apps/mis gg_main (apps/mis/kernel.cu:
 * 215-231).  d_state (int32, nnodes entries) receives the reference's
 * node_data: 1 = in the set, 2 = excluded (NON_INDEPENDENT).  Priorities
 * follow the reference: one xorshift128 stream per thread of a launch of
 * prio_threads threads (0 = the reference's grid on this device, 8 CTAs of
 * 256 threads per SM), so the set is the reference's on the same GPU.
 * stats->levels = rounds ("Total steps"), stats->vertices_reached = the
 * set's size, stats->edges_scanned = neighbour words read, stats->pushes =
 * worklist entries over all rounds.
 * ------------------------------------------------------------------------- */
GFT_API gft_status gft_mis(gft_engine *e, const gft_graph *g, int32_t *d_state, uint32_t prio_threads,
                           const gft_tuning *tune, void *stream, gft_stats *stats);
GFT_API gft_status gft_mis_host(gft_engine *e, const gft_graph *g, int32_t *h_state, uint32_t prio_threads,
                                const gft_tuning *tune, void *stream, gft_stats *stats);
/* Writes the reference's MIS text (apps/mis/support.cu:18-40): the set's
 * size, then one member id per line.  path "-" writes to stdout. */
GFT_API gft_status gft_write_mis_output(const char *path, uint32_t nnodes, const int32_t *h_state);

/* Reach statistics of a result already on the device: V_r (vertices with a
 * finite value) and E_r (sum of their out-degrees, the edges a top-down
 * traversal must scan).  Waits for `stream`. */
GFT_API gft_status gft_reach_stats(const gft_graph *g, const int32_t *d_val, void *stream, uint64_t *v_r, uint64_t *e_r);

/* Writes values in the reference's output format, "%d %d\n" or "%d INF\n"
 * per node (apps/bfs/support.cu:27-45, apps/sssp/support.cu:34-53).
 * path "-" writes to stdout. */
GFT_API gft_status gft_write_output(const char *path, uint32_t nnodes, const int32_t *h_val);

/* Output path for large results (no counterpart in the reference, whose
 * output() formats every line with one fprintf, apps/sssp/support.cu:34-53;
 * the text of a 16.8 M-vertex result is ~250 MB).
 * gft_write_output_gz: the same text as gft_write_output, gzip-compressed
 * (zlib `level` 1..9, 0 = 1).  Blocks of 2^20 lines are formatted and
 * deflated on all host threads, each block a complete gzip member; members
 * are written in order, so the file is one valid gzip stream (RFC 1952
 * allows concatenated members) that gunzip, zcat or zlib read back as the
 * text file.
 * gft_write_node_data / gft_read_node_data: a binary dump of a result
 * array: the 8 bytes "GFTNODE1", u32 element type (GFT_ELEM_I32: levels,
 * distances, labels, MIS states; GFT_ELEM_F32: PageRank ranks), u32 0, u64
 * nnodes, then nnodes little-endian 4-byte values.  gft_read_node_data
 * with h_val NULL only returns nnodes and the type; otherwise h_val must
 * hold *nnodes values on entry (the capacity) and receives them. */
#define GFT_ELEM_I32 0u
#define GFT_ELEM_F32 1u
GFT_API gft_status gft_write_output_gz(const char *path, uint32_t nnodes, const int32_t *h_val, int level);
GFT_API gft_status gft_write_node_data(const char *path, uint32_t nnodes, const void *h_val, uint32_t elem_type);
GFT_API gft_status gft_read_node_data(const char *path, uint32_t *nnodes, uint32_t *elem_type, void *h_val);

#ifdef __cplusplus
}
#endif
#endif /* GFT_H */
