/*
 * oracle.c -- CPU oracle for the worklist BFS / SSSP hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke()
 * entry and the CPU-baseline leg of bench.py load it (as liboracle.so through
 * ctypes).  Nothing in the galoisgpu_b200 package links, loads or calls it;
 * the product path has no CPU fallback.
 *
 * It restates, serially and in plain C, what LonestarGPU v3 computes on the
 * path (all citations relative to the reference project root):
 *
 *   - .gr v1 parse                rt/src/csr_graph.cu:187-228
 *   - BFS levels                  apps/bfs/kernel.cu:20-32 (init: src 0, else
 *                                 INF), :86-92/:194-199 (visit sets LEVEL),
 *                                 :380-393 (LEVEL starts at 1)
 *   - SSSP distances              apps/sssp/kernel.cu:23-35 (init),
 *                                 :129-143/:244-259 (relax with int add and
 *                                 atomicMin), :455-478 (driver)
 *   - output text                 apps/bfs/support.cu:27-45,
 *                                 apps/sssp/support.cu:34-53
 *   - connected components        apps/cc/kernel.cu:18-29 (init: label v),
 *                                 :249-330 (hooking over every edge, both
 *                                 endpoints), :449-462 (a component is a
 *                                 vertex that is its own label),
 *                                 apps/cc/support.cu:16-36 (output)
 *   - PageRank (residual push)    apps/pr/kernel.cu:17-20 (ALPHA, EPSILON),
 *                                 :26-47 (init_1), :49-63 (init_2),
 *                                 :127-236 (pop and push), :271-305 (driver),
 *                                 apps/pr/support.cu:47-104 (output)
 *   - maximal independent set     apps/mis/kernel.cu:9-17 (states, seeds),
 *                                 :18-41 (per-thread xorshift priorities),
 *                                 :65-103 (mark local maxima), :104-149
 *                                 (drop marked vertices and neighbours),
 *                                 :151-169 (rounds), apps/mis/support.cu:18-40
 *                                 (output)
 *
 * The reference's BFS and SSSP results are schedule independent: BFS levels
 * are hop distances and SSSP distances are the unique shortest-path lengths
 * (atomicMin is monotone), so a FIFO BFS and a binary-heap Dijkstra give the
 * same numbers bit for bit as long as no distance overflows int32.
 *
 * The reference's CC labels are not canonical: its hooks are racy plain
 * stores (apps/cc/kernel.cu:263,293,329), so which vertex of a component
 * ends up as the label depends on the schedule.  The partition into
 * components is not, and neither is the count.  This restatement labels
 * every vertex with the smallest vertex id of its component; parity with the
 * reference is checked on the partition.
 *
 * PageRank accumulates float residuals with atomicAdd in whatever order the
 * GPU runs, so its ranks are not bit-reproducible even between two runs of
 * the reference; this restatement processes each level of its worklist in
 * vertex order with the same float arithmetic, and parity is a tolerance.
 *
 * Parity of this restatement is pinned against outputs of the reference's
 * own CUDA build (oracle/ref/Makefile builds it from the reference sources;
 * tests/golden/make_golden.py records its outputs as fixtures).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_INF 0x7FFFFFFF /* INT_MAX: apps/bfs/kernel.cu:16, apps/sssp/kernel.cu:18 */

/* ------------------------------------------------------------------ */
/* .gr v1 parse (rt/src/csr_graph.cu:187-228).                          */
/* Returns 0 on success, negative on error.  Arrays are malloc'd; free  */
/* with orc_free.  edge_data is NULL when sizeEdgeTy == 0 (the          */
/* reference then leaves its calloc'd zeros, csr_graph.cu:211,223).     */
/* ------------------------------------------------------------------ */
int orc_gr_read(const char *path, uint32_t *nnodes, uint32_t *nedges,
                uint32_t **row_start, uint32_t **edge_dst, int32_t **edge_data)
{
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    uint64_t hdr[4];
    if (fread(hdr, 8, 4, f) != 4) { fclose(f); return -2; }
    if (hdr[0] != 1) { fclose(f); return -3; }            /* version asserted == 1 */
    uint64_t size_edge_ty = hdr[1], nn = hdr[2], ne = hdr[3];
    if (nn >= 0xFFFFFFFFull || ne >= 0xFFFFFFFFull) { fclose(f); return -4; }
    uint64_t *out_idx = (uint64_t *)malloc((nn ? nn : 1) * 8);
    uint32_t *rs = (uint32_t *)malloc((nn + 1) * 4);
    uint32_t *dst = (uint32_t *)malloc((ne ? ne : 1) * 4);
    int32_t *w = NULL;
    if (!out_idx || !rs || !dst) { fclose(f); return -5; }
    if (fread(out_idx, 8, nn, f) != nn) goto trunc;
    if (fread(dst, 4, ne, f) != ne) goto trunc;
    if (ne % 2) { uint32_t pad; if (fread(&pad, 4, 1, f) != 1 && size_edge_ty) goto trunc; }
    if (size_edge_ty) {
        w = (int32_t *)malloc((ne ? ne : 1) * 4);
        /* weights are read as unsigned and stored into int (csr_graph.cu:199,223-224) */
        if (fread(w, 4, ne, f) != ne) goto trunc;
    }
    fclose(f);
    rs[0] = 0;
    for (uint64_t i = 0; i < nn; i++) {
        if (out_idx[i] > ne || (i && out_idx[i] < out_idx[i - 1])) { free(out_idx); free(rs); free(dst); free(w); return -6; }
        rs[i + 1] = (uint32_t)out_idx[i];
    }
    if (nn && out_idx[nn - 1] != ne) { free(out_idx); free(rs); free(dst); free(w); return -6; }
    for (uint64_t e = 0; e < ne; e++)
        if (dst[e] >= nn) { free(out_idx); free(rs); free(dst); free(w); return -7; }
    free(out_idx);
    *nnodes = (uint32_t)nn; *nedges = (uint32_t)ne;
    *row_start = rs; *edge_dst = dst; *edge_data = w;
    return 0;
trunc:
    fclose(f); free(out_idx); free(rs); free(dst); free(w);
    return -8;
}

void orc_free(void *p) { free(p); }

/* ------------------------------------------------------------------ */
/* BFS: FIFO queue.  level[src] = 0, every other vertex INF, and a      */
/* vertex discovered while expanding level L-1 gets level L             */
/* (apps/bfs/kernel.cu:20-32, :194-199, :388).                          */
/* parent (optional): the vertex that discovered it, src for src.       */
/* Returns the number of vertices reached.                              */
/* ------------------------------------------------------------------ */
uint64_t orc_bfs(uint32_t nnodes, const uint32_t *row_start, const uint32_t *edge_dst,
                 uint32_t src, int32_t *level, uint32_t *parent)
{
    for (uint32_t v = 0; v < nnodes; v++) { level[v] = ORC_INF; if (parent) parent[v] = 0xFFFFFFFFu; }
    if (src >= nnodes) return 0;
    uint32_t *q = (uint32_t *)malloc((size_t)nnodes * 4);
    size_t head = 0, tail = 0;
    level[src] = 0; if (parent) parent[src] = src;
    q[tail++] = src;
    while (head < tail) {
        uint32_t u = q[head++];
        int32_t nl = level[u] + 1;
        for (uint32_t e = row_start[u]; e < row_start[u + 1]; e++) {
            uint32_t v = edge_dst[e];
            if (level[v] == ORC_INF) { level[v] = nl; if (parent) parent[v] = u; q[tail++] = v; }
        }
    }
    free(q);
    return tail;
}

/* ------------------------------------------------------------------ */
/* SSSP: binary-heap Dijkstra with lazy deletion.  dist[src] = 0, INF   */
/* otherwise (apps/sssp/kernel.cu:23-35).  A relaxation computes        */
/* dist[u] + w in int arithmetic (:131,:246,:284); the result is the    */
/* unique shortest-path distance, computed here in 64 bits and clamped  */
/* check: returns -1 if any finite distance would exceed INT_MAX-1      */
/* (the reference would overflow there), else the number reached.       */
/* ------------------------------------------------------------------ */
typedef struct { int64_t d; uint32_t v; } heap_item;

static void heap_push(heap_item *h, size_t *n, heap_item it)
{
    size_t i = (*n)++;
    while (i) {
        size_t p = (i - 1) / 2;
        if (h[p].d < it.d || (h[p].d == it.d && h[p].v <= it.v)) break;
        h[i] = h[p]; i = p;
    }
    h[i] = it;
}

static heap_item heap_pop(heap_item *h, size_t *n)
{
    heap_item top = h[0], last = h[--(*n)];
    size_t i = 0;
    for (;;) {
        size_t l = 2 * i + 1, r = l + 1, m = i;
        heap_item best = last;
        if (l < *n && (h[l].d < best.d || (h[l].d == best.d && h[l].v < best.v))) { m = l; best = h[l]; }
        if (r < *n && (h[r].d < best.d || (h[r].d == best.d && h[r].v < best.v))) { m = r; best = h[r]; }
        if (m == i) break;
        h[i] = h[m]; i = m;
    }
    h[i] = last;
    return top;
}

int64_t orc_sssp(uint32_t nnodes, const uint32_t *row_start, const uint32_t *edge_dst,
                 const int32_t *edge_data, uint32_t src, int32_t *dist, uint32_t *parent)
{
    for (uint32_t v = 0; v < nnodes; v++) { dist[v] = ORC_INF; if (parent) parent[v] = 0xFFFFFFFFu; }
    if (src >= nnodes) return 0;
    uint64_t ne = row_start[nnodes];
    size_t cap = (size_t)ne + 2, n = 0;
    heap_item *h = (heap_item *)malloc(cap * sizeof(heap_item));
    int64_t *d = (int64_t *)malloc((size_t)nnodes * 8);
    unsigned char *done = (unsigned char *)calloc(nnodes, 1);
    for (uint32_t v = 0; v < nnodes; v++) d[v] = INT64_MAX;
    d[src] = 0; if (parent) parent[src] = src;
    heap_item s = {0, src};
    heap_push(h, &n, s);
    int64_t reached = 0, overflow = 0;
    while (n) {
        heap_item it = heap_pop(h, &n);
        if (done[it.v] || it.d != d[it.v]) continue;
        done[it.v] = 1; reached++;
        for (uint32_t e = row_start[it.v]; e < row_start[it.v + 1]; e++) {
            uint32_t v = edge_dst[e];
            int64_t nd = it.d + (int64_t)edge_data[e];
            if (nd < d[v]) {
                d[v] = nd; if (parent) parent[v] = it.v;
                heap_item x = {nd, v};
                heap_push(h, &n, x);
            }
        }
    }
    for (uint32_t v = 0; v < nnodes; v++) {
        if (d[v] == INT64_MAX) continue;
        if (d[v] >= ORC_INF) overflow = 1;
        dist[v] = (int32_t)d[v];
    }
    free(h); free(d); free(done);
    return overflow ? -1 : reached;
}

/* ------------------------------------------------------------------ */
/* Parent-tree validators.  For each reached v != src there must be an  */
/* edge (p, v) with val[p] + step == val[v] (step 1 for BFS, the edge   */
/* weight for SSSP); parent[src] == src; an unreached vertex has        */
/* val INF.  Duplicate (p, v) edges are fine: any copy with the right   */
/* weight proves it.  Returns the number of violations (0 = valid).    */
/* ------------------------------------------------------------------ */
static int has_edge_with(uint32_t p, uint32_t v, const uint32_t *row_start, const uint32_t *edge_dst,
                         const int32_t *edge_data, int64_t need)
{
    for (uint32_t e = row_start[p]; e < row_start[p + 1]; e++)
        if (edge_dst[e] == v && (edge_data ? (int64_t)edge_data[e] : 1) == need) return 1;
    return 0;
}

uint64_t orc_check_tree(uint32_t nnodes, const uint32_t *row_start, const uint32_t *edge_dst,
                        const int32_t *edge_data /* NULL for BFS */, uint32_t src,
                        const int32_t *val, const uint32_t *parent)
{
    uint64_t bad = 0;
    for (uint32_t v = 0; v < nnodes; v++) {
        if (val[v] == ORC_INF) continue;
        if (v == src) { if (parent[v] != src || val[v] != 0) bad++; continue; }
        uint32_t p = parent[v];
        if (p >= nnodes || val[p] == ORC_INF) { bad++; continue; }
        int64_t need = (int64_t)val[v] - (int64_t)val[p];
        if (need < 0 || !has_edge_with(p, v, row_start, edge_dst, edge_data, need)) bad++;
    }
    return bad;
}

/* Reach statistics used for GTEPS: V_r = reached vertices, E_r = sum of */
/* out-degrees over reached vertices (the CSR edges a top-down          */
/* traversal scans).                                                    */
void orc_reach_stats(uint32_t nnodes, const uint32_t *row_start, const int32_t *val,
                     uint64_t *v_r, uint64_t *e_r)
{
    uint64_t vr = 0, er = 0;
    for (uint32_t v = 0; v < nnodes; v++)
        if (val[v] != ORC_INF) { vr++; er += row_start[v + 1] - row_start[v]; }
    *v_r = vr; *e_r = er;
}

/* ------------------------------------------------------------------ */
/* Output text exactly as the reference writes it: "%d %d\n" or         */
/* "%d INF\n" per node, i = 0..nnodes-1 (apps/bfs/support.cu:39-45).    */
/* ------------------------------------------------------------------ */
int orc_write_output(const char *path, uint32_t nnodes, const int32_t *val)
{
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    for (int i = 0; i < (int)nnodes; i++) {
        if (val[i] == ORC_INF) fprintf(f, "%d INF\n", i);
        else fprintf(f, "%d %d\n", i, val[i]);
    }
    return fclose(f) ? -2 : 0;
}

/* Parse the reference's output text back into values; returns the      */
/* number of lines parsed or negative on a malformed line.               */
int64_t orc_read_output(const char *path, uint32_t nnodes, int32_t *val)
{
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char line[128];
    int64_t n = 0;
    while (fgets(line, sizeof line, f)) {
        long idx; char tok[64];
        if (sscanf(line, "%ld %63s", &idx, tok) != 2 || idx < 0 || (uint64_t)idx >= nnodes) { fclose(f); return -2; }
        if (strcmp(tok, "INF") == 0) val[idx] = ORC_INF;
        else val[idx] = (int32_t)strtol(tok, NULL, 10);
        n++;
    }
    fclose(f);
    return n;
}

/* ------------------------------------------------------------------ */
/* Connected components (weak: every edge joins its endpoints, as the   */
/* reference's hooking treats it, apps/cc/kernel.cu:249-330).  label[v] */
/* = the smallest vertex id of v's component.  Union-find with path     */
/* halving; the smaller root always becomes the parent.  Returns the    */
/* number of components (apps/cc/kernel.cu:449-462).                    */
/* ------------------------------------------------------------------ */
static uint32_t uf_find(uint32_t *p, uint32_t x)
{
    while (p[x] != x) {
        p[x] = p[p[x]];
        x = p[x];
    }
    return x;
}

uint64_t orc_cc(uint32_t nnodes, const uint32_t *row_start, const uint32_t *edge_dst, int32_t *label)
{
    uint32_t *p = (uint32_t *)malloc((size_t)(nnodes ? nnodes : 1) * 4);
    for (uint32_t v = 0; v < nnodes; v++) p[v] = v;
    for (uint32_t u = 0; u < nnodes; u++)
        for (uint32_t e = row_start[u]; e < row_start[u + 1]; e++) {
            uint32_t a = uf_find(p, u), b = uf_find(p, edge_dst[e]);
            if (a < b) p[b] = a;
            else if (b < a) p[a] = b;
        }
    uint64_t comps = 0;
    for (uint32_t v = 0; v < nnodes; v++) {
        label[v] = (int32_t)uf_find(p, v);
        comps += label[v] == (int32_t)v;
    }
    free(p);
    return comps;
}

/* CC output text as the reference writes it (apps/cc/support.cu:16-36):  */
/* per node "%d %d\n" (id, label), then per out-edge j of that node        */
/* "\te %d: %d %d %d\n" (j, dst, edge_data[j], label[dst]); edge_data is   */
/* 0 for an unweighted graph (the reference's calloc'd array).             */
int orc_write_cc_output(const char *path, uint32_t nnodes, const uint32_t *row_start, const uint32_t *edge_dst,
                        const int32_t *edge_data, const int32_t *label)
{
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    for (int i = 0; i < (int)nnodes; i++) {
        fprintf(f, "%d %d\n", i, label[i]);
        for (int j = (int)row_start[i]; j < (int)row_start[i + 1]; j++) {
            uint32_t d = edge_dst[j];
            fprintf(f, "\te %d: %d %d %d\n", j, (int)d, edge_data ? edge_data[j] : 0, label[d]);
        }
    }
    return fclose(f) ? -2 : 0;
}

/* ------------------------------------------------------------------ */
/* PageRank by residual push (apps/pr/kernel.cu).  Constants and the    */
/* mixed float/double arithmetic of the reference:                      */
/*   rank[v]  = 1.0 - ALPHA                          (init_1, :37)      */
/*   res[dst] += (float)(1.0 / outdeg(v)) per edge    (:38-45)           */
/*   res[v]  *= (1.0 - ALPHA) * ALPHA, in double      (init_2, :60)      */
/* then every vertex is in the first worklist, and each worklist vertex */
/* u takes r = res[u], res[u] = 0, rank[u] += r, and pushes             */
/* r * ALPHA / outdeg(u) to each neighbour; a neighbour whose residual  */
/* crosses EPSILON from below joins the next worklist (:140-143,        */
/* :184-192).  Worklists are processed level by level, each in order.  */
/* Returns the number of iterations (worklists processed); the edges   */
/* pushed along go to *edges_pushed when it is not NULL.                */
/* ------------------------------------------------------------------ */
#define ORC_PR_ALPHA 0.85f
#define ORC_PR_EPSILON 0.000001f

int64_t orc_pr(uint32_t nnodes, const uint32_t *row_start, const uint32_t *edge_dst, int64_t max_iterations,
               float *rank, uint64_t *edges_pushed)
{
    uint64_t pushed = 0;
    float *res = (float *)calloc(nnodes ? nnodes : 1, sizeof(float));
    uint32_t *cur = (uint32_t *)malloc((size_t)(nnodes ? nnodes : 1) * 4);
    uint32_t *nxt = (uint32_t *)malloc((size_t)(nnodes ? nnodes : 1) * 4);
    for (uint32_t v = 0; v < nnodes; v++) rank[v] = (float)(1.0 - (double)ORC_PR_ALPHA);
    for (uint32_t v = 0; v < nnodes; v++) {
        uint32_t deg = row_start[v + 1] - row_start[v];
        if (!deg) continue;
        float upd = (float)(1.0 / deg);
        for (uint32_t e = row_start[v]; e < row_start[v + 1]; e++) res[edge_dst[e]] += upd;
    }
    for (uint32_t v = 0; v < nnodes; v++)
        res[v] = (float)((double)res[v] * ((1.0 - (double)ORC_PR_ALPHA) * (double)ORC_PR_ALPHA));
    size_t ncur = 0;
    for (uint32_t v = 0; v < nnodes; v++) cur[ncur++] = v;
    int64_t iter = 0;
    while (ncur && iter < max_iterations) {
        size_t nn = 0;
        for (size_t i = 0; i < ncur; i++) {
            uint32_t u = cur[i];
            float r = res[u];
            res[u] = 0;
            rank[u] += r;
            uint32_t deg = row_start[u + 1] - row_start[u];
            if (!deg) continue;
            float upd = r * ORC_PR_ALPHA / (float)deg;
            pushed += deg;
            for (uint32_t e = row_start[u]; e < row_start[u + 1]; e++) {
                uint32_t d = edge_dst[e];
                float prev = res[d];
                float now = prev + upd;
                res[d] = now;
                if (now > ORC_PR_EPSILON && prev < ORC_PR_EPSILON) nxt[nn++] = d;
            }
        }
        uint32_t *t = cur; cur = nxt; nxt = t;
        ncur = nn;
        iter++;
    }
    free(res); free(cur); free(nxt);
    if (edges_pushed) *edges_pushed = pushed;
    return iter;
}

/* PageRank output (apps/pr/support.cu:95-101): "%d %f\n" per node. */
int orc_write_pr_output(const char *path, uint32_t nnodes, const float *rank)
{
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    for (int i = 0; i < (int)nnodes; i++) fprintf(f, "%d %f\n", i, (double)rank[i]);
    return fclose(f) ? -2 : 0;
}

/* ---------------------------------------------------------------------- */
/* Maximal independent set (apps/mis).                                     */
/*                                                                        */
/* Priorities (apps/mis/kernel.cu:18-41): thread t of a launch of          */
/* `nthreads` threads runs Marsaglia's xorshift128 from the state          */
/* (SEED1..SEED4) ^ t and gives its k-th output to vertex t + k*nthreads.   */
/* The reference launches it with kernel_sizing's grid (skelapp/skel.cu:   */
/* 37-43): 8 CTAs per SM of 256 threads.                                   */
/*                                                                        */
/* Rounds (:151-169): every vertex still on the worklist is MARKED when no */
/* out-neighbour other than itself that is not NON_INDEPENDENT beats it in */
/* (priority, id) order (:65-103, unsigned priorities, larger id wins a     */
/* tie); then every worklist vertex that is MARKED, or has a MARKED         */
/* out-neighbour, leaves the worklist, and an unmarked one becomes          */
/* NON_INDEPENDENT (:104-149).  Marking reads only states fixed before the */
/* round (a vertex marked in the same round is still not NON_INDEPENDENT), */
/* so the result does not depend on the schedule.  Returns the rounds run;  */
/* state[v] ends 1 (in the set) or 2 (excluded), 0 only for n == 0.        */
/* ---------------------------------------------------------------------- */
#define ORC_MIS_UNMARKED 0
#define ORC_MIS_MARKED 1
#define ORC_MIS_NON_INDEPENDENT 2

void orc_mis_priorities(uint32_t nnodes, uint32_t nthreads, uint32_t *prio)
{
    for (uint32_t t = 0; t < nthreads && t < nnodes; t++) {
        uint32_t x = 0x12345678u ^ t, y = 0xabbdef12u ^ t, z = 0xcafe1234u ^ t, w = 0x09832516u ^ t;
        for (uint64_t v = t; v < nnodes; v += nthreads) {
            uint32_t tt = x ^ (x << 11);
            x = y;
            y = z;
            z = w;
            w = w ^ (w >> 19) ^ tt ^ (tt >> 8);
            prio[v] = w;
        }
    }
}

int64_t orc_mis(uint32_t nnodes, const uint32_t *row_start, const uint32_t *edge_dst, uint32_t nthreads,
                int32_t *state)
{
    uint32_t *prio = (uint32_t *)malloc((size_t)(nnodes ? nnodes : 1) * 4);
    uint32_t *cur = (uint32_t *)malloc((size_t)(nnodes ? nnodes : 1) * 4);
    uint32_t *nxt = (uint32_t *)malloc((size_t)(nnodes ? nnodes : 1) * 4);
    orc_mis_priorities(nnodes, nthreads, prio);
    for (uint32_t v = 0; v < nnodes; v++) state[v] = ORC_MIS_UNMARKED;
    size_t ncur = 0;
    for (uint32_t v = 0; v < nnodes; v++) cur[ncur++] = v;
    int64_t steps = 0;
    while (ncur) {
        /* mark: decisions read states fixed before this pass */
        for (size_t i = 0; i < ncur; i++) {
            uint32_t u = cur[i], best = prio[u], best_id = u;
            for (uint32_t e = row_start[u]; e < row_start[u + 1]; e++) {
                uint32_t d = edge_dst[e];
                if (d == u || state[d] == ORC_MIS_NON_INDEPENDENT) continue;
                if (prio[d] > best || (prio[d] == best && d > best_id)) {
                    best = prio[d];
                    best_id = d;
                }
            }
            if (best_id == u) nxt[i] = 1;
            else nxt[i] = 0;
        }
        for (size_t i = 0; i < ncur; i++)
            if (nxt[i]) state[cur[i]] = ORC_MIS_MARKED;
        /* drop */
        size_t nn = 0;
        for (size_t i = 0; i < ncur; i++) {
            uint32_t u = cur[i];
            int drop = state[u] == ORC_MIS_MARKED;
            for (uint32_t e = row_start[u]; !drop && e < row_start[u + 1]; e++)
                if (state[edge_dst[e]] == ORC_MIS_MARKED) drop = 1;
            if (!drop) nxt[nn++] = u;
            else if (state[u] == ORC_MIS_UNMARKED) state[u] = ORC_MIS_NON_INDEPENDENT;
        }
        uint32_t *t = cur;
        cur = nxt;
        nxt = t;
        ncur = nn;
        steps++;
    }
    free(prio); free(cur); free(nxt);
    return steps;
}

/* MIS output (apps/mis/support.cu:18-40): the set's size, then its ids. */
int orc_write_mis_output(const char *path, uint32_t nnodes, const int32_t *state)
{
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    unsigned count = 0;
    for (uint32_t i = 0; i < nnodes; i++) count += state[i] == ORC_MIS_MARKED;
    fprintf(f, "%u\n", count);
    for (int i = 0; i < (int)nnodes; i++)
        if (state[i] == ORC_MIS_MARKED) fprintf(f, "%d\n", i);
    return fclose(f) ? -2 : 0;
}
