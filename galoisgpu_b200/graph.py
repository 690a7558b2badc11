"""Python host API of the traversal engine, mirroring the reference's
interface for the BFS / SSSP path.

Reference counterparts (paths within the reference project):

* :class:`CSRGraph` -- ``CSRGraph`` (rt/include/csr_graph.h:27-103) with its
  accessors ``getOutDegree``/``getFirstEdge``/``getAbsDestination``/
  ``getAbsWeight`` and ``read`` (rt/src/csr_graph.cu:152-241);
  ``copy_to_gpu`` (rt/src/csr_graph.cu:250-261) returns a :class:`DeviceGraph`.
* :meth:`Engine.bfs` / :meth:`Engine.sssp` -- ``gg_main`` of apps/bfs
  (apps/bfs/kernel.cu:380-393) and apps/sssp (apps/sssp/kernel.cu:455-480):
  ``start_node`` (apps/bfs/support.cu:10) and ``delta`` (the ``-d`` option,
  apps/sssp/support.cu:56, default 10000) have the same meaning; the result
  is the reference's ``node_data`` array (int32, ``INF`` = INT_MAX).
* :func:`output` -- ``output`` (apps/bfs/support.cu:27-45).

Every traversal runs in libgft.so on the GPU; nothing here computes a
result on the CPU.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import GFT_INF, GFT_NO_PARENT, BatchStats, Csr, GenParams, Query, Stats, Tuning, check, load

INF = GFT_INF  # apps/bfs/kernel.cu:16, apps/sssp/kernel.cu:18
DEFAULT_DELTA = 10000  # apps/sssp/support.cu:56

# Graph500 R-MAT probabilities in parts per 2^32.
RMAT_A = round(0.57 * 2**32)
RMAT_B = round(0.19 * 2**32)
RMAT_C = round(0.19 * 2**32)


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _i32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _take_csr(csr: Csr) -> tuple[np.ndarray, np.ndarray, np.ndarray | None]:
    """Copies a library-allocated gft_csr into numpy arrays and frees it."""
    lib = load()
    try:
        n, m = csr.nnodes, csr.nedges
        rs = np.ctypeslib.as_array(csr.row_start, shape=(n + 1,)).copy()
        dst = np.ctypeslib.as_array(csr.edge_dst, shape=(max(m, 1),))[:m].copy()
        w = None
        if csr.edge_data:
            w = np.ctypeslib.as_array(csr.edge_data, shape=(max(m, 1),))[:m].copy()
        return rs, dst, w
    finally:
        lib.gft_csr_free(C.byref(csr))


class CSRGraph:
    """Host CSR graph: uint32 ``row_start`` (nnodes+1), uint32 ``edge_dst``,
    optional int32 ``edge_data`` (None for an unweighted graph)."""

    def __init__(self, row_start, edge_dst, edge_data=None):
        self.row_start = np.ascontiguousarray(row_start, dtype=np.uint32)
        self.edge_dst = np.ascontiguousarray(edge_dst, dtype=np.uint32)
        self.edge_data = None if edge_data is None else np.ascontiguousarray(edge_data, dtype=np.int32)
        if self.row_start.ndim != 1 or len(self.row_start) < 1:
            raise ValueError("row_start must have nnodes + 1 entries")
        if int(self.row_start[-1]) != len(self.edge_dst):
            raise ValueError("row_start[nnodes] must equal the number of edges")
        if self.edge_data is not None and len(self.edge_data) != len(self.edge_dst):
            raise ValueError("edge_data must have one entry per edge")

    # -- reference-style accessors (rt/include/csr_graph.h:52-94) ----------
    @property
    def nnodes(self) -> int:
        return len(self.row_start) - 1

    @property
    def nedges(self) -> int:
        return len(self.edge_dst)

    @property
    def weighted(self) -> bool:
        return self.edge_data is not None

    def getOutDegree(self, src: int) -> int:
        return int(self.row_start[src + 1]) - int(self.row_start[src])

    def getFirstEdge(self, src: int) -> int:
        return int(self.row_start[src])

    def getAbsDestination(self, abs_edge: int) -> int:
        return int(self.edge_dst[abs_edge])

    def getAbsWeight(self, abs_edge: int) -> int:
        return 0 if self.edge_data is None else int(self.edge_data[abs_edge])

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_start.astype(np.int64))

    # -- C struct view -------------------------------------------------------
    def _csr(self) -> Csr:
        c = Csr()
        c.nnodes = self.nnodes
        c.nedges = self.nedges
        c.row_start = _u32p(self.row_start)
        c.edge_dst = _u32p(self.edge_dst)
        c.edge_data = _i32p(self.edge_data) if self.edge_data is not None else C.POINTER(C.c_int32)()
        return c

    # -- .gr files -------------------------------------------------------------
    @classmethod
    def read(cls, path: str | Path) -> "CSRGraph":
        """Parses a .gr v1 file (rt/src/csr_graph.cu:152-241)."""
        csr = Csr()
        check(load().gft_gr_read(str(path).encode(), C.byref(csr)))
        return cls(*_take_csr(csr))

    @classmethod
    def read_chunked(cls, path: str | Path) -> "CSRGraph":
        """The same parse through the parallel chunked reader that
        DeviceGraph.load_gr uses, into host arrays."""
        csr = Csr()
        check(load().gft_gr_read_chunked(str(path).encode(), C.byref(csr)))
        return cls(*_take_csr(csr))

    def write(self, path: str | Path) -> None:
        c = self._csr()
        check(load().gft_gr_write(str(path).encode(), C.byref(c)))

    # -- seeded synthetic graphs ----------------------------------------------
    @classmethod
    def grid(cls, rows: int, cols: int, seed: int = 0, max_weight: int = 1) -> "CSRGraph":
        csr = Csr()
        check(load().gft_gen_grid(rows, cols, seed, max_weight, C.byref(csr)))
        return cls(*_take_csr(csr))._mark_symmetric()

    @classmethod
    def road(cls, side: int, seed: int = 1, delete_ppm: int = 50000, shortcut_ppm: int = 1000,
             max_weight: int = 10000) -> "CSRGraph":
        csr = Csr()
        check(load().gft_gen_road(side, seed, delete_ppm, shortcut_ppm, max_weight, C.byref(csr)))
        return cls(*_take_csr(csr))._mark_symmetric()

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, seed: int = 1, max_weight: int = 0,
             a: int = RMAT_A, b: int = RMAT_B, c: int = RMAT_C) -> "CSRGraph":
        csr = Csr()
        check(load().gft_gen_rmat(scale, edge_factor, a, b, c, seed, max_weight, C.byref(csr)))
        return cls(*_take_csr(csr))._mark_symmetric()

    # The generators emit both directions of every edge.  A graph read from
    # a file or built from arrays is marked only by the caller (symmetric =
    # True), and only when every edge u->v has v->u.
    symmetric = False

    def _mark_symmetric(self) -> "CSRGraph":
        self.symmetric = True
        return self

    def pick_sources(self, seed: int, k: int) -> list[int]:
        out = (C.c_uint32 * k)()
        c = self._csr()
        check(load().gft_pick_sources(C.byref(c), seed, k, out))
        return list(out)

    def copy_to_gpu(self, device: int = 0, stream=None) -> "DeviceGraph":
        c = self._csr()
        h = C.c_void_p()
        check(load().gft_graph_upload(device, C.byref(c), _stream_ptr(stream), C.byref(h)))
        d = DeviceGraph(h, device)
        if self.symmetric:
            d.symmetric = True
        return d


def _stream_ptr(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(int(stream.cuda_stream))


class DeviceGraph:
    """A graph resident in device memory (owned by libgft)."""

    def __init__(self, handle: C.c_void_p, device: int):
        self._h = handle
        self.device = device
        n, m, w = C.c_uint32(), C.c_uint32(), C.c_int()
        check(load().gft_graph_info(self._h, C.byref(n), C.byref(m), C.byref(w)))
        self.nnodes, self.nedges, self.weighted = n.value, m.value, bool(w.value)

    @classmethod
    def generate(cls, kind: str, device: int = 0, seed: int = 1, stream=None, **kw) -> "DeviceGraph":
        """Builds a seeded synthetic graph directly on the device; same graph
        as the matching :class:`CSRGraph` constructor."""
        p = GenParams()
        p.seed = seed
        if kind == "grid":
            p.kind, p.rows, p.cols = 0, kw["rows"], kw["cols"]
            p.max_weight = kw.get("max_weight", 1)
        elif kind == "road":
            p.kind, p.rows = 1, kw["side"]
            p.delete_ppm = kw.get("delete_ppm", 50000)
            p.shortcut_ppm = kw.get("shortcut_ppm", 1000)
            p.max_weight = kw.get("max_weight", 10000)
        elif kind == "rmat":
            p.kind, p.scale = 2, kw["scale"]
            p.edge_factor = kw.get("edge_factor", 16)
            p.a_q32, p.b_q32, p.c_q32 = kw.get("a", RMAT_A), kw.get("b", RMAT_B), kw.get("c", RMAT_C)
            p.max_weight = kw.get("max_weight", 0)
        else:
            raise ValueError(f"unknown graph kind {kind!r}")
        h = C.c_void_p()
        check(load().gft_graph_generate(device, C.byref(p), _stream_ptr(stream), C.byref(h)))
        return cls(h, device)

    @classmethod
    def load_gr(cls, path: str | Path, device: int = 0, stream=None) -> "DeviceGraph":
        """Reads a .gr file straight into device memory (parallel chunked
        reads into pinned staging, overlapped with the copies); replaces
        CSRGraph::read + copy_to_gpu (rt/src/csr_graph.cu:152-261)."""
        h = C.c_void_p()
        check(load().gft_graph_load_gr(device, str(path).encode(), _stream_ptr(stream), C.byref(h)))
        return cls(h, device)

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise ValueError("graph was freed")
        return self._h

    @property
    def symmetric(self) -> bool:
        """Whether BFS may run bottom-up levels (gft_graph_set_symmetric)."""
        v = C.c_int()
        check(load().gft_graph_is_symmetric(self.handle, C.byref(v)))
        return bool(v.value)

    @symmetric.setter
    def symmetric(self, value: bool) -> None:
        check(load().gft_graph_set_symmetric(self.handle, 1 if value else 0))

    def arrays(self) -> tuple[int, int, int]:
        rs, dst, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(load().gft_graph_arrays(self.handle, C.byref(rs), C.byref(dst), C.byref(w)))
        return rs.value or 0, dst.value or 0, w.value or 0

    def pick_sources(self, seed: int, k: int) -> list[int]:
        """Same draw as CSRGraph.pick_sources, reading only row_start."""
        out = (C.c_uint32 * k)()
        check(load().gft_graph_pick_sources(self.handle, seed, k, out))
        return list(out)

    def download(self) -> CSRGraph:
        csr = Csr()
        check(load().gft_graph_download(self.handle, C.byref(csr)))
        return CSRGraph(*_take_csr(csr))

    def free(self) -> None:
        if self._h is not None:
            load().gft_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


@dataclass
class Tune:
    """Per-query tunables (zero = engine default)."""

    block_threads: int = 0
    blocks_per_sm: int = 0
    hub_degree: int = 0
    timeout_ms: int = 0
    test_skip_block: int = -1
    max_blocks: int = 0
    group_blocks: int = 0
    group_min_nodes: int = 0
    direction: int = 0  # BFS: 0 = direction-optimising on graphs marked symmetric, 1 = top-down only
    cta_small: int = 0  # SSSP on the grid: iterations up to this many vertices on one CTA (0 = default, 2**32-1 = never)
    fuse_budget: int = 0  # SSSP: near vertices a warp expands in the iteration that found them (0 = default, 2**32-1 = never)
    queue_tile: int = 0  # grid kernels: push-buffer entries per warp, 64 / 128 / 256 (0 = default)
    warp_degree: int = 0  # vertices of at least this many edges are expanded by a whole warp (0 = 32)

    def c(self) -> Tuning:
        return Tuning(self.block_threads, self.blocks_per_sm, self.hub_degree, self.timeout_ms, self.test_skip_block,
                      self.max_blocks, self.group_blocks, self.group_min_nodes, self.direction, self.cta_small,
                      self.fuse_budget, self.queue_tile, self.warp_degree)


class Engine:
    """Per-device traversal engine; owns the traversal scratch.  Calls on one
    engine are serialised; use one engine per thread for concurrency."""

    def __init__(self, device: int = 0):
        self.device = device
        h = C.c_void_p()
        check(load().gft_engine_create(device, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            load().gft_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def scratch_bytes(self) -> int:
        return int(load().gft_engine_scratch_bytes(self._h))

    @staticmethod
    def _tune(tune):
        if tune is None:
            return None
        return C.byref(tune.c() if isinstance(tune, Tune) else tune)

    def bfs(self, graph: DeviceGraph, start_node: int = 0, out=None, parent=None, tune: Tune | None = None,
            stream=None) -> dict:
        """BFS levels into the int32 device tensor ``out`` (allocated when
        None); optional uint32-sized ``parent`` tensor.  Returns the stats."""
        import torch

        dev = torch.device("cuda", graph.device)
        if out is None:
            out = torch.empty(graph.nnodes, dtype=torch.int32, device=dev)
        st = Stats()
        check(
            load().gft_bfs(
                self._h, graph.handle, start_node, C.c_void_p(out.data_ptr()),
                C.c_void_p(parent.data_ptr() if parent is not None else 0), self._tune(tune),
                _stream_ptr(stream if stream is not None else torch.cuda.current_stream(dev)), C.byref(st),
            )
        )
        return {"out": out, "parent": parent, **st.as_dict()}

    def sssp(self, graph: DeviceGraph, start_node: int = 0, delta: int = DEFAULT_DELTA, out=None, parent=None,
             tune: Tune | None = None, stream=None) -> dict:
        import torch

        dev = torch.device("cuda", graph.device)
        if out is None:
            out = torch.empty(graph.nnodes, dtype=torch.int32, device=dev)
        st = Stats()
        check(
            load().gft_sssp(
                self._h, graph.handle, start_node, delta, C.c_void_p(out.data_ptr()),
                C.c_void_p(parent.data_ptr() if parent is not None else 0), self._tune(tune),
                _stream_ptr(stream if stream is not None else torch.cuda.current_stream(dev)), C.byref(st),
            )
        )
        return {"out": out, "parent": parent, **st.as_dict()}

    def msbfs(self, graph: DeviceGraph, sources: list[int], max_levels: int = 32, symmetric: bool = False,
              planes=None, stream=None) -> dict:
        """Multi-source BFS of up to 256 sources; returns the frontier planes
        (a uint32 device tensor) and stats.  levels(i) gives source i's
        int32 levels."""
        import torch

        k = len(sources)
        plane = load().gft_msbfs_plane_bytes(graph.nnodes, k)
        if planes is None:
            planes = torch.empty(max_levels * plane // 4, dtype=torch.int32, device=f"cuda:{graph.device}")
        src = (C.c_uint32 * k)(*sources)
        st = Stats()
        dev = torch.device("cuda", graph.device)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        check(load().gft_msbfs(self._h, graph.handle, src, k, C.c_void_p(planes.data_ptr()), max_levels,
                               1 if symmetric else 0, _stream_ptr(s), C.byref(st)))
        res = {"planes": planes, "k": k, **st.as_dict()}

        def levels(i: int, out=None):
            if out is None:
                out = torch.empty(graph.nnodes, dtype=torch.int32, device=dev)
            check(load().gft_msbfs_levels(C.c_void_p(planes.data_ptr()), graph.nnodes, k, st.levels, i,
                                          C.c_void_p(out.data_ptr()), _stream_ptr(s)))
            return out

        res["levels_of"] = levels
        return res

    def cc(self, graph: DeviceGraph, out=None, tune: Tune | None = None, stream=None) -> dict:
        """Connected components (apps/cc): ``out[v]`` (int32 device tensor)
        becomes the smallest vertex id of v's weakly connected component.
        Returns the stats plus ``components``."""
        import torch

        dev = torch.device("cuda", graph.device)
        if out is None:
            out = torch.empty(graph.nnodes, dtype=torch.int32, device=dev)
        st, comps = Stats(), C.c_uint64()
        check(load().gft_cc(self._h, graph.handle, C.c_void_p(out.data_ptr()), self._tune(tune),
                            _stream_ptr(stream if stream is not None else torch.cuda.current_stream(dev)),
                            C.byref(st), C.byref(comps)))
        return {"out": out, "components": comps.value, **st.as_dict()}

    def cc_host(self, graph: DeviceGraph, out: np.ndarray, tune: Tune | None = None, stream=None) -> dict:
        """Connected components into a host int32 array (end to end)."""
        st, comps = Stats(), C.c_uint64()
        check(load().gft_cc_host(self._h, graph.handle, C.c_void_p(out.ctypes.data), self._tune(tune),
                                 _stream_ptr(stream), C.byref(st), C.byref(comps)))
        return {"components": comps.value, **st.as_dict()}

    def pr(self, graph: DeviceGraph, out=None, max_iterations: int = 0xFFFFFFFF, tune: Tune | None = None,
           stream=None) -> dict:
        """PageRank by residual push (apps/pr): ``out`` (float32 device tensor)
        receives the unnormalised ranks; ``levels`` = worklist rounds run."""
        import torch

        dev = torch.device("cuda", graph.device)
        if out is None:
            out = torch.empty(graph.nnodes, dtype=torch.float32, device=dev)
        st = Stats()
        check(load().gft_pr(self._h, graph.handle, C.c_void_p(out.data_ptr()), max_iterations, self._tune(tune),
                            _stream_ptr(stream if stream is not None else torch.cuda.current_stream(dev)),
                            C.byref(st)))
        return {"out": out, **st.as_dict()}

    def pr_host(self, graph: DeviceGraph, out: np.ndarray, max_iterations: int = 0xFFFFFFFF,
                tune: Tune | None = None, stream=None) -> dict:
        """PageRank into a host float32 array (end to end)."""
        st = Stats()
        check(load().gft_pr_host(self._h, graph.handle, C.c_void_p(out.ctypes.data), max_iterations,
                                 self._tune(tune), _stream_ptr(stream), C.byref(st)))
        return st.as_dict()

    def mis(self, graph: DeviceGraph, out=None, prio_threads: int = 0, tune: Tune | None = None, stream=None) -> dict:
        """Maximal independent set (apps/mis): ``out`` (int32 device tensor)
        receives the reference's node_data, 1 = in the set, 2 = excluded.
        ``prio_threads`` = 0 uses the reference's priority streams on this
        device (8 CTAs of 256 threads per SM).  ``levels`` = rounds,
        ``vertices_reached`` = the set's size."""
        import torch

        dev = torch.device("cuda", graph.device)
        if out is None:
            out = torch.empty(graph.nnodes, dtype=torch.int32, device=dev)
        st = Stats()
        check(load().gft_mis(self._h, graph.handle, C.c_void_p(out.data_ptr()), prio_threads, self._tune(tune),
                             _stream_ptr(stream if stream is not None else torch.cuda.current_stream(dev)),
                             C.byref(st)))
        return {"out": out, **st.as_dict()}

    def mis_host(self, graph: DeviceGraph, out: np.ndarray, prio_threads: int = 0, tune: Tune | None = None,
                 stream=None) -> dict:
        """Maximal independent set into a host int32 array (end to end)."""
        st = Stats()
        check(load().gft_mis_host(self._h, graph.handle, C.c_void_p(out.ctypes.data), prio_threads,
                                  self._tune(tune), _stream_ptr(stream), C.byref(st)))
        return st.as_dict()

    def bfs_host(self, graph: DeviceGraph, start_node: int, out: np.ndarray, parent: np.ndarray | None = None,
                 tune: Tune | None = None, stream=None) -> dict:
        """End-to-end query with host result buffers (int32 / uint32 numpy)."""
        st = Stats()
        check(
            load().gft_bfs_host(
                self._h, graph.handle, start_node, C.c_void_p(out.ctypes.data),
                C.c_void_p(parent.ctypes.data if parent is not None else 0), self._tune(tune),
                _stream_ptr(stream), C.byref(st),
            )
        )
        return st.as_dict()

    def sssp_host(self, graph: DeviceGraph, start_node: int, out: np.ndarray, delta: int = DEFAULT_DELTA,
                  parent: np.ndarray | None = None, tune: Tune | None = None, stream=None) -> dict:
        st = Stats()
        check(
            load().gft_sssp_host(
                self._h, graph.handle, start_node, delta, C.c_void_p(out.ctypes.data),
                C.c_void_p(parent.ctypes.data if parent is not None else 0), self._tune(tune),
                _stream_ptr(stream), C.byref(st),
            )
        )
        return st.as_dict()

    def _host_many(self, app: str, graph: DeviceGraph, sources, out: np.ndarray, delta: int, tune: Tune | None,
                   stream) -> list[dict]:
        src = np.ascontiguousarray(np.asarray(sources, dtype=np.uint32))
        k = len(src)
        if out.dtype != np.int32 or not out.flags["C_CONTIGUOUS"] or out.size < k * graph.nnodes:
            raise ValueError(f"out must be a C-contiguous int32 array of at least {k} x {graph.nnodes} entries")
        stats = (Stats * max(k, 1))()
        args = [self._h, graph.handle, C.c_void_p(src.ctypes.data), k]
        args += [delta] if app == "sssp" else []
        args += [C.c_void_p(out.ctypes.data), self._tune(tune), _stream_ptr(stream), C.cast(stats, C.c_void_p)]
        check(getattr(load(), f"gft_{app}_host_many")(*args))
        return [stats[i].as_dict() for i in range(k)]

    def bfs_host_many(self, graph: DeviceGraph, sources, out: np.ndarray, tune: Tune | None = None,
                      stream=None) -> list[dict]:
        """BFS from each of `sources` into the rows of the host array `out`
        (k x nnodes int32; pinned memory lets each query's copy back overlap
        the next query).  Row i equals bfs_host from sources[i].  Returns the
        per-query stats."""
        return self._host_many("bfs", graph, sources, out, 0, tune, stream)

    def sssp_host_many(self, graph: DeviceGraph, sources, out: np.ndarray, delta: int = DEFAULT_DELTA,
                       tune: Tune | None = None, stream=None) -> list[dict]:
        """SSSP from each of `sources` into the rows of the host array `out`,
        as bfs_host_many."""
        return self._host_many("sssp", graph, sources, out, delta, tune, stream)


class Batch:
    """Many queries in one persistent launch, replayed as a CUDA graph
    (gft_batch_*).  `queries` are dicts with keys graph, app ('bfs' or
    'sssp'), src, optional delta, out (int32 device tensor, allocated when
    absent) and parent (BFS only)."""

    def __init__(self, engine: "Engine", queries: list[dict], tune: Tune | None = None):
        import torch

        self.engine = engine
        self.queries = []
        self._keep = []
        arr = (Query * len(queries))()
        for i, q in enumerate(queries):
            g: DeviceGraph = q["graph"]
            out = q.get("out")
            if out is None:
                out = torch.empty(g.nnodes, dtype=torch.int32, device=f"cuda:{g.device}")
            par = q.get("parent")
            arr[i].graph = g.handle
            arr[i].app = 1 if q["app"] == "sssp" else 0
            arr[i].src = q["src"]
            arr[i].delta = q.get("delta", DEFAULT_DELTA) if q["app"] == "sssp" else 0
            arr[i].d_out = out.data_ptr()
            arr[i].d_parent = par.data_ptr() if par is not None else None
            self.queries.append({**q, "out": out, "parent": par})
            self._keep += [g, out, par]
        self._arr = arr
        h = C.c_void_p()
        check(load().gft_batch_create(engine._h, arr, len(queries), engine._tune(tune), C.byref(h)))
        self._h = h

    def set_source(self, i: int, src: int) -> None:
        check(load().gft_batch_set_source(self._h, i, src))
        self.queries[i]["src"] = src

    def submit(self, stream=None) -> None:
        import torch

        dev = self.queries[0]["graph"].device
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        check(load().gft_batch_submit(self._h, _stream_ptr(s)))

    def wait(self) -> dict:
        st = BatchStats()
        check(load().gft_batch_wait(self._h, self._arr, C.byref(st)))
        for i, q in enumerate(self.queries):
            a = self._arr[i]
            q.update(status=a.status, levels=a.levels, iterations=a.iterations, edges_scanned=a.edges_scanned,
                     device_ms=a.device_ms)
        return st.as_dict()

    def run(self, stream=None) -> dict:
        self.submit(stream)
        return self.wait()

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            load().gft_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reach_stats(graph: DeviceGraph, values, stream=None) -> tuple[int, int]:
    """(V_r, E_r) of a device result tensor."""
    vr, er = C.c_uint64(), C.c_uint64()
    check(load().gft_reach_stats(graph.handle, C.c_void_p(values.data_ptr()), _stream_ptr(stream),
                                 C.byref(vr), C.byref(er)))
    return vr.value, er.value


def output(path: str | Path, values: np.ndarray) -> None:
    """Writes ``"%d %d"`` / ``"%d INF"`` lines (apps/bfs/support.cu:27-45)."""
    v = np.ascontiguousarray(values, dtype=np.int32)
    check(load().gft_write_output(str(path).encode(), len(v), C.c_void_p(v.ctypes.data)))


def output_gz(path: str | Path, values: np.ndarray, level: int = 1) -> None:
    """The text of :func:`output`, gzip-compressed in parallel blocks (one
    gzip member per 2^20 lines; readable as one stream by any gzip reader)."""
    v = np.ascontiguousarray(values, dtype=np.int32)
    check(load().gft_write_output_gz(str(path).encode(), len(v), C.c_void_p(v.ctypes.data), level))


def write_node_data(path: str | Path, values: np.ndarray) -> None:
    """Binary dump of a result array (int32 levels/distances/labels/states,
    or float32 ranks) behind a 24-byte header."""
    v = np.ascontiguousarray(values)
    if v.dtype == np.float32:
        kind = 1
    else:
        v, kind = np.ascontiguousarray(v, dtype=np.int32), 0
    check(load().gft_write_node_data(str(path).encode(), len(v), C.c_void_p(v.ctypes.data), kind))


def read_node_data(path: str | Path) -> np.ndarray:
    """Reads a dump written by :func:`write_node_data` (or the CLI's -b)."""
    n, kind = C.c_uint32(), C.c_uint32()
    check(load().gft_read_node_data(str(path).encode(), C.byref(n), C.byref(kind), None))
    out = np.empty(n.value, dtype=np.float32 if kind.value == 1 else np.int32)
    check(load().gft_read_node_data(str(path).encode(), C.byref(n), C.byref(kind), C.c_void_p(out.ctypes.data)))
    return out


def write_cc_output(path: str | Path, graph: CSRGraph, labels: np.ndarray) -> None:
    """CC labels in the reference's format: a node line and one line per
    out-edge (apps/cc/support.cu:16-36)."""
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    c = graph._csr()
    check(load().gft_write_cc_output(str(path).encode(), C.byref(c), C.c_void_p(lab.ctypes.data)))


def write_pr_output(path: str | Path, ranks: np.ndarray) -> None:
    """Ranks as the reference writes them: "%d %f" per node
    (apps/pr/support.cu:95-101)."""
    r = np.ascontiguousarray(ranks, dtype=np.float32)
    check(load().gft_write_pr_output(str(path).encode(), len(r), C.c_void_p(r.ctypes.data)))


def write_mis_output(path: str | Path, state: np.ndarray) -> None:
    """The set as the reference writes it: its size, then one member id per
    line (apps/mis/support.cu:18-40)."""
    st = np.ascontiguousarray(state, dtype=np.int32)
    check(load().gft_write_mis_output(str(path).encode(), len(st), C.c_void_p(st.ctypes.data)))


__all__ = [
    "Batch",
    "CSRGraph",
    "DeviceGraph",
    "Engine",
    "Tune",
    "INF",
    "GFT_NO_PARENT",
    "DEFAULT_DELTA",
    "reach_stats",
    "output",
    "output_gz",
    "write_node_data",
    "read_node_data",
    "write_cc_output",
    "write_pr_output",
    "write_mis_output",
    "_lib",
]
