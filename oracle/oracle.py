"""ctypes binding of the CPU oracle (oracle/oracle.c -> oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's CPU-baseline leg.  The galoisgpu_b200 package
never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
INF = 0x7FFFFFFF
NO_PARENT = 0xFFFFFFFF

_lib = None


def build() -> Path:
    src = HERE / "oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        u32p, i32p = C.POINTER(C.c_uint32), C.POINTER(C.c_int32)
        lib.orc_gr_read.restype = C.c_int
        lib.orc_gr_read.argtypes = [C.c_char_p, u32p, u32p, C.POINTER(u32p), C.POINTER(u32p), C.POINTER(i32p)]
        lib.orc_free.argtypes = [C.c_void_p]
        lib.orc_bfs.restype = C.c_uint64
        lib.orc_bfs.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        lib.orc_sssp.restype = C.c_int64
        lib.orc_sssp.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        lib.orc_check_tree.restype = C.c_uint64
        lib.orc_check_tree.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                       C.c_void_p]
        lib.orc_reach_stats.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64),
                                        C.POINTER(C.c_uint64)]
        lib.orc_write_output.restype = C.c_int
        lib.orc_write_output.argtypes = [C.c_char_p, C.c_uint32, C.c_void_p]
        lib.orc_read_output.restype = C.c_int64
        lib.orc_read_output.argtypes = [C.c_char_p, C.c_uint32, C.c_void_p]
        lib.orc_cc.restype = C.c_uint64
        lib.orc_cc.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_pr.restype = C.c_int64
        lib.orc_pr.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.POINTER(C.c_uint64)]
        lib.orc_write_pr_output.restype = C.c_int
        lib.orc_write_pr_output.argtypes = [C.c_char_p, C.c_uint32, C.c_void_p]
        lib.orc_mis.restype = C.c_int64
        lib.orc_mis.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        lib.orc_mis_priorities.restype = None
        lib.orc_mis_priorities.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p]
        lib.orc_write_mis_output.restype = C.c_int
        lib.orc_write_mis_output.argtypes = [C.c_char_p, C.c_uint32, C.c_void_p]
        lib.orc_write_cc_output.restype = C.c_int
        lib.orc_write_cc_output.argtypes = [C.c_char_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = lib
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


def gr_read(path: str | os.PathLike):
    """Returns (row_start, edge_dst, edge_data or None); raises on a parse error."""
    lib = load()
    n, m = C.c_uint32(), C.c_uint32()
    rs, dst = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    w = C.POINTER(C.c_int32)()
    r = lib.orc_gr_read(str(path).encode(), C.byref(n), C.byref(m), C.byref(rs), C.byref(dst), C.byref(w))
    if r != 0:
        raise ValueError(f"oracle: cannot parse {path} (code {r})")
    try:
        a_rs = np.ctypeslib.as_array(rs, shape=(n.value + 1,)).copy()
        a_dst = np.ctypeslib.as_array(dst, shape=(max(m.value, 1),))[: m.value].copy()
        a_w = np.ctypeslib.as_array(w, shape=(max(m.value, 1),))[: m.value].copy() if w else None
    finally:
        lib.orc_free(C.cast(rs, C.c_void_p))
        lib.orc_free(C.cast(dst, C.c_void_p))
        if w:
            lib.orc_free(C.cast(w, C.c_void_p))
    return a_rs, a_dst, a_w


def bfs(row_start, edge_dst, src: int, parent: bool = False):
    rs = np.ascontiguousarray(row_start, dtype=np.uint32)
    dst = np.ascontiguousarray(edge_dst, dtype=np.uint32)
    n = len(rs) - 1
    level = np.empty(n, dtype=np.int32)
    par = np.empty(n, dtype=np.uint32) if parent else None
    load().orc_bfs(n, _p(rs), _p(dst), src, _p(level), _p(par))
    return (level, par) if parent else level


def sssp(row_start, edge_dst, edge_data, src: int, parent: bool = False):
    """Dijkstra; edge_data None means every weight is 0 (as the reference's
    calloc'd edge_data for an unweighted .gr)."""
    rs = np.ascontiguousarray(row_start, dtype=np.uint32)
    dst = np.ascontiguousarray(edge_dst, dtype=np.uint32)
    w = (np.zeros(len(dst), dtype=np.int32) if edge_data is None
         else np.ascontiguousarray(edge_data, dtype=np.int32))
    n = len(rs) - 1
    dist = np.empty(n, dtype=np.int32)
    par = np.empty(n, dtype=np.uint32) if parent else None
    r = load().orc_sssp(n, _p(rs), _p(dst), _p(w), src, _p(dist), _p(par))
    if r < 0:
        raise OverflowError("oracle: a shortest-path distance exceeds INT_MAX - 1")
    return (dist, par) if parent else dist


def check_tree(row_start, edge_dst, edge_data, src: int, values, parent) -> int:
    """Number of parent-tree violations (0 = valid); edge_data None = BFS."""
    rs = np.ascontiguousarray(row_start, dtype=np.uint32)
    dst = np.ascontiguousarray(edge_dst, dtype=np.uint32)
    w = None if edge_data is None else np.ascontiguousarray(edge_data, dtype=np.int32)
    v = np.ascontiguousarray(values, dtype=np.int32)
    p = np.ascontiguousarray(parent, dtype=np.uint32)
    return int(load().orc_check_tree(len(rs) - 1, _p(rs), _p(dst), _p(w), src, _p(v), _p(p)))


def reach_stats(row_start, values) -> tuple[int, int]:
    rs = np.ascontiguousarray(row_start, dtype=np.uint32)
    v = np.ascontiguousarray(values, dtype=np.int32)
    vr, er = C.c_uint64(), C.c_uint64()
    load().orc_reach_stats(len(rs) - 1, _p(rs), _p(v), C.byref(vr), C.byref(er))
    return vr.value, er.value


def write_output(path, values) -> None:
    v = np.ascontiguousarray(values, dtype=np.int32)
    if load().orc_write_output(str(path).encode(), len(v), _p(v)) != 0:
        raise OSError(f"oracle: cannot write {path}")


def read_output(path, nnodes: int) -> np.ndarray:
    v = np.full(nnodes, -1, dtype=np.int32)
    r = load().orc_read_output(str(path).encode(), nnodes, _p(v))
    if r != nnodes:
        raise ValueError(f"oracle: {path}: parsed {r} lines, expected {nnodes}")
    return v


def cc(row_start, edge_dst) -> tuple[np.ndarray, int]:
    """Connected components: (label per vertex = smallest vertex id of its
    component, number of components)."""
    rs = np.ascontiguousarray(row_start, dtype=np.uint32)
    dst = np.ascontiguousarray(edge_dst, dtype=np.uint32)
    n = len(rs) - 1
    label = np.empty(max(n, 1), dtype=np.int32)[:n]
    comps = load().orc_cc(n, _p(rs), _p(dst), _p(label))
    return label, int(comps)


def write_cc_output(path, row_start, edge_dst, edge_data, label) -> None:
    rs = np.ascontiguousarray(row_start, dtype=np.uint32)
    dst = np.ascontiguousarray(edge_dst, dtype=np.uint32)
    w = None if edge_data is None else np.ascontiguousarray(edge_data, dtype=np.int32)
    lab = np.ascontiguousarray(label, dtype=np.int32)
    rc = load().orc_write_cc_output(str(path).encode(), len(rs) - 1, _p(rs), _p(dst), _p(w) if w is not None else None,
                                    _p(lab))
    if rc != 0:
        raise OSError(f"orc_write_cc_output({path}) failed: {rc}")


def canonical_labels(label) -> np.ndarray:
    """Relabels a partition so every vertex carries the smallest vertex id of
    its class: the form in which partitions from different labelings (the
    reference's schedule-dependent roots, this oracle's minima) compare."""
    lab = np.asarray(label, dtype=np.int64)
    n = len(lab)
    first = np.full(max(n, int(lab.max()) + 1 if n else 0), n, dtype=np.int64)
    np.minimum.at(first, lab, np.arange(n, dtype=np.int64))
    return first[lab].astype(np.int32)


# The reference's MIS priority streams on a B200: kernel_sizing launches 8
# CTAs of 256 threads per SM (skelapp/skel.cu:37-43), 148 SMs.
MIS_THREADS_B200 = 8 * 148 * 256


def mis_priorities(nnodes: int, nthreads: int = MIS_THREADS_B200) -> np.ndarray:
    """apps/mis/kernel.cu:18-41: per-thread xorshift128 priorities."""
    out = np.empty(max(nnodes, 1), dtype=np.uint32)[:nnodes]
    load().orc_mis_priorities(nnodes, nthreads, _p(out))
    return out


def mis(row_start, edge_dst, nthreads: int = MIS_THREADS_B200) -> tuple[np.ndarray, int]:
    """Maximal independent set by the reference's rounds: (int32 state per
    vertex, 1 = in the set, 2 = excluded; rounds run)."""
    rs = np.ascontiguousarray(row_start, dtype=np.uint32)
    dst = np.ascontiguousarray(edge_dst, dtype=np.uint32)
    n = len(rs) - 1
    state = np.empty(max(n, 1), dtype=np.int32)[:n]
    steps = load().orc_mis(n, _p(rs), _p(dst), nthreads, _p(state))
    return state, int(steps)


def write_mis_output(path, state) -> None:
    st = np.ascontiguousarray(state, dtype=np.int32)
    if load().orc_write_mis_output(str(path).encode(), len(st), _p(st)) != 0:
        raise OSError(f"cannot write {path}")


def read_mis_output(path, nnodes: int) -> np.ndarray:
    """Parses the reference's MIS text (count, then member ids) into a
    membership mask; checks the count line."""
    lines = Path(path).read_text().split()
    count = int(lines[0])
    ids = np.array([int(x) for x in lines[1:]], dtype=np.int64)
    if len(ids) != count:
        raise ValueError(f"{path}: count line says {count}, {len(ids)} ids follow")
    mask = np.zeros(nnodes, dtype=bool)
    mask[ids] = True
    return mask


def pr(row_start, edge_dst, max_iterations: int = 2**62, stats: dict | None = None) -> tuple[np.ndarray, int]:
    """PageRank by residual push: (float32 rank per vertex, iterations); the
    edges pushed along go to stats["edges_pushed"] when stats is given."""
    rs = np.ascontiguousarray(row_start, dtype=np.uint32)
    dst = np.ascontiguousarray(edge_dst, dtype=np.uint32)
    n = len(rs) - 1
    rank = np.empty(max(n, 1), dtype=np.float32)[:n]
    pushed = C.c_uint64()
    it = load().orc_pr(n, _p(rs), _p(dst), max_iterations, _p(rank), C.byref(pushed))
    if stats is not None:
        stats["edges_pushed"] = pushed.value
    return rank, int(it)


def write_pr_output(path, rank) -> None:
    r = np.ascontiguousarray(rank, dtype=np.float32)
    rc = load().orc_write_pr_output(str(path).encode(), len(r), _p(r))
    if rc != 0:
        raise OSError(f"orc_write_pr_output({path}) failed: {rc}")


def read_pr_output(path, nnodes: int) -> np.ndarray:
    """Ranks from a reference PageRank output file ("%d %f" lines)."""
    rank = np.full(nnodes, np.nan, dtype=np.float64)
    with open(path) as f:
        for ln in f:
            i, v = ln.split()
            rank[int(i)] = float(v)
    return rank
