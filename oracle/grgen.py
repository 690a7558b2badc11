"""ctypes binding of oracle/libgrgen.so: the engine's seeded host
generators, built without the engine library, plus a .gr v1 writer.

TEST AND MEASUREMENT INFRASTRUCTURE ONLY: bench.py's reference arm uses it
to build the same seeded input graphs as the engine's arm and write them as
the .gr files the reference build reads, without loading libgft.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libgrgen.so"

# R-MAT quadrant probabilities a, b, c (Graph500) in parts per 2^32, as the
# engine's Python API passes them.
RMAT_ABC_Q32 = (round(0.57 * 2**32), round(0.19 * 2**32), round(0.19 * 2**32))


class _Csr(C.Structure):
    _fields_ = [("nnodes", C.c_uint32), ("nedges", C.c_uint32), ("row_start", C.POINTER(C.c_uint32)),
                ("edge_dst", C.POINTER(C.c_uint32)), ("edge_data", C.POINTER(C.c_int32))]


_lib = None


def load():
    global _lib
    if _lib is None:
        srcs = [HERE / "grgen.cpp", HERE.parent / "galoisgpu_b200" / "csrc" / "gen_host.cpp"]
        if not LIB.exists() or any(s.exists() and LIB.stat().st_mtime < s.stat().st_mtime for s in srcs):
            subprocess.run(["make", "-s", "-C", str(HERE), "libgrgen.so"], check=True)
        lib = C.CDLL(str(LIB))
        lib.gft_gen_grid.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(_Csr)]
        lib.gft_gen_road.argtypes = [C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(_Csr)]
        lib.gft_gen_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                     C.c_uint32, C.POINTER(_Csr)]
        lib.gft_pick_sources.argtypes = [C.POINTER(_Csr), C.c_uint64, C.c_uint32, C.POINTER(C.c_uint32)]
        lib.gft_csr_free.argtypes = [C.POINTER(_Csr)]
        lib.grgen_write_gr.argtypes = [C.c_char_p, C.POINTER(_Csr)]
        lib.grgen_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


class HostGraph:
    """A generated CSR graph held by libgrgen (freed with close())."""

    def __init__(self, csr: _Csr):
        self._c = csr

    @property
    def nnodes(self) -> int:
        return self._c.nnodes

    @property
    def nedges(self) -> int:
        return self._c.nedges

    @property
    def row_start(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._c.row_start, shape=(self.nnodes + 1,))

    @property
    def edge_dst(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._c.edge_dst, shape=(max(self.nedges, 1),))[: self.nedges]

    @property
    def edge_data(self) -> np.ndarray | None:
        if not self._c.edge_data:
            return None
        return np.ctypeslib.as_array(self._c.edge_data, shape=(max(self.nedges, 1),))[: self.nedges]

    def pick_sources(self, seed: int, k: int) -> list[int]:
        out = (C.c_uint32 * k)()
        _check(load().gft_pick_sources(C.byref(self._c), seed, k, out), "pick_sources")
        return list(out)

    def write_gr(self, path: str | os.PathLike) -> None:
        if load().grgen_write_gr(str(path).encode(), C.byref(self._c)) != 0:
            raise OSError(f"grgen: cannot write {path}")

    def close(self) -> None:
        if self._c.row_start:
            load().gft_csr_free(C.byref(self._c))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"grgen {what}: status {status}: {load().grgen_last_error().decode()}")


def generate(kind: str, seed: int, **kw) -> HostGraph:
    """kind 'grid' (rows, cols, max_weight=1), 'road' (side, max_weight=10000,
    delete_ppm=50000, shortcut_ppm=1000) or 'rmat' (scale, edge_factor,
    max_weight=0): the engine's generators with the engine's defaults."""
    lib, c = load(), _Csr()
    if kind == "grid":
        _check(lib.gft_gen_grid(kw["rows"], kw["cols"], seed, kw.get("max_weight", 1), C.byref(c)), "grid")
    elif kind == "road":
        _check(lib.gft_gen_road(kw["side"], seed, kw.get("delete_ppm", 50000), kw.get("shortcut_ppm", 1000),
                                kw.get("max_weight", 10000), C.byref(c)), "road")
    elif kind == "rmat":
        a, b, cq = RMAT_ABC_Q32
        _check(lib.gft_gen_rmat(kw["scale"], kw.get("edge_factor", 16), a, b, cq, seed, kw.get("max_weight", 0),
                                C.byref(c)), "rmat")
    else:
        raise ValueError(f"unknown graph kind {kind!r}")
    return HostGraph(c)
