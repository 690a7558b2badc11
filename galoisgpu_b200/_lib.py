"""ctypes binding of libgft.so (the C ABI declared in include/gft.h).

The library is built in-tree (``python -m galoisgpu_b200.build``).  Loading
fails loudly when it is missing: there is no Python or CPU fallback for any
traversal.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().with_name("libgft.so")

GFT_INF = 0x7FFFFFFF
GFT_NO_PARENT = 0xFFFFFFFF

STATUS_NAMES = {
    0: "GFT_OK",
    1: "GFT_ERR_INVALID_ARG",
    2: "GFT_ERR_IO",
    3: "GFT_ERR_FORMAT",
    4: "GFT_ERR_CUDA",
    5: "GFT_ERR_OOM",
    6: "GFT_ERR_TIMEOUT",
    7: "GFT_ERR_OVERFLOW",
    8: "GFT_ERR_NOT_SUPPORTED",
    9: "GFT_ERR_BUSY",
}


class GftError(RuntimeError):
    """A libgft call returned a non-zero gft_status."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, f"status {status}")
        super().__init__(f"{self.status_name}: {message}")


class Csr(C.Structure):
    _fields_ = [
        ("nnodes", C.c_uint32),
        ("nedges", C.c_uint32),
        ("row_start", C.POINTER(C.c_uint32)),
        ("edge_dst", C.POINTER(C.c_uint32)),
        ("edge_data", C.POINTER(C.c_int32)),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("levels", C.c_uint32),
        ("iterations", C.c_uint32),
        ("vertices_reached", C.c_uint64),
        ("edges_scanned", C.c_uint64),
        ("pushes", C.c_uint64),
        ("kernel_ms", C.c_float),
        ("grid_blocks", C.c_uint32),
        ("block_threads", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [
        ("block_threads", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("hub_degree", C.c_uint32),
        ("timeout_ms", C.c_uint32),
        ("test_skip_block", C.c_int32),
        ("max_blocks", C.c_uint32),
        ("group_blocks", C.c_uint32),
        ("group_min_nodes", C.c_uint32),
        ("direction", C.c_uint32),
        ("cta_small", C.c_uint32),
        ("fuse_budget", C.c_uint32),
        ("queue_tile", C.c_uint32),
        ("warp_degree", C.c_uint32),
    ]


class GenParams(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("rows", C.c_uint32),
        ("cols", C.c_uint32),
        ("scale", C.c_uint32),
        ("edge_factor", C.c_uint32),
        ("a_q32", C.c_uint32),
        ("b_q32", C.c_uint32),
        ("c_q32", C.c_uint32),
        ("delete_ppm", C.c_uint32),
        ("shortcut_ppm", C.c_uint32),
        ("max_weight", C.c_uint32),
        ("seed", C.c_uint64),
    ]


class Query(C.Structure):
    _fields_ = [
        ("graph", C.c_void_p),
        ("app", C.c_uint32),
        ("src", C.c_uint32),
        ("delta", C.c_int32),
        ("d_out", C.c_void_p),
        ("d_parent", C.c_void_p),
        ("status", C.c_int),
        ("levels", C.c_uint32),
        ("iterations", C.c_uint32),
        ("edges_scanned", C.c_uint64),
        ("device_ms", C.c_float),
    ]


class BatchStats(C.Structure):
    _fields_ = [
        ("queries", C.c_uint32),
        ("launch_ms", C.c_float),
        ("busy_ms", C.c_float),
        ("edges_scanned", C.c_uint64),
        ("grid_blocks", C.c_uint32),
        ("block_threads", C.c_uint32),
        ("scratch_bytes", C.c_size_t),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class ServeConfig(C.Structure):
    _fields_ = [
        ("lanes", C.c_uint32),
        ("max_batch", C.c_uint32),
        ("lane_arena_bytes", C.c_size_t),
        ("block_threads", C.c_uint32),
        ("hub_degree", C.c_uint32),
        ("lane_blocks", C.c_uint32),
        ("group_blocks", C.c_uint32),
        ("group_min_nodes", C.c_uint32),
        ("sparse_degree", C.c_uint32),
        ("queue_capacity", C.c_uint32),
        ("max_lanes_per_request", C.c_uint32),
        ("wide_lanes", C.c_uint32),
        ("wide_min_edges", C.c_uint32),
        ("resident", C.c_uint32),
        ("idle_exit_us", C.c_uint32),
    ]


class Completion(C.Structure):
    _fields_ = [
        ("ticket", C.c_uint64),
        ("status", C.c_int),
        ("latency_ms", C.c_double),
        ("queue_ms", C.c_double),
        ("lane", C.c_uint32),
        ("batch_size", C.c_uint32),
        ("width", C.c_uint32),
        ("levels", C.c_uint32),
        ("edges_scanned", C.c_uint64),
    ]


# name -> (restype, argtypes); every symbol include/gft.h declares.
_P = C.c_void_p
_SIGS: dict[str, tuple] = {
    "gft_version": (C.c_int, []),
    "gft_last_error": (C.c_char_p, []),
    "gft_status_string": (C.c_char_p, [C.c_int]),
    "gft_gr_read": (C.c_int, [C.c_char_p, C.POINTER(Csr)]),
    "gft_gr_read_chunked": (C.c_int, [C.c_char_p, C.POINTER(Csr)]),
    "gft_graph_load_gr": (C.c_int, [C.c_int, C.c_char_p, _P, C.POINTER(_P)]),
    "gft_ingest_release": (None, []),
    "gft_write_output_gz": (C.c_int, [C.c_char_p, C.c_uint32, _P, C.c_int]),
    "gft_write_node_data": (C.c_int, [C.c_char_p, C.c_uint32, _P, C.c_uint32]),
    "gft_read_node_data": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), _P]),
    "gft_gr_write": (C.c_int, [C.c_char_p, C.POINTER(Csr)]),
    "gft_csr_free": (None, [C.POINTER(Csr)]),
    "gft_gen_grid": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(Csr)]),
    "gft_gen_road": (C.c_int, [C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(Csr)]),
    "gft_gen_rmat": (
        C.c_int,
        [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(Csr)],
    ),
    "gft_pick_sources": (C.c_int, [C.POINTER(Csr), C.c_uint64, C.c_uint32, C.POINTER(C.c_uint32)]),
    "gft_graph_upload": (C.c_int, [C.c_int, C.POINTER(Csr), _P, C.POINTER(_P)]),
    "gft_graph_wrap": (C.c_int, [C.c_int, C.c_uint32, C.c_uint32, _P, _P, _P, C.POINTER(_P)]),
    "gft_graph_generate": (C.c_int, [C.c_int, C.POINTER(GenParams), _P, C.POINTER(_P)]),
    "gft_graph_info": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_int)]),
    "gft_graph_arrays": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "gft_graph_set_symmetric": (C.c_int, [_P, C.c_int]),
    "gft_graph_is_symmetric": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "gft_graph_download": (C.c_int, [_P, C.POINTER(Csr)]),
    "gft_graph_pick_sources": (C.c_int, [_P, C.c_uint64, C.c_uint32, C.POINTER(C.c_uint32)]),
    "gft_graph_free": (None, [_P]),
    "gft_engine_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "gft_engine_destroy": (None, [_P]),
    "gft_engine_scratch_bytes": (C.c_size_t, [_P]),
    "gft_bfs": (C.c_int, [_P, _P, C.c_uint32, _P, _P, C.POINTER(Tuning), _P, C.POINTER(Stats)]),
    "gft_sssp": (C.c_int, [_P, _P, C.c_uint32, C.c_int32, _P, _P, C.POINTER(Tuning), _P, C.POINTER(Stats)]),
    "gft_bfs_host": (C.c_int, [_P, _P, C.c_uint32, _P, _P, C.POINTER(Tuning), _P, C.POINTER(Stats)]),
    "gft_sssp_host": (C.c_int, [_P, _P, C.c_uint32, C.c_int32, _P, _P, C.POINTER(Tuning), _P, C.POINTER(Stats)]),
    "gft_bfs_host_many": (C.c_int, [_P, _P, _P, C.c_uint32, _P, C.POINTER(Tuning), _P, _P]),
    "gft_sssp_host_many": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_int32, _P, C.POINTER(Tuning), _P, _P]),
    "gft_reach_stats": (C.c_int, [_P, _P, _P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "gft_cc": (C.c_int, [_P, _P, _P, C.POINTER(Tuning), _P, C.POINTER(Stats), C.POINTER(C.c_uint64)]),
    "gft_cc_host": (C.c_int, [_P, _P, _P, C.POINTER(Tuning), _P, C.POINTER(Stats), C.POINTER(C.c_uint64)]),
    "gft_write_cc_output": (C.c_int, [C.c_char_p, C.POINTER(Csr), _P]),
    "gft_pr": (C.c_int, [_P, _P, _P, C.c_uint32, C.POINTER(Tuning), _P, C.POINTER(Stats)]),
    "gft_pr_host": (C.c_int, [_P, _P, _P, C.c_uint32, C.POINTER(Tuning), _P, C.POINTER(Stats)]),
    "gft_write_pr_output": (C.c_int, [C.c_char_p, C.c_uint32, _P]),
    "gft_mis": (C.c_int, [_P, _P, _P, C.c_uint32, C.POINTER(Tuning), _P, C.POINTER(Stats)]),
    "gft_mis_host": (C.c_int, [_P, _P, _P, C.c_uint32, C.POINTER(Tuning), _P, C.POINTER(Stats)]),
    "gft_write_mis_output": (C.c_int, [C.c_char_p, C.c_uint32, _P]),
    "gft_bfs_noalloc": (C.c_int, [_P, C.c_uint32, _P, _P, C.POINTER(Tuning), _P, C.POINTER(Stats)]),
    "gft_write_output": (C.c_int, [C.c_char_p, C.c_uint32, _P]),
    "gft_batch_create": (C.c_int, [_P, C.POINTER(Query), C.c_uint32, C.POINTER(Tuning), C.POINTER(_P)]),
    "gft_batch_set_source": (C.c_int, [_P, C.c_uint32, C.c_uint32]),
    "gft_batch_submit": (C.c_int, [_P, _P]),
    "gft_batch_wait": (C.c_int, [_P, C.POINTER(Query), C.POINTER(BatchStats)]),
    "gft_batch_destroy": (None, [_P]),
    "gft_msbfs_plane_bytes": (C.c_size_t, [C.c_uint32, C.c_uint32]),
    "gft_msbfs": (C.c_int, [_P, _P, C.POINTER(C.c_uint32), C.c_uint32, _P, C.c_uint32, C.c_uint32, _P,
                            C.POINTER(Stats)]),
    "gft_msbfs_levels": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P]),
    "gft_serve_config_default": (C.c_int, [C.POINTER(ServeConfig)]),
    "gft_serve_open": (C.c_int, [_P, C.POINTER(ServeConfig), C.POINTER(_P)]),
    "gft_serve_enqueue": (C.c_int, [_P, C.POINTER(Query), C.POINTER(C.c_uint64)]),
    "gft_serve_poll": (C.c_int, [_P, C.POINTER(Completion), C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32]),
    "gft_serve_stats": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "gft_serve_close": (C.c_int, [_P]),
}

_lock = threading.Lock()
_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Loads libgft.so (once) and declares every exported signature."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is not built; run `python -m galoisgpu_b200.build` "
                "(there is no fallback implementation)"
            )
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def declared_symbols() -> list[str]:
    return list(_SIGS)


def check(status: int) -> None:
    """Raises GftError for a non-zero status, with the library's message."""
    if status != 0:
        msg = load().gft_last_error()
        raise GftError(status, msg.decode() if msg else "")
