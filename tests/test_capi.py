"""The C ABI surface: libgft.so loads, exports every entry point include/gft.h
declares (and nothing the header does not), and reports errors as status
codes with messages -- no exit(), no crash -- including on a machine
without a GPU."""

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gft.h"


def header_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^GFT_API\s+[\w\s\*]+?\b(gft_\w+)\s*\(", text, flags=re.M)))


def exported_symbols(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True).stdout
    return sorted({ln.split()[-1] for ln in out.splitlines() if " T " in ln and ln.split()[-1].startswith("gft_")})


def test_header_and_library_agree(gft):
    from galoisgpu_b200 import _lib

    hs = header_symbols()
    assert len(hs) >= 25
    assert exported_symbols(_lib.LIB_PATH) == hs
    assert sorted(_lib.declared_symbols()) == hs  # the ctypes binding declares them all


def test_every_symbol_resolves(gft):
    lib = C.CDLL(str(gft._lib.LIB_PATH))
    for s in header_symbols():
        assert getattr(lib, s) is not None


def test_version_and_strings(gft):
    lib = gft.load()
    assert lib.gft_version() == 1
    assert lib.gft_status_string(0) == b"ok"
    assert lib.gft_status_string(6) == b"device wait timed out"


def test_null_arguments_are_errors_not_crashes(gft):
    lib = gft.load()
    assert lib.gft_gr_read(None, None) == 1
    assert b"null" in lib.gft_last_error()
    assert lib.gft_bfs(None, None, 0, None, None, None, None, None) == 1
    assert lib.gft_sssp(None, None, 0, 1, None, None, None, None, None) == 1
    assert lib.gft_bfs_host(None, None, 0, None, None, None, None, None) == 1
    assert lib.gft_bfs_host_many(None, None, None, 1, None, None, None, None) == 1
    assert lib.gft_sssp_host_many(None, None, None, 1, 1, None, None, None, None) == 1
    assert b"engine is NULL" in lib.gft_last_error()
    assert lib.gft_graph_info(None, None, None, None) == 1
    lib.gft_graph_free(None)
    lib.gft_engine_destroy(None)
    lib.gft_csr_free(None)


def test_no_gpu_is_a_status(gft):
    """On a machine without a usable sm_100 device, creating an engine
    returns a CUDA / not-supported status with a message."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = gft.load()
    h = C.c_void_p()
    st = lib.gft_engine_create(0, C.byref(h))
    assert st in (4, 8, 1)
    assert lib.gft_last_error()


def test_last_error_is_per_thread(gft):
    import threading

    lib = gft.load()
    lib.gft_gr_read(b"/nonexistent/a.gr", C.byref(gft._lib.Csr()))
    msgs = []

    def other():
        msgs.append(lib.gft_last_error())

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert msgs == [b""]
    assert b"/nonexistent/a.gr" in lib.gft_last_error()


def test_cli_binaries_are_the_right_apps():
    """bin/bfs takes the BFS options of apps/bfs/support.cu (no -d),
    bin/sssp adds -d (apps/sssp/support.cu) and bin/cc takes neither -s nor
    -d (apps/cc/support.cu); each prints the usage and exits non-zero
    without arguments, which needs no GPU."""
    import subprocess

    from galoisgpu_b200 import build as b

    if not (b.BIN / "bfs").exists():
        b.build()
    for app, has_delta, has_src in (("bfs", False, True), ("sssp", True, True), ("cc", False, False),
                                    ("pr", False, False), ("mis", False, False)):
        r = subprocess.run([str(b.BIN / app)], capture_output=True, text=True, timeout=60)
        assert r.returncode != 0
        assert "usage:" in r.stderr and ("[-s startNode]" in r.stderr) == has_src, r.stderr
        assert ("-d delta" in r.stderr) == has_delta, r.stderr
