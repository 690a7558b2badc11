"""The allocation-free BFS entry point (gft_bfs_noalloc), called through the
C ABI, against the regular entry point (gft_bfs).

gft_bfs_noalloc exists for callers that cannot call cudaMalloc themselves or
have the library do it (another component owns the device memory, or the
call sits on a path where an allocation's implicit synchronisation is not
allowed).  Its scratch is a fixed device array shared by all calls, so this
test makes two calls in a row on the same scratch and checks each against
gft_bfs, bit for bit, plus the parent tree.  The file is named to be
collected last."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_NODES = 1 << 20


def _noalloc(gft, dg, src, level, parent, stream=0):
    st = gft._lib.Stats()
    status = gft.load().gft_bfs_noalloc(dg.handle, src, C.c_void_p(level.data_ptr()),
                                        C.c_void_p(parent.data_ptr() if parent is not None else 0), None,
                                        C.c_void_p(stream), C.byref(st))
    return status, st


def test_noalloc_matches_gft_bfs_twice(gft, orc, engine):
    import torch

    g = gft.CSRGraph.rmat(16, 16, seed=9)
    dg = g.copy_to_gpu()
    srcs = g.pick_sources(4, 2)
    for src in srcs:  # two calls in a row on the shared scratch
        level = torch.full((g.nnodes,), -1, dtype=torch.int32, device="cuda")
        parent = torch.full((g.nnodes,), -1, dtype=torch.int32, device="cuda")
        status, st = _noalloc(gft, dg, src, level, parent)
        assert status == 0, gft.load().gft_last_error()
        want = engine.bfs(dg, src)["out"].cpu().numpy()
        got = level.cpu().numpy()
        np.testing.assert_array_equal(got, want)
        assert orc.check_tree(g.row_start, g.edge_dst, None, src, got, parent.cpu().numpy().view(np.uint32)) == 0
        assert st.levels > 0


def test_noalloc_on_a_second_graph_and_without_parent(gft, engine):
    import torch

    g = gft.CSRGraph.road(700, seed=2)  # 490,000 vertices
    dg = g.copy_to_gpu()
    for src in (0, g.nnodes - 1):
        level = torch.empty(g.nnodes, dtype=torch.int32, device="cuda")
        status, _ = _noalloc(gft, dg, src, level, None)
        assert status == 0, gft.load().gft_last_error()
        np.testing.assert_array_equal(level.cpu().numpy(), engine.bfs(dg, src)["out"].cpu().numpy())


def test_noalloc_rejects_graphs_over_the_limit(gft):
    import torch

    rs = torch.zeros(MAX_NODES + 2, dtype=torch.int32, device="cuda")
    h = C.c_void_p()
    assert gft.load().gft_graph_wrap(0, MAX_NODES + 1, 0, C.c_void_p(rs.data_ptr()), C.c_void_p(rs.data_ptr()),
                                     None, C.byref(h)) == 0
    dg = gft.DeviceGraph(h, 0)
    level = torch.empty(MAX_NODES + 1, dtype=torch.int32, device="cuda")
    status, _ = _noalloc(gft, dg, 0, level, None)
    assert status == 1
    assert b"limit" in gft.load().gft_last_error()
    dg.free()
