"""Multi-source BFS (bitsets, top-down / bottom-up per level) gives, for
every source, the same levels as a single-source BFS and the CPU oracle."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k,symmetric", [(256, True), (256, False), (50, True), (1, True), (33, False)])
def test_msbfs_matches_single_bfs(gft, orc, engine, k, symmetric):
    g = gft.CSRGraph.rmat(14, 16, seed=8)
    dg = g.copy_to_gpu()
    srcs = g.pick_sources(5, k)
    r = engine.msbfs(dg, srcs, max_levels=24, symmetric=symmetric)
    assert r["levels"] >= 2
    for i in range(0, k, max(1, k // 17)):
        got = r["levels_of"](i).cpu().numpy()
        np.testing.assert_array_equal(got, orc.bfs(g.row_start, g.edge_dst, srcs[i]))


def test_msbfs_road_and_duplicates(gft, orc, engine):
    g = gft.CSRGraph.road(60, seed=3)
    dg = g.copy_to_gpu()
    srcs = [0, 5, 5, 1799, 3599, 0]  # repeated sources are independent queries
    r = engine.msbfs(dg, srcs, max_levels=200, symmetric=True)
    for i, s in enumerate(srcs):
        np.testing.assert_array_equal(r["levels_of"](i).cpu().numpy(), orc.bfs(g.row_start, g.edge_dst, s))


def test_msbfs_level_overflow_is_a_status(gft, engine):
    g = gft.CSRGraph.grid(1, 100, 0, 0)
    dg = g.copy_to_gpu()
    with pytest.raises(gft.GftError) as ei:
        engine.msbfs(dg, [0], max_levels=10)
    assert ei.value.status_name == "GFT_ERR_OVERFLOW"
    r = engine.msbfs(dg, [0], max_levels=101)
    assert r["levels"] == 100


@pytest.mark.parametrize("k", [128, 256])
def test_msbfs_sources_in_small_components(gft, orc, engine, k):
    """Sources whose search ends early (a path of three vertices, a pair)
    drop out of the set of sources a vertex still waits for, so the other
    vertices can stop scanning; every source's levels still match the
    oracle, bottom-up levels included."""
    g0 = gft.CSRGraph.rmat(14, 16, seed=8)
    n0 = g0.nnodes
    rs0 = g0.row_start.astype(np.int64)
    src_of = np.repeat(np.arange(n0, dtype=np.int64), np.diff(rs0))
    extra = np.array([(0, 1), (1, 0), (1, 2), (2, 1), (3, 4), (4, 3)], dtype=np.int64) + n0
    a = np.concatenate([src_of, extra[:, 0]])
    b = np.concatenate([g0.edge_dst.astype(np.int64), extra[:, 1]])
    n = n0 + 5
    order = np.lexsort((b, a))
    dst = b[order].astype(np.uint32)
    rs = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum(np.bincount(a, minlength=n), out=rs[1:])
    g = gft.CSRGraph(rs, dst, None)
    dg = g.copy_to_gpu()
    small = [n0, n0 + 2, n0 + 3, n0 + 1]
    srcs = g0.pick_sources(5, k - len(small))
    srcs = srcs[: k // 3] + small[:2] + srcs[k // 3:] + small[2:]
    assert len(srcs) == k
    r = engine.msbfs(dg, srcs, max_levels=24, symmetric=True)
    for i, s in enumerate(srcs):
        np.testing.assert_array_equal(r["levels_of"](i).cpu().numpy(), orc.bfs(rs, dst, s))
