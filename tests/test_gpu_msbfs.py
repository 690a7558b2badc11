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
