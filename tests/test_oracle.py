"""The CPU oracle on known answers, and its validators catching mistakes
planted in oracle outputs (never in GPU results)."""

import numpy as np
import pytest

from graphs import from_edges, path, star, undirected

INF = 0x7FFFFFFF


def test_bfs_grid_closed_form(gft, orc):
    g = gft.CSRGraph.grid(64, 48, 0, 1)
    lvl = orc.bfs(g.row_start, g.edge_dst, 0)
    r, c = np.divmod(np.arange(g.nnodes), 48)
    np.testing.assert_array_equal(lvl, r + c)


def test_bfs_path_star_disconnected(orc):
    rs, dst, _ = path(10)
    np.testing.assert_array_equal(orc.bfs(rs, dst, 0), np.arange(10))
    np.testing.assert_array_equal(orc.bfs(rs, dst, 9), np.arange(10)[::-1])
    rs, dst, _ = star(300)
    lvl = orc.bfs(rs, dst, 5)
    assert lvl[5] == 0 and lvl[0] == 1 and (np.delete(lvl, [0, 5]) == 2).all()
    rs, dst, _ = undirected(6, [(0, 1), (3, 4)])
    np.testing.assert_array_equal(orc.bfs(rs, dst, 0), [0, 1, INF, INF, INF, INF])


def test_sssp_known_answers(orc):
    # 0 -1-> 1 -1-> 2 and a direct 0 -5-> 2: the two-hop path wins.
    rs, dst, w = from_edges(4, [(0, 1), (1, 2), (0, 2), (2, 3)], [1, 1, 5, 10])
    np.testing.assert_array_equal(orc.sssp(rs, dst, w, 0), [0, 1, 2, 12])
    # Unweighted graph = all-zero weights (the reference calloc's edge_data).
    np.testing.assert_array_equal(orc.sssp(rs, dst, None, 0), [0, 0, 0, 0])
    np.testing.assert_array_equal(orc.sssp(rs, dst, w, 3), [INF, INF, INF, 0])


def test_sssp_matches_bfs_with_unit_weights(gft, orc):
    g = gft.CSRGraph.road(80, seed=2, max_weight=1)
    s = g.pick_sources(1, 1)[0]
    np.testing.assert_array_equal(orc.sssp(g.row_start, g.edge_dst, g.edge_data, s),
                                  orc.bfs(g.row_start, g.edge_dst, s))


def test_sssp_overflow_is_detected(orc):
    rs, dst, w = from_edges(3, [(0, 1), (1, 2)], [0x7FFFFFF0, 0x7FFFFFF0])
    with pytest.raises(OverflowError):
        orc.sssp(rs, dst, w, 0)


def test_tree_validator_accepts_oracle_trees(gft, orc):
    g = gft.CSRGraph.rmat(11, 8, seed=4, max_weight=50)
    s = g.pick_sources(3, 1)[0]
    lvl, par = orc.bfs(g.row_start, g.edge_dst, s, parent=True)
    assert orc.check_tree(g.row_start, g.edge_dst, None, s, lvl, par) == 0
    dist, par = orc.sssp(g.row_start, g.edge_dst, g.edge_data, s, parent=True)
    assert orc.check_tree(g.row_start, g.edge_dst, g.edge_data, s, dist, par) == 0


def test_tree_validator_catches_planted_mistakes(gft, orc):
    g = gft.CSRGraph.road(40, seed=1)
    s = 0
    dist, par = orc.sssp(g.row_start, g.edge_dst, g.edge_data, s, parent=True)
    reached = np.nonzero((dist != INF) & (np.arange(g.nnodes) != s))[0]
    v = int(reached[len(reached) // 2])
    bad = par.copy()
    bad[v] = (par[v] + 1) % g.nnodes  # a non-neighbour or wrong-distance parent
    assert orc.check_tree(g.row_start, g.edge_dst, g.edge_data, s, dist, bad) >= 1
    bad = par.copy()
    bad[s] = v
    assert orc.check_tree(g.row_start, g.edge_dst, g.edge_data, s, dist, bad) >= 1
    wrong = dist.copy()
    wrong[v] += 1
    assert orc.check_tree(g.row_start, g.edge_dst, g.edge_data, s, wrong, par) >= 1


def test_reach_stats(gft, orc):
    rs, dst, _ = undirected(5, [(0, 1), (1, 2), (3, 4)])
    lvl = orc.bfs(rs, dst, 0)
    assert orc.reach_stats(rs, lvl) == (3, 4)


def test_output_roundtrip(orc, tmp_path):
    v = np.array([0, INF, 7, -3], dtype=np.int32)
    p = tmp_path / "o.txt"
    orc.write_output(p, v)
    assert p.read_text() == "0 0\n1 INF\n2 7\n3 -3\n"
    np.testing.assert_array_equal(orc.read_output(p, 4), v)
