"""Seeded synthetic graphs: determinism, symmetry, canonical rows, sizes."""

import hashlib

import numpy as np
import pytest


def _digest(g):
    h = hashlib.sha256(g.row_start.tobytes() + g.edge_dst.tobytes())
    if g.edge_data is not None:
        h.update(g.edge_data.tobytes())
    return h.hexdigest()


def _check_canonical(g, weighted):
    rs, dst = g.row_start.astype(np.int64), g.edge_dst.astype(np.int64)
    assert rs[0] == 0 and rs[-1] == len(dst)
    assert (np.diff(rs) >= 0).all()
    src = np.repeat(np.arange(g.nnodes), np.diff(rs))
    assert (src != dst).all(), "self loop"
    key = src * g.nnodes + dst
    assert (np.diff(key) > 0).all(), "rows not strictly sorted (duplicate or unsorted)"
    rkey = dst * g.nnodes + src
    order = np.argsort(rkey)
    assert np.array_equal(rkey[order], key), "not symmetric"
    if weighted:
        assert (g.edge_data >= 1).all()
        np.testing.assert_array_equal(g.edge_data[order], g.edge_data)  # same weight both ways


def test_grid_shape_and_weights(gft):
    g = gft.CSRGraph.grid(256, 256)
    assert g.nnodes == 65536 and g.nedges == 261120  # 2 * (2 * 256 * 255)
    assert (g.edge_data == 1).all()
    _check_canonical(g, True)
    row = g.edge_dst[g.row_start[257]:g.row_start[258]]
    np.testing.assert_array_equal(row, [1, 256, 258, 513])


def test_grid_path_degenerate(gft):
    g = gft.CSRGraph.grid(1, 5, 0, 0)
    np.testing.assert_array_equal(g.degrees(), [1, 2, 2, 2, 1])


def test_road_properties(gft):
    g = gft.CSRGraph.road(256, seed=1)
    _check_canonical(g, True)
    grid_arcs = 2 * 2 * 256 * 255
    assert 0.93 * grid_arcs < g.nedges < 0.97 * grid_arcs + 2 * 200
    assert g.edge_data.max() <= 10000


def test_rmat_properties(gft):
    g = gft.CSRGraph.rmat(14, 16, seed=1, max_weight=255)
    _check_canonical(g, True)
    assert g.nnodes == 1 << 14
    assert g.edge_data.max() <= 255
    deg = g.degrees()
    assert deg.max() > 50 * deg.mean()  # power-law hubs


@pytest.mark.parametrize("make", [
    lambda gft, s: gft.CSRGraph.road(96, seed=s),
    lambda gft, s: gft.CSRGraph.rmat(12, 8, seed=s, max_weight=255),
    lambda gft, s: gft.CSRGraph.grid(33, 17, s, 100),
])
def test_seed_determinism(gft, make):
    a, b, c = make(gft, 5), make(gft, 5), make(gft, 6)
    assert _digest(a) == _digest(b)
    assert _digest(a) != _digest(c)


def test_pick_sources(gft):
    g = gft.CSRGraph.rmat(12, 8, seed=1)
    s = g.pick_sources(2, 64)
    assert len(set(s)) == 64
    assert all(g.getOutDegree(v) > 0 for v in s)
    assert s == g.pick_sources(2, 64)
    with pytest.raises(gft.GftError):
        gft.CSRGraph.grid(1, 1, 0, 0).pick_sources(1, 1)
