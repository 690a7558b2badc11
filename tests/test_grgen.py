"""oracle/libgrgen.so (the input graphs of the reference-build measurement,
built without the engine library) against the engine's own generators and
.gr writer: same arrays, same sources, same file bytes."""

import numpy as np
import pytest


@pytest.fixture(scope="module")
def grgen():
    from oracle import grgen

    return grgen


@pytest.mark.parametrize("kind,kw,seed", [
    ("grid", dict(rows=37, cols=53), 0),
    ("road", dict(side=120), 1),
    ("rmat", dict(scale=12, edge_factor=16), 1),
    ("rmat", dict(scale=11, edge_factor=8, max_weight=255), 5),
])
def test_same_graph_sources_and_file(gft, grgen, tmp_path, kind, kw, seed):
    mine = grgen.generate(kind, seed, **kw)
    if kind == "grid":
        ref = gft.CSRGraph.grid(kw["rows"], kw["cols"], seed, 1)
    elif kind == "road":
        ref = gft.CSRGraph.road(kw["side"], seed=seed)
    else:
        ref = gft.CSRGraph.rmat(kw["scale"], kw["edge_factor"], seed=seed, max_weight=kw.get("max_weight", 0))
    np.testing.assert_array_equal(mine.row_start, ref.row_start)
    np.testing.assert_array_equal(mine.edge_dst, ref.edge_dst)
    if ref.edge_data is None:
        assert mine.edge_data is None
    else:
        np.testing.assert_array_equal(mine.edge_data, ref.edge_data)
    assert mine.pick_sources(2, 9) == ref.pick_sources(2, 9)
    a, b = tmp_path / "a.gr", tmp_path / "b.gr"
    mine.write_gr(a)
    ref.write(b)
    assert a.read_bytes() == b.read_bytes()
    mine.close()
