"""gft_graph_load_gr (a .gr file straight into device memory through pinned
chunked reads overlapped with the copies) against the host reader plus
upload: the same device arrays, the same query results, the same errors."""

import numpy as np
import pytest

from test_gr_io import write_raw

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [
    lambda g: g.road(1100, seed=4),        # several chunks per section, weighted
    lambda g: g.rmat(17, 16, seed=3),      # unweighted, skewed
    lambda g: g.grid(3, 5, 0, 0),
])
def test_load_gr_equals_read_and_upload(gft, engine, tmp_path, make):
    g = make(gft.CSRGraph)
    p = tmp_path / "g.gr"
    g.write(p)
    d = gft.DeviceGraph.load_gr(p)
    back = d.download()
    np.testing.assert_array_equal(back.row_start, g.row_start)
    np.testing.assert_array_equal(back.edge_dst, g.edge_dst)
    assert (back.edge_data is None) == (g.edge_data is None)
    if g.edge_data is not None:
        np.testing.assert_array_equal(back.edge_data, g.edge_data)
    ref = g.copy_to_gpu()
    src = g.pick_sources(1, 1)[0]
    np.testing.assert_array_equal(engine.bfs(d, src)["out"].cpu().numpy(), engine.bfs(ref, src)["out"].cpu().numpy())
    if g.edge_data is not None:
        np.testing.assert_array_equal(engine.sssp(d, src, delta=5000)["out"].cpu().numpy(),
                                      engine.sssp(ref, src, delta=5000)["out"].cpu().numpy())
    d.free()
    ref.free()


def test_load_gr_empty_graph(gft, tmp_path):
    g = gft.CSRGraph(np.zeros(5, dtype=np.uint32), np.zeros(0, dtype=np.uint32))
    p = tmp_path / "e.gr"
    g.write(p)
    d = gft.DeviceGraph.load_gr(p)
    assert d.nnodes == 4 and d.nedges == 0
    d.free()


@pytest.mark.parametrize("case", ["dst", "monotone", "truncated", "missing"])
def test_load_gr_errors(gft, tmp_path, case):
    p = tmp_path / "bad.gr"
    if case == "dst":  # found by the device check
        write_raw(p, 2, [1, 2], [1, 5])
    elif case == "monotone":
        write_raw(p, 3, [2, 1, 3], [1, 2, 0])
    elif case == "truncated":
        write_raw(p, 3, [1, 2, 3], [1, 2, 0], [4, 5, 6])
        p.write_bytes(p.read_bytes()[:52])
    with pytest.raises(gft.GftError) as ei:
        gft.DeviceGraph.load_gr(p)
    assert ei.value.status_name == ("GFT_ERR_IO" if case == "missing" else "GFT_ERR_FORMAT")
