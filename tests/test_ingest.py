"""The parallel chunked .gr reader (gft_gr_read_chunked, the host side of
gft_graph_load_gr's pipeline) against the serial reader: the same arrays
byte for byte, including files that span many 8 MB chunks, and the same
errors, including a broken offset exactly at a chunk boundary."""

import struct

import numpy as np
import pytest

from test_gr_io import write_raw

IDX_PER_CHUNK = (8 << 20) // 8 - 1  # end offsets per chunk (one slot holds the previous offset)


def _same(a, b):
    np.testing.assert_array_equal(a.row_start, b.row_start)
    np.testing.assert_array_equal(a.edge_dst, b.edge_dst)
    assert (a.edge_data is None) == (b.edge_data is None)
    if a.edge_data is not None:
        np.testing.assert_array_equal(a.edge_data, b.edge_data)


@pytest.mark.parametrize("make", [
    lambda g: g.road(1100, seed=4),                 # 1.21 M nodes, ~4.6 M weighted edges: several chunks each
    lambda g: g.rmat(16, 16, seed=3),               # unweighted, skewed
    lambda g: g.grid(3, 5, 0, 0),                   # tiny, unweighted
    lambda g: g(np.zeros(6, dtype=np.uint32), np.zeros(0, dtype=np.uint32)),  # no edges
])
def test_chunked_reader_matches_serial_reader(gft, tmp_path, make):
    g = make(gft.CSRGraph)
    p = tmp_path / "g.gr"
    g.write(p)
    _same(gft.CSRGraph.read_chunked(p), gft.CSRGraph.read(p))
    _same(gft.CSRGraph.read_chunked(p), g)


def test_hand_written_odd_file_without_pad(gft, tmp_path):
    p = tmp_path / "np.gr"
    write_raw(p, 3, [1, 2, 3], [1, 2, 0], None, pad=False)
    _same(gft.CSRGraph.read_chunked(p), gft.CSRGraph.read(p))


def _err(gft, p):
    with pytest.raises(gft.GftError) as e1:
        gft.CSRGraph.read_chunked(p)
    with pytest.raises(gft.GftError) as e2:
        gft.CSRGraph.read(p)
    assert e1.value.status_name == e2.value.status_name
    return e1.value.status_name


@pytest.mark.parametrize("case", ["version", "dst", "monotone", "ends_short", "size_edge_ty", "missing"])
def test_same_errors_as_serial_reader(gft, tmp_path, case):
    p = tmp_path / "bad.gr"
    if case == "version":
        write_raw(p, 2, [1, 1], [1], version=2)
    elif case == "dst":
        write_raw(p, 2, [1, 2], [1, 5])
    elif case == "monotone":
        write_raw(p, 3, [2, 1, 3], [1, 2, 0])
    elif case == "ends_short":
        write_raw(p, 3, [1, 2, 2], [1, 2, 0])
    elif case == "size_edge_ty":
        write_raw(p, 2, [1, 1], [1], size_edge_ty=8)
    want = "GFT_ERR_IO" if case == "missing" else "GFT_ERR_FORMAT"
    assert _err(gft, p) == want


@pytest.mark.parametrize("cut", [8, 33, 40, 52, 60])
def test_truncated(gft, tmp_path, cut):
    p = tmp_path / "t.gr"
    write_raw(p, 3, [1, 2, 3], [1, 2, 0], [4, 5, 6])
    p.write_bytes(p.read_bytes()[:cut])
    assert _err(gft, p) == "GFT_ERR_FORMAT"


def test_offsets_broken_at_a_chunk_boundary(gft, tmp_path):
    """The first offset of the second index chunk is checked against the last
    one of the first chunk."""
    n = IDX_PER_CHUNK + 10
    ends = np.arange(1, n + 1, dtype=np.uint64)  # one edge per node
    dst = (np.arange(n, dtype=np.uint32) + 1) % n
    p = tmp_path / "b.gr"
    with open(p, "wb") as f:
        f.write(struct.pack("<4Q", 1, 0, n, n))
        bad = ends.copy()
        bad[IDX_PER_CHUNK] = bad[IDX_PER_CHUNK - 1] - 1  # a decrease right at the boundary
        f.write(bad.tobytes())
        f.write(dst.tobytes())
    assert _err(gft, p) == "GFT_ERR_FORMAT"
    # The same file without the decrease reads fine.
    with open(p, "r+b") as f:
        f.seek(32)
        f.write(ends.tobytes())
    _same(gft.CSRGraph.read_chunked(p), gft.CSRGraph.read(p))
