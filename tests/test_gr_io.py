""".gr v1 reader/writer (gft_gr_read / gft_gr_write) against the layout the
reference parses (rt/src/csr_graph.cu:187-228), checked byte by byte with
struct and against the oracle's independent parser."""

import struct

import numpy as np
import pytest

from graphs import from_edges


def write_raw(path, nnodes, row_end, dst, weights=None, version=1, pad=True, size_edge_ty=None):
    with open(path, "wb") as f:
        f.write(struct.pack("<4Q", version, (4 if weights is not None else 0) if size_edge_ty is None else size_edge_ty,
                            nnodes, len(dst)))
        f.write(struct.pack(f"<{nnodes}Q", *row_end))
        f.write(struct.pack(f"<{len(dst)}I", *dst))
        if len(dst) % 2 and pad:
            f.write(b"\0\0\0\0")
        if weights is not None:
            f.write(struct.pack(f"<{len(weights)}I", *weights))


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("nedges_odd", [False, True])
def test_read_matches_hand_written_file(gft, orc, tmp_path, weighted, nedges_odd):
    edges = [(0, 1), (1, 2), (2, 0), (2, 3)] + ([(3, 1)] if nedges_odd else [])
    rs, dst, _ = from_edges(4, edges)
    w = [7, 1, 4000000000, 9, 3][: len(dst)] if weighted else None
    p = tmp_path / "g.gr"
    write_raw(p, 4, rs[1:].tolist(), dst.tolist(), w)
    g = gft.CSRGraph.read(p)
    np.testing.assert_array_equal(g.row_start, rs)
    np.testing.assert_array_equal(g.edge_dst, dst)
    if weighted:
        # u32 on disk, int in memory (csr_graph.cu:199,223-224): 4e9 wraps negative.
        np.testing.assert_array_equal(g.edge_data, np.array(w, dtype=np.uint32).view(np.int32))
    else:
        assert g.edge_data is None
    ors, odst, ow = orc.gr_read(p)
    np.testing.assert_array_equal(ors, g.row_start)
    np.testing.assert_array_equal(odst, g.edge_dst)


def test_writer_layout_is_byte_exact(gft, tmp_path):
    rs, dst, w = from_edges(3, [(0, 1), (0, 2), (2, 1)], [5, 6, 7])
    p = tmp_path / "w.gr"
    gft.CSRGraph(rs, dst, w).write(p)
    q = tmp_path / "r.gr"
    write_raw(q, 3, rs[1:].tolist(), dst.tolist(), w.tolist())
    assert p.read_bytes() == q.read_bytes()


def test_unweighted_odd_file_without_pad_is_accepted(gft, tmp_path):
    rs, dst, _ = from_edges(3, [(0, 1), (1, 2), (2, 0)])
    p = tmp_path / "np.gr"
    write_raw(p, 3, rs[1:].tolist(), dst.tolist(), None, pad=False)
    g = gft.CSRGraph.read(p)
    np.testing.assert_array_equal(g.edge_dst, dst)


def test_roundtrip_generated(gft, orc, tmp_path):
    for g in (gft.CSRGraph.road(64, seed=3), gft.CSRGraph.rmat(10, 8, seed=2), gft.CSRGraph.grid(5, 7, 0, 0)):
        p = tmp_path / "x.gr"
        g.write(p)
        h = gft.CSRGraph.read(p)
        np.testing.assert_array_equal(h.row_start, g.row_start)
        np.testing.assert_array_equal(h.edge_dst, g.edge_dst)
        assert (h.edge_data is None) == (g.edge_data is None)
        if g.edge_data is not None:
            np.testing.assert_array_equal(h.edge_data, g.edge_data)


def _err(gft, p):
    with pytest.raises(gft.GftError) as ei:
        gft.CSRGraph.read(p)
    return ei.value.status_name


def test_rejects_bad_version(gft, tmp_path):
    p = tmp_path / "v.gr"
    write_raw(p, 2, [1, 1], [1], version=2)
    assert _err(gft, p) == "GFT_ERR_FORMAT"


def test_rejects_destination_out_of_range(gft, tmp_path):
    # The reference only prints a warning here (csr_graph.cu:219) and later
    # reads out of bounds; the engine refuses the file.
    p = tmp_path / "d.gr"
    write_raw(p, 2, [1, 2], [1, 5])
    assert _err(gft, p) == "GFT_ERR_FORMAT"


def test_rejects_non_monotone_offsets(gft, tmp_path):
    p = tmp_path / "m.gr"
    write_raw(p, 3, [2, 1, 3], [1, 2, 0])
    assert _err(gft, p) == "GFT_ERR_FORMAT"


@pytest.mark.parametrize("cut", [8, 33, 40, 52, 60])
def test_rejects_truncated(gft, tmp_path, cut):
    p = tmp_path / "t.gr"
    write_raw(p, 3, [1, 2, 3], [1, 2, 0], [4, 5, 6])
    data = p.read_bytes()
    p.write_bytes(data[:cut])
    assert _err(gft, p) == "GFT_ERR_FORMAT"


def test_rejects_missing_file(gft, tmp_path):
    assert _err(gft, tmp_path / "nope.gr") == "GFT_ERR_IO"


def test_bad_size_edge_ty(gft, tmp_path):
    p = tmp_path / "s.gr"
    write_raw(p, 2, [1, 1], [1], size_edge_ty=8)
    assert _err(gft, p) == "GFT_ERR_FORMAT"


def test_empty_graph_roundtrip(gft, tmp_path):
    g = gft.CSRGraph(np.zeros(4, dtype=np.uint32), np.zeros(0, dtype=np.uint32))
    p = tmp_path / "e.gr"
    g.write(p)
    h = gft.CSRGraph.read(p)
    assert h.nnodes == 3 and h.nedges == 0


def test_output_format(gft, tmp_path):
    """'%d %d' / '%d INF' lines, i = 0..n-1 (apps/bfs/support.cu:39-45)."""
    p = tmp_path / "o.txt"
    gft.output(p, np.array([0, 0x7FFFFFFF, 5, 123456789], dtype=np.int32))
    assert p.read_text() == "0 0\n1 INF\n2 5\n3 123456789\n"
