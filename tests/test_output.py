"""The output path for large results: the gzip text writer must decompress
to exactly the text writer's bytes (the reference's format), and the binary
dump must decode to the same values the text holds, on the golden cases
(values the reference's own build produced) and on a multi-block array."""

import gzip

import numpy as np
import pytest

from conftest import ROOT

INF = 0x7FFFFFFF


def _golden():
    d = np.load(ROOT / "tests" / "golden" / "values.npz")
    return [(k, d[k].astype(np.int32)) for k in sorted(d.files)[:12]]


def _big():
    rng = np.random.default_rng(5)
    v = rng.integers(0, 2**31 - 1, size=(1 << 20) * 2 + 12345, dtype=np.int64).astype(np.int32)
    v[rng.integers(0, len(v), size=5000)] = INF
    return v


@pytest.mark.parametrize("level", [1, 6])
def test_gz_text_equals_text(gft, tmp_path, level):
    for name, v in _golden() + [("big", _big())]:
        t, z = tmp_path / "o.txt", tmp_path / "o.txt.gz"
        gft.output(t, v)
        gft.output_gz(z, v, level)
        assert gzip.decompress(z.read_bytes()) == t.read_bytes(), name


def test_gz_empty(gft, tmp_path):
    z = tmp_path / "e.gz"
    gft.output_gz(z, np.zeros(0, dtype=np.int32))
    assert gzip.decompress(z.read_bytes()) == b""


def test_node_data_roundtrip_matches_text(gft, orc, tmp_path):
    for name, v in _golden() + [("big", _big())]:
        b, t = tmp_path / "o.bin", tmp_path / "o.txt"
        gft.write_node_data(b, v)
        got = gft.read_node_data(b)
        assert got.dtype == np.int32
        np.testing.assert_array_equal(got, v)
        gft.output(t, v)
        np.testing.assert_array_equal(orc.read_output(t, len(v)), got)
        assert b.stat().st_size == 24 + 4 * len(v)


def test_node_data_float_ranks(gft, tmp_path):
    r = np.random.default_rng(1).random(1000).astype(np.float32)
    b = tmp_path / "r.bin"
    gft.write_node_data(b, r)
    got = gft.read_node_data(b)
    assert got.dtype == np.float32
    np.testing.assert_array_equal(got, r)


def test_node_data_errors(gft, tmp_path):
    b = tmp_path / "x.bin"
    b.write_bytes(b"NOTADUMP" + bytes(16))
    with pytest.raises(gft.GftError) as ei:
        gft.read_node_data(b)
    assert ei.value.status_name == "GFT_ERR_FORMAT"
    gft.write_node_data(b, np.arange(10, dtype=np.int32))
    b.write_bytes(b.read_bytes()[:-4])
    with pytest.raises(gft.GftError) as ei:
        gft.read_node_data(b)
    assert ei.value.status_name == "GFT_ERR_FORMAT"
