"""Connected components: the CPU oracle pinned to the reference's own CUDA
build (partition and component count, tests/golden/cc_*; the reference's
labels depend on its racy hooking schedule, so only the partition is
comparable), the product's output writer against the reference format, and
gft_cc on the GPU against the oracle, label for label."""

import json
from pathlib import Path

import numpy as np
import pytest

from test_golden import _graph

GOLDEN = Path(__file__).resolve().parent / "golden"
CC_MANIFEST = json.loads((GOLDEN / "cc_manifest.json").read_text())
CC_VALUES = np.load(GOLDEN / "cc_values.npz")


@pytest.mark.parametrize("key", sorted(CC_MANIFEST))
def test_oracle_cc_matches_reference_partition(gft, orc, key):
    e = CC_MANIFEST[key]
    g = _graph(gft, e["recipe"], e["graph"])
    label, comps = orc.cc(g.row_start, g.edge_dst)
    assert comps == e["components"]
    np.testing.assert_array_equal(label, CC_VALUES[key])  # already the canonical (smallest-id) form
    np.testing.assert_array_equal(orc.canonical_labels(label), label)


def test_product_cc_writer_matches_oracle_text(gft, orc, tmp_path):
    for key in ("rmat12w.cc", "disconnected.cc", "grid64x40w.cc"):
        e = CC_MANIFEST[key]
        g = _graph(gft, e["recipe"], e["graph"])
        label, _ = orc.cc(g.row_start, g.edge_dst)
        a, b = tmp_path / "a.txt", tmp_path / "b.txt"
        orc.write_cc_output(a, g.row_start, g.edge_dst, g.edge_data, label)
        gft.write_cc_output(b, g, label)
        assert a.read_bytes() == b.read_bytes(), key


def test_cc_cases_cover_several_shapes():
    counts = {k: e["components"] for k, e in CC_MANIFEST.items()}
    assert len(counts) >= 10 and max(counts.values()) > 100 and min(counts.values()) == 1


@pytest.mark.gpu
def test_gpu_cc_matches_reference_golden(gft, engine):
    for key, e in sorted(CC_MANIFEST.items()):
        g = _graph(gft, e["recipe"], e["graph"])
        r = engine.cc(g.copy_to_gpu())
        np.testing.assert_array_equal(r["out"].cpu().numpy(), CC_VALUES[key], err_msg=key)
        assert r["components"] == e["components"], key


@pytest.mark.gpu
@pytest.mark.parametrize("symmetric", [True, False])
def test_gpu_cc_matches_oracle(gft, orc, engine, symmetric):
    """Larger graphs, with and without the symmetry mark (unmarked, every
    directed edge is joined), including hub vertices above the chunking
    degree and many small components."""
    graphs = [gft.CSRGraph.rmat(16, 16, seed=5), gft.CSRGraph.rmat(15, 4, seed=6), gft.CSRGraph.road(300, seed=9),
              gft.CSRGraph.grid(40, 700, 0, 1)]
    for g in graphs:
        dg = g.copy_to_gpu()
        dg.symmetric = symmetric
        want, comps = orc.cc(g.row_start, g.edge_dst)
        for _ in range(2):
            r = engine.cc(dg)
            np.testing.assert_array_equal(r["out"].cpu().numpy(), want)
            assert r["components"] == comps


@pytest.mark.gpu
def test_gpu_cc_directed_and_host_variant(gft, orc, engine):
    """A directed graph (weak components) through the host-buffer call."""
    rng = np.random.default_rng(3)
    n, m = 50_000, 60_000
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order].astype(np.uint32)
    rs = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum(np.bincount(src, minlength=n), out=rs[1:])
    g = gft.CSRGraph(rs, dst, None)
    want, comps = orc.cc(rs, dst)
    out = np.empty(n, dtype=np.int32)
    r = engine.cc_host(g.copy_to_gpu(), out)
    np.testing.assert_array_equal(out, want)
    assert r["components"] == comps
