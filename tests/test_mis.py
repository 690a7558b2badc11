"""Maximal independent set (apps/mis on this engine): the CPU oracle pinned to
the reference's own CUDA build (tests/golden/mis_*), the product's output
writer against the reference format, and gft_mis on the GPU against the
oracle and the golden sets.

The reference's set is a function of its priorities, which come from one
xorshift128 stream per thread of its launch grid (apps/mis/kernel.cu:18-41;
8 CTAs of 256 threads per SM, skelapp/skel.cu:37-43): the marking and
dropping rounds read only states that the round itself cannot change in a
way that matters.  So parity is exact: the same set, the same round count
("Total steps"), given the same priority-thread count.
"""

import json
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from test_golden import _graph

GOLDEN = Path(__file__).resolve().parent / "golden"
MIS_MANIFEST = json.loads((GOLDEN / "mis_manifest.json").read_text())
MIS_VALUES = np.load(GOLDEN / "mis_values.npz")
ROOT = Path(__file__).resolve().parent.parent


def golden_mask(key: str) -> np.ndarray:
    e = MIS_MANIFEST[key]
    return np.unpackbits(MIS_VALUES[key], bitorder="little", count=e["nnodes"]).astype(bool)


def xorshift_priorities(n: int, nthreads: int) -> np.ndarray:
    """Marsaglia's xorshift128 per thread, in plain Python: thread t starts
    from the seeds ^ t and gives its k-th output to vertex t + k*nthreads."""
    out = np.zeros(n, dtype=np.uint32)
    m = 0xFFFFFFFF
    for t in range(min(n, nthreads)):
        x, y, z, w = 0x12345678 ^ t, 0xABBDEF12 ^ t, 0xCAFE1234 ^ t, 0x09832516 ^ t
        for v in range(t, n, nthreads):
            tt = (x ^ (x << 11)) & m
            x, y, z = y, z, w
            w = (w ^ (w >> 19) ^ tt ^ (tt >> 8)) & m
            out[v] = w
    return out


def is_independent_and_maximal(g, inset: np.ndarray) -> tuple[bool, bool]:
    rs = np.asarray(g.row_start, dtype=np.int64)
    dst = np.asarray(g.edge_dst, dtype=np.int64)
    src = np.repeat(np.arange(g.nnodes), np.diff(rs))
    real = src != dst
    independent = not np.any(inset[src] & inset[dst] & real)
    covered = np.zeros(g.nnodes, dtype=bool)
    np.logical_or.at(covered, src[real], inset[dst[real]])
    return independent, bool(np.all(inset | covered))


def test_oracle_priorities_are_xorshift128_per_thread(orc):
    for n, nt in ((1000, 4096), (1000, 64), (777, 7), (33, 1)):
        np.testing.assert_array_equal(orc.mis_priorities(n, nt), xorshift_priorities(n, nt))


@pytest.mark.parametrize("key", sorted(MIS_MANIFEST))
def test_oracle_mis_matches_reference(gft, orc, key):
    e = MIS_MANIFEST[key]
    g = _graph(gft, e["recipe"], e["graph"])
    assert e["runs_identical"]  # the reference itself is deterministic
    state, steps = orc.mis(g.row_start, g.edge_dst, e["prio_threads"])
    np.testing.assert_array_equal(state == 1, golden_mask(key))
    assert set(np.unique(state)) <= {1, 2}
    assert steps == e["steps_runs"][0]


def test_mis_golden_sets_are_independent_and_maximal(gft):
    for key, e in MIS_MANIFEST.items():
        g = _graph(gft, e["recipe"], e["graph"])
        if not g.symmetric:
            continue
        ind, mx = is_independent_and_maximal(g, golden_mask(key))
        assert ind and mx, key


def test_product_mis_writer_matches_oracle_text(gft, orc, tmp_path):
    e = MIS_MANIFEST["rmat12w.mis"]
    g = _graph(gft, e["recipe"], "rmat12w")
    state, _ = orc.mis(g.row_start, g.edge_dst, e["prio_threads"])
    a, b = tmp_path / "a.txt", tmp_path / "b.txt"
    orc.write_mis_output(a, state)
    gft.write_mis_output(b, state)
    assert a.read_bytes() == b.read_bytes()
    np.testing.assert_array_equal(orc.read_mis_output(a, g.nnodes), state == 1)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------


def _device_prio_threads():
    import torch

    return 8 * torch.cuda.get_device_properties(0).multi_processor_count * 256


@pytest.mark.gpu
@pytest.mark.parametrize("key", sorted(MIS_MANIFEST))
def test_gpu_mis_matches_reference_golden(gft, engine, key):
    e = MIS_MANIFEST[key]
    g = _graph(gft, e["recipe"], e["graph"])
    r = engine.mis(g.copy_to_gpu(), prio_threads=e["prio_threads"])
    state = r["out"].cpu().numpy()
    np.testing.assert_array_equal(state == 1, golden_mask(key))
    assert set(np.unique(state)) <= {1, 2}
    assert r["levels"] == e["steps_runs"][0]
    assert r["vertices_reached"] == e["set_size"]


@pytest.mark.gpu
def test_gpu_mis_default_priorities_are_the_references_on_this_device(gft, orc, engine):
    g = gft.CSRGraph.road(120, seed=9)
    r = engine.mis(g.copy_to_gpu())
    want, steps = orc.mis(g.row_start, g.edge_dst, _device_prio_threads())
    np.testing.assert_array_equal(r["out"].cpu().numpy(), want)
    assert r["levels"] == steps


@pytest.mark.gpu
@pytest.mark.parametrize("tune", [None, {"max_blocks": 1}, {"max_blocks": 1 << 30},
                                  {"block_threads": 256, "blocks_per_sm": 4, "max_blocks": 1 << 30}],
                         ids=["auto", "one-cta", "grid", "grid256x4"])
def test_gpu_mis_matches_oracle(gft, orc, engine, tune):
    """Larger graphs than the golden ones (more vertices than priority
    streams, hubs scanned by whole warps), a directed graph, and one
    priority-thread count that is not the device's."""
    graphs = (gft.CSRGraph.rmat(16, 16, seed=21), gft.CSRGraph.road(700, seed=22),
              gft.CSRGraph.grid(40, 1500, 0, 1), gft.CSRGraph.rmat(15, 8, seed=23, max_weight=0))
    for i, g in enumerate(graphs):
        dg = g.copy_to_gpu()
        if i == 3:  # directed: drop the symmetry of the generator's edge list
            rs = np.asarray(g.row_start)
            keep = np.repeat(np.arange(g.nnodes), np.diff(rs)) < np.asarray(g.edge_dst)
            dst = np.asarray(g.edge_dst)[keep]
            deg = np.bincount(np.repeat(np.arange(g.nnodes), np.diff(rs))[keep], minlength=g.nnodes)
            g = gft.CSRGraph(np.concatenate([[0], np.cumsum(deg)]).astype(np.uint32), dst.astype(np.uint32), None)
            dg = g.copy_to_gpu()
        for nt in (_device_prio_threads(), 4099):
            want, steps = orc.mis(g.row_start, g.edge_dst, nt)
            r = engine.mis(dg, prio_threads=nt, tune=gft.Tune(**tune) if tune else None)
            np.testing.assert_array_equal(r["out"].cpu().numpy(), want)
            assert r["levels"] == steps


@pytest.mark.gpu
def test_gpu_mis_host_variant_and_full_size_properties(gft, engine):
    dg = gft.DeviceGraph.generate("rmat", seed=5, scale=20, edge_factor=16)
    host = dg.download()
    out = np.empty(dg.nnodes, dtype=np.int32)
    st = engine.mis_host(dg, out)
    ind, mx = is_independent_and_maximal(host, out == 1)
    assert ind and mx
    assert st["vertices_reached"] == int((out == 1).sum())
    assert set(np.unique(out)) <= {1, 2}
    r = engine.mis(dg)
    np.testing.assert_array_equal(r["out"].cpu().numpy(), out)  # deterministic


def _run_mis_cli(prog: Path, key: str, tmp_path: Path, gft):
    e = MIS_MANIFEST[key]
    g = _graph(gft, e["recipe"], e["graph"])
    gr = tmp_path / f"{e['graph']}.gr"
    g.write(gr)
    out = tmp_path / f"{key}.out"
    r = subprocess.run([str(prog), "-o", str(out), str(gr)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    steps = int(re.search(r"Total steps: (\d+)", r.stdout).group(1))
    return out.read_text(), steps, g


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["rmat14.mis", "road200s7.mis", "star5000.mis", "selfloops_dups.mis"])
def test_mis_cli_and_dropin_match_reference(gft, orc, tmp_path, key):
    e = MIS_MANIFEST[key]
    if e["prio_threads"] != _device_prio_threads():
        pytest.skip("golden sets were made on a GPU with another SM count")
    want = tmp_path / "want.txt"
    state = np.where(golden_mask(key), 1, 2).astype(np.int32)
    orc.write_mis_output(want, state)
    for prog in (ROOT / "galoisgpu_b200" / "bin" / "mis", ROOT / "oracle" / "_ref" / "mis_gft"):
        if not prog.exists():
            assert prog.name == "mis_gft", "galoisgpu_b200/bin is built by __graft_entry__.build()"
            continue
        text, steps, _ = _run_mis_cli(prog, key, tmp_path, gft)
        assert text == want.read_text()
        assert steps == e["steps_runs"][0]
