"""PageRank (residual push, apps/pr on this engine): the CPU oracle pinned to
the reference's own CUDA build (tests/golden/pr_*), the product's output
writer against the reference format, and gft_pr on the GPU against the
oracle and the golden ranks.

Ranks are float sums accumulated with atomicAdd in whatever order the GPU
runs, in the reference as here, so two runs of the reference itself differ
(by up to 4.2e-5 on the golden graphs, recorded in pr_manifest.json).  The
tolerance used throughout is |a - b| <= RTOL * max(1, |b|), RTOL = 1e-4: the
largest relative difference between the oracle and the reference on the
golden graphs is 5.2e-5, on the 5000-leaf star whose hub holds rank 2298.

A few vertices per run may miss RTOL for a second reason, the reference's:
its crossing test `prev + update > EPSILON && prev < EPSILON`
(apps/pr/kernel.cu:190,222) fails when a residual sum rounds to exactly
EPSILON, and that vertex is never queued again, so the residual it gathers
afterwards never reaches its rank.  Which vertex lands there depends on the
summation order: 0-4 per run on the 32768-vertex R-MAT below in shuffled
sequential schedules of the oracle (which restates that test).  Such a vertex
falls short by what it gathers in the remaining rounds, a few 1e-5 relative.
gft_pr builds each worklist from the residuals above EPSILON instead, so it
has no such vertex, but the oracle and the golden ranks may.  So up to
MAX_STUCK vertices per graph may miss RTOL, and they must still be within
LOOSE_RTOL."""

import json
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from test_golden import _graph

RTOL = 1e-4
GOLDEN = Path(__file__).resolve().parent / "golden"
PR_MANIFEST = json.loads((GOLDEN / "pr_manifest.json").read_text())
PR_VALUES = np.load(GOLDEN / "pr_values.npz")
ROOT = Path(__file__).resolve().parent.parent


MAX_STUCK = 8
LOOSE_RTOL = 1e-3


def close(a, b) -> bool:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    err = np.abs(a - b) / np.maximum(1.0, np.abs(b))
    return bool(np.count_nonzero(err > RTOL) <= MAX_STUCK and np.all(err <= LOOSE_RTOL))


def test_close_allows_only_a_few_stuck_vertices():
    b = np.linspace(1.0, 3.0, 1000)
    a = b.copy()
    a[:MAX_STUCK] -= 3e-4 * b[:MAX_STUCK]
    assert close(a, b)
    a[MAX_STUCK] -= 3e-4 * b[MAX_STUCK]
    assert not close(a, b)  # one too many
    c = b.copy()
    c[0] *= 1 - 2 * LOOSE_RTOL
    assert not close(c, b)  # beyond the loose bound


@pytest.mark.parametrize("key", sorted(PR_MANIFEST))
def test_oracle_pr_matches_reference(gft, orc, key):
    e = PR_MANIFEST[key]
    g = _graph(gft, e["recipe"], e["graph"])
    rank, it = orc.pr(g.row_start, g.edge_dst)
    assert it > 0
    assert close(rank, PR_VALUES[key]), key


def test_pr_golden_noise_is_within_tolerance():
    for key, e in PR_MANIFEST.items():
        assert e["max_abs_diff_between_runs"] <= RTOL * max(1.0, e["rank_max"]), key


def test_product_pr_writer_matches_oracle_text(gft, orc, tmp_path):
    g = _graph(gft, PR_MANIFEST["rmat12w.pr"]["recipe"], "rmat12w")
    rank, _ = orc.pr(g.row_start, g.edge_dst)
    a, b = tmp_path / "a.txt", tmp_path / "b.txt"
    orc.write_pr_output(a, rank)
    gft.write_pr_output(b, rank)
    assert a.read_bytes() == b.read_bytes()


def test_pr_iteration_limit_on_the_oracle(gft, orc):
    g = gft.CSRGraph.road(60, seed=2)
    _, it = orc.pr(g.row_start, g.edge_dst, max_iterations=5)
    assert it == 5


@pytest.mark.gpu
def test_gpu_pr_matches_reference_golden(gft, engine):
    for key, e in sorted(PR_MANIFEST.items()):
        g = _graph(gft, e["recipe"], e["graph"])
        r = engine.pr(g.copy_to_gpu())
        assert close(r["out"].cpu().numpy(), PR_VALUES[key]), key


@pytest.mark.gpu
@pytest.mark.parametrize("tune", [None, {"hub_degree": 32}, {"block_threads": 256, "blocks_per_sm": 4}])
def test_gpu_pr_matches_oracle(gft, orc, engine, tune):
    """Larger graphs, including hubs above the grid-wide split degree (a
    hub's update is stored at its pop and used by the hub phase)."""
    for g in (gft.CSRGraph.rmat(15, 16, seed=12), gft.CSRGraph.road(250, seed=13), gft.CSRGraph.grid(30, 900, 0, 1)):
        want, _ = orc.pr(g.row_start, g.edge_dst)
        r = engine.pr(g.copy_to_gpu(), tune=gft.Tune(**tune) if tune else None)
        assert r["levels"] > 0
        assert close(r["out"].cpu().numpy(), want)


@pytest.mark.gpu
def test_gpu_pr_iteration_limit_and_host_variant(gft, orc, engine):
    g = gft.CSRGraph.road(120, seed=14)
    dg = g.copy_to_gpu()
    r = engine.pr(dg, max_iterations=3)
    assert r["levels"] == 3
    out = np.empty(g.nnodes, dtype=np.float32)
    st = engine.pr_host(dg, out)
    want, _ = orc.pr(g.row_start, g.edge_dst)
    assert st["levels"] > 3 and close(out, want)


def _run_pr_cli(prog: Path, key: str, tmp_path: Path, gft):
    e = PR_MANIFEST[key]
    g = _graph(gft, e["recipe"], e["graph"])
    gr = tmp_path / f"{e['graph']}.gr"
    g.write(gr)
    out = tmp_path / f"{key}.out"
    r = subprocess.run([str(prog), "-o", str(out), str(gr)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert re.search(r"PR took \d+ iterations", r.stdout) and re.search(r"sum: [0-9.]+ \(\d+\)", r.stdout)
    ranks = np.array([float(ln.split()[1]) for ln in out.read_text().splitlines()])
    return ranks


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["rmat14.pr", "road128.pr", "star5000.pr", "disconnected.pr"])
def test_pr_cli_and_dropin_match_reference(gft, tmp_path, key):
    assert close(_run_pr_cli(ROOT / "galoisgpu_b200" / "bin" / "pr", key, tmp_path, gft), PR_VALUES[key])
    dropin = ROOT / "oracle" / "_ref" / "pr_gft"
    if dropin.exists():
        assert close(_run_pr_cli(dropin, key, tmp_path, gft), PR_VALUES[key])
