"""The autotuner's search (coordinate descent over every launch-time axis)
against a stand-in engine with a known optimum, and the committed tuned
parameters: every workload records every axis."""

import json
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


class _FakeGraph:
    nnodes = 8
    device = 0


class _FakeEngine:
    """Kernel time as a separable function of the tunables, with its minimum
    at OPT; SSSP at 1024 threads rejects tiles above 128, as the engine does."""

    OPT = dict(block_threads=1024, blocks_per_sm=3, hub_degree=1024, queue_tile=128, warp_degree=64, delta=40000,
               fuse_budget=512)
    ORDER = dict(block_threads=(256, 512, 1024), blocks_per_sm=(1, 2, 3, 4), hub_degree=(256, 1024, 4096, 16384, 65536),
                 queue_tile=(64, 128, 256), warp_degree=(8, 16, 32, 64, 128),
                 delta=(2500, 5000, 10000, 20000, 40000, 80000, 160000, 320000),
                 fuse_budget=(2**32 - 1, 64, 128, 256, 512, 1024))

    def __init__(self, gft):
        self.gft = gft
        self.calls = 0

    def _ms(self, values):
        return 1.0 + sum(abs(self.ORDER[k].index(v) - self.ORDER[k].index(self.OPT[k])) for k, v in values.items())

    def _run(self, tune, delta=None):
        self.calls += 1
        v = {k: getattr(tune, k) for k in ("block_threads", "blocks_per_sm", "hub_degree", "queue_tile", "warp_degree")}
        if delta is not None:
            if tune.block_threads == 1024 and tune.queue_tile > 128:
                raise self.gft.GftError(1, "queue_tile")  # GFT_ERR_INVALID_ARG
            v["delta"] = delta
            v["fuse_budget"] = tune.fuse_budget
        return {"kernel_ms": self._ms(v)}

    def sssp(self, graph, s, delta, out, tune):
        return self._run(tune, delta)

    def bfs(self, graph, s, out, tune):
        return self._run(tune)


def test_search_reaches_the_optimum_and_skips_unbuilt_tiles(gft):
    from galoisgpu_b200 import autotune as at

    assert gft.GftError(1, "x").status_name == "GFT_ERR_INVALID_ARG"
    eng = _FakeEngine(gft)
    best = at.autotune(eng, _FakeGraph(), "sssp", [0, 1], reps=1, rounds=6, uniform=True, out=object())
    for k, v in _FakeEngine.OPT.items():
        assert getattr(best, k) == v, (k, getattr(best, k))
    assert best.ms == 1.0
    assert all(t["ms"] == float("inf") or t["ms"] >= 1.0 for t in best.trials)
    bfs = at.autotune(_FakeEngine(gft), _FakeGraph(), "bfs", [0], reps=1, rounds=6, out=object())
    assert (bfs.block_threads, bfs.queue_tile, bfs.warp_degree) == (1024, 128, 64)


def test_cta_size_and_count_are_swept_together(gft):
    """An optimum that no single-axis step reaches: the start (512, 2) costs
    3, one step on the CTA size reaches (1024, 2) at 2, and from there no
    single step on either axis reaches (512, 4) at 1."""
    from galoisgpu_b200 import autotune as at

    class Ridge(_FakeEngine):
        def _ms(self, values):
            shape = {(512, 4): 1.0, (1024, 2): 2.0, (512, 2): 3.0}.get(
                (values["block_threads"], values["blocks_per_sm"]), 5.0)
            return shape + 0.01 * sum(abs(self.ORDER[k].index(v) - self.ORDER[k].index(self.OPT[k]))
                                      for k, v in values.items() if k not in ("block_threads", "blocks_per_sm"))

    best = at.autotune(Ridge(gft), _FakeGraph(), "bfs", [0], reps=1, rounds=4, out=object())
    assert (best.block_threads, best.blocks_per_sm) == (512, 4)
    assert {"block_threads", "blocks_per_sm"} <= set(best.trials[0])


def test_start_point_is_the_engine_default():
    from galoisgpu_b200 import autotune as at

    s = at.start_point("sssp", uniform=True)
    assert (s.block_threads, s.blocks_per_sm, s.queue_tile, s.warp_degree, s.fuse_budget) == (512, 2, 256, 32, 256)
    assert at.start_point("sssp", uniform=False).fuse_budget == at.NEVER


@pytest.mark.parametrize("name", ["sssp-road-4096", "bfs-rmat-24"])
def test_committed_tuning_records_every_axis(name):
    from galoisgpu_b200 import autotune as at

    raw = json.loads((ROOT / "galoisgpu_b200" / "tuned_b200.json").read_text())
    t = raw[name]
    for axis in ("block_threads", "blocks_per_sm", "hub_degree", "queue_tile", "warp_degree"):
        assert axis in t and t[axis] > 0, axis
    if name.startswith("sssp"):
        assert t["delta"] > 0 and "fuse_budget" in t
    assert t["trials"], "the sweep is recorded"
    loaded = at.load(ROOT / "galoisgpu_b200" / "tuned_b200.json")[name]
    assert loaded.tune().queue_tile == t["queue_tile"]
