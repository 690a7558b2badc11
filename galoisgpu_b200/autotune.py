"""Autotuner for the traversal kernels.

Replaces the reference's OpenTuner scripts (tuning/lsgtuner.py:123-219,
tuning/bfstuner.py, tuning/sssptuner.py), which rebuilt the binary per block
size and scraped its output.  Here every tunable is a launch-time parameter,
so a candidate costs only a few queries on a resident graph:

  block_threads   CTA size of the persistent kernel (256 / 512 / 1024) and
  blocks_per_sm   persistent CTAs per SM (capped by occupancy), swept as one
                  axis of pairs: the best pair can be worse than its
                  neighbours on both single axes (BFS on RMAT-24: 512 x 4
                  0.70 ms, 1024 x 2 0.74 ms, 512 x 2 0.96 ms, 1024 x 4 capped
                  to 1024 x 2), which a one-axis step never crosses
  hub_degree      degree at which a frontier vertex is split across the grid
  queue_tile      push-buffer entries per warp (64 / 128 / 256; kernels are
                  built for each, so the tile is picked per launch; the
                  reference's tuner rebuilt for its compile-time tile,
                  rt/include/ggcuda.h:19-22)
  warp_degree     degree from which a whole warp expands a vertex (smaller
                  edge lists are flattened across the warp)
  delta           SSSP bucket width (distances do not depend on it)
  fuse_budget     SSSP near vertices a warp expands in the iteration that
                  found them (bucket fusion; NEVER = off)

A candidate the engine rejects (an SSSP tile of 256 at 1024 threads, whose
near and far buffers would not fit static shared memory) is skipped.

The search is a coordinate descent from the engine defaults: each axis is
swept with the others fixed at the best values so far, for `rounds` rounds;
every candidate is timed as the median device time of `reps` queries over
the given sources.  Results are JSON (``save`` / ``load``), keyed by a
workload name.

    python -m galoisgpu_b200.autotune --workload sssp-road-4096 --out tuned.json
"""

from __future__ import annotations

import argparse
import json
import statistics
import sys
from dataclasses import asdict, dataclass, field
from pathlib import Path

from ._lib import GftError
from .graph import DEFAULT_DELTA, DeviceGraph, Engine, Tune

BLOCKS = (256, 512, 1024)
BLOCKS_PER_SM = (1, 2, 3, 4)
SHAPE = ("block_threads", "blocks_per_sm")  # swept together
SHAPES = tuple((b, k) for b in BLOCKS for k in BLOCKS_PER_SM)
HUB_DEGREES = (256, 1024, 4096, 16384, 65536)
QUEUE_TILES = (64, 128, 256)
WARP_DEGREES = (8, 16, 32, 64, 128)
DELTAS = (2500, 5000, 10000, 20000, 40000, 80000, 160000, 320000)
NEVER = 2**32 - 1  # fuse_budget: no bucket fusion
FUSE_BUDGETS = (NEVER, 64, 128, 256, 512, 1024)
UNIFORM_MAX_DEGREE = 32  # the engine's uniform-degree graphs (static chunks, fusion on by default)


@dataclass
class Tuned:
    app: str
    block_threads: int = 512
    blocks_per_sm: int = 2
    hub_degree: int = 4096
    queue_tile: int = 256
    warp_degree: int = 32
    delta: int = DEFAULT_DELTA
    fuse_budget: int = NEVER
    ms: float = float("inf")
    trials: list = field(default_factory=list)

    def tune(self) -> Tune:
        return Tune(block_threads=self.block_threads, blocks_per_sm=self.blocks_per_sm, hub_degree=self.hub_degree,
                    queue_tile=self.queue_tile, warp_degree=self.warp_degree,
                    fuse_budget=self.fuse_budget if self.app == "sssp" else 0)


def start_point(app: str, uniform: bool) -> Tuned:
    """The engine's defaults, spelled out (so every axis has a value)."""
    t = Tuned(app)
    if app == "sssp":
        t.fuse_budget = 256 if uniform else NEVER
    return t


def _time(engine: Engine, graph: DeviceGraph, app: str, sources, cand: Tuned, reps: int, out) -> float:
    ms = []
    try:
        for _ in range(reps):
            for s in sources:
                if app == "sssp":
                    r = engine.sssp(graph, s, delta=cand.delta, out=out, tune=cand.tune())
                else:
                    r = engine.bfs(graph, s, out=out, tune=cand.tune())
                ms.append(r["kernel_ms"])
    except GftError as e:
        if e.status_name != "GFT_ERR_INVALID_ARG":
            raise
        return float("inf")  # a combination the engine does not build
    return statistics.median(ms)


def _fields(axes: dict) -> list:
    """Tuned fields the axes cover (an axis is a field name or a tuple of them)."""
    out = []
    for a in axes:
        out.extend(a if isinstance(a, tuple) else (a,))
    return out


def _get(t: Tuned, axis):
    return tuple(getattr(t, f) for f in axis) if isinstance(axis, tuple) else getattr(t, axis)


def _set(t: Tuned, axis, value) -> None:
    if isinstance(axis, tuple):
        for f, v in zip(axis, value):
            setattr(t, f, v)
    else:
        setattr(t, axis, value)


def autotune(engine: Engine, graph: DeviceGraph, app: str, sources, reps: int = 3, rounds: int = 2,
             axes: dict | None = None, log=None, uniform: bool = False, out=None) -> Tuned:
    """Coordinate-descent search from the engine defaults (`uniform`: the
    graph's degrees are at most UNIFORM_MAX_DEGREE); returns the best
    configuration found.  `out`: the queries' output array (default: a new
    device array)."""
    if out is None:
        import torch

        out = torch.empty(graph.nnodes, dtype=torch.int32, device=f"cuda:{graph.device}")
    axes = dict(axes or {})
    if "block_threads" not in axes and "blocks_per_sm" not in axes:
        axes.setdefault(SHAPE, SHAPES)
    axes.setdefault("hub_degree", HUB_DEGREES)
    axes.setdefault("queue_tile", QUEUE_TILES)
    axes.setdefault("warp_degree", WARP_DEGREES)
    if app == "sssp":
        axes.setdefault("delta", DELTAS)
        axes.setdefault("fuse_budget", FUSE_BUDGETS)
    fields = _fields(axes)
    best = start_point(app, uniform)
    best.ms = _time(engine, graph, app, sources, best, reps, out)
    best.trials.append({**{k: getattr(best, k) for k in fields}, "ms": best.ms})
    for _ in range(rounds):
        improved = False
        for axis, values in axes.items():
            for v in values:
                if _get(best, axis) == v:
                    continue
                cand = Tuned(**{**asdict(best), "trials": []})
                _set(cand, axis, v)
                if app == "sssp" and cand.block_threads == 1024:
                    cand.queue_tile = min(cand.queue_tile, 128)  # the largest SSSP tile built at 1024 threads
                t = _time(engine, graph, app, sources, cand, reps, out)
                best.trials.append({**{k: getattr(cand, k) for k in fields}, "ms": t})
                if log:
                    name = "x".join(axis) if isinstance(axis, tuple) else axis
                    log(f"{name}={v}: {t:.3f} ms (best {best.ms:.3f})")
                if t < best.ms * 0.99:
                    for k in fields:
                        setattr(best, k, getattr(cand, k))
                    best.ms = t
                    improved = True
        if not improved:
            break
    return best


def save(path: str | Path, results: dict[str, Tuned], about: str | None = None) -> None:
    doc = {"_about": about} if about else {}
    doc.update({k: asdict(v) for k, v in results.items()})
    Path(path).write_text(json.dumps(doc, indent=1))


def load(path: str | Path) -> dict[str, Tuned]:
    raw = json.loads(Path(path).read_text())
    out = {}
    for k, v in raw.items():
        if k.startswith("_"):
            continue
        v = dict(v)
        v.setdefault("app", "sssp" if k.startswith("sssp") else "bfs")
        out[k] = Tuned(**{f: x for f, x in v.items() if f in Tuned.__dataclass_fields__})
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--kind", choices=("road", "rmat", "grid"), required=True)
    ap.add_argument("--app", choices=("bfs", "sssp"), required=True)
    ap.add_argument("--size", type=int, required=True, help="road/grid side or rmat scale")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--sources", type=int, default=2)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--rounds", type=int, default=2)
    ap.add_argument("--name", required=True)
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    if a.kind == "road":
        g = DeviceGraph.generate("road", seed=a.seed, side=a.size)
    elif a.kind == "rmat":
        g = DeviceGraph.generate("rmat", seed=a.seed, scale=a.size, max_weight=255 if a.app == "sssp" else 0)
    else:
        g = DeviceGraph.generate("grid", seed=a.seed, rows=a.size, cols=a.size)
    host = g.download()
    srcs = host.pick_sources(a.seed, a.sources)
    eng = Engine(g.device)
    res = autotune(eng, g, a.app, srcs, reps=a.reps, rounds=a.rounds,
                   log=lambda m: print(m, file=sys.stderr, flush=True),
                   uniform=int(host.degrees().max()) <= UNIFORM_MAX_DEGREE)
    about = None
    if Path(a.out).exists():
        about = json.loads(Path(a.out).read_text()).get("_about")
    results = load(a.out) if Path(a.out).exists() else {}
    results[a.name] = res
    save(a.out, results, about)
    print(json.dumps({a.name: {k: v for k, v in asdict(res).items() if k != "trials"}}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
