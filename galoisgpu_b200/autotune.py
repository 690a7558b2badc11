"""Autotuner for the traversal kernels.

Replaces the reference's OpenTuner scripts (tuning/lsgtuner.py:123-219,
tuning/bfstuner.py, tuning/sssptuner.py), which rebuilt the binary per block
size and scraped its output.  Here every tunable is a launch-time parameter,
so a candidate costs only a few queries on a resident graph:

  block_threads   CTA size of the persistent kernel (256 / 512 / 1024)
  blocks_per_sm   persistent CTAs per SM (capped by occupancy)
  hub_degree      degree at which a frontier vertex is split across the grid
  delta           SSSP bucket width (distances do not depend on it)

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

from .graph import DEFAULT_DELTA, DeviceGraph, Engine, Tune

BLOCKS = (256, 512, 1024)
BLOCKS_PER_SM = (1, 2, 3, 4)
HUB_DEGREES = (256, 1024, 4096, 16384, 65536)
DELTAS = (2500, 5000, 10000, 20000, 40000, 80000, 160000, 320000)


@dataclass
class Tuned:
    app: str
    block_threads: int = 512
    blocks_per_sm: int = 2
    hub_degree: int = 4096
    delta: int = DEFAULT_DELTA
    ms: float = float("inf")
    trials: list = field(default_factory=list)

    def tune(self) -> Tune:
        return Tune(block_threads=self.block_threads, blocks_per_sm=self.blocks_per_sm, hub_degree=self.hub_degree)


def _time(engine: Engine, graph: DeviceGraph, app: str, sources, cand: Tuned, reps: int, out) -> float:
    ms = []
    for _ in range(reps):
        for s in sources:
            if app == "sssp":
                r = engine.sssp(graph, s, delta=cand.delta, out=out, tune=cand.tune())
            else:
                r = engine.bfs(graph, s, out=out, tune=cand.tune())
            ms.append(r["kernel_ms"])
    return statistics.median(ms)


def autotune(engine: Engine, graph: DeviceGraph, app: str, sources, reps: int = 3, rounds: int = 2,
             axes: dict | None = None, log=None) -> Tuned:
    """Coordinate-descent search; returns the best configuration found."""
    import torch

    out = torch.empty(graph.nnodes, dtype=torch.int32, device=f"cuda:{graph.device}")
    axes = dict(axes or {})
    axes.setdefault("block_threads", BLOCKS)
    axes.setdefault("blocks_per_sm", BLOCKS_PER_SM)
    axes.setdefault("hub_degree", HUB_DEGREES)
    if app == "sssp":
        axes.setdefault("delta", DELTAS)
    best = Tuned(app)
    best.ms = _time(engine, graph, app, sources, best, reps, out)
    best.trials.append({**{k: getattr(best, k) for k in axes}, "ms": best.ms})
    for _ in range(rounds):
        improved = False
        for axis, values in axes.items():
            for v in values:
                if getattr(best, axis) == v:
                    continue
                cand = Tuned(**{**asdict(best), "trials": []})
                setattr(cand, axis, v)
                t = _time(engine, graph, app, sources, cand, reps, out)
                best.trials.append({**{k: getattr(cand, k) for k in axes}, "ms": t})
                if log:
                    log(f"{axis}={v}: {t:.3f} ms (best {best.ms:.3f})")
                if t < best.ms * 0.99:
                    for k in axes:
                        setattr(best, k, getattr(cand, k))
                    best.ms = t
                    improved = True
        if not improved:
            break
    return best


def save(path: str | Path, results: dict[str, Tuned]) -> None:
    Path(path).write_text(json.dumps({k: asdict(v) for k, v in results.items()}, indent=1))


def load(path: str | Path) -> dict[str, Tuned]:
    raw = json.loads(Path(path).read_text())
    return {k: Tuned(**v) for k, v in raw.items()}


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
                   log=lambda m: print(m, file=sys.stderr, flush=True))
    results = load(a.out) if Path(a.out).exists() else {}
    results[a.name] = res
    save(a.out, results)
    print(json.dumps({a.name: {k: v for k, v in asdict(res).items() if k != "trials"}}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
