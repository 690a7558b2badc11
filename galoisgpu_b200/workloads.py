"""Seeded multi-graph workloads for batching and serving.

batch set (512 queries): graph i has a node count log-uniform in
[1e3, 2e6] (draw i of a SplitMix64 stream seeded 1000); even i is a road
grid of side round(sqrt(V)) (weights uniform [1, 10000]), odd i an R-MAT of
scale round(log2 V) with edge factor 8 (weights uniform [1, 255]); graph i
uses seed 1000 + i and one SSSP source drawn with that seed.

serving set (8 resident graphs): road grids 1024^2, 2048^2, 3072^2, 4096^2
(weights [1, 10000]) and R-MAT scales 18, 20, 22, 23 (edge factor 8, weights
[1, 255]), seed 1.

The reference's downloaded inputs are not available; these stand in for
them with the configured shapes, sizes and weight ranges.
"""

from __future__ import annotations

import math

from .graph import DeviceGraph

_M64 = (1 << 64) - 1
_GAMMA = 0x9E3779B97F4A7C15


def _mix64(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def uniform(seed: int, i: int) -> float:
    """Draw i of the SplitMix64 sequence keyed by `seed`, in [0, 1)."""
    return (_mix64((seed + (i + 1) * _GAMMA) & _M64) >> 11) * 2.0**-53


def batch_specs(n: int = 512, seed: int = 1000, vmin: float = 1e3, vmax: float = 2e6) -> list[dict]:
    out = []
    for i in range(n):
        v = vmin * (vmax / vmin) ** uniform(seed, i)
        if i % 2 == 0:
            side = max(2, round(math.sqrt(v)))
            out.append({"kind": "road", "side": side, "seed": seed + i, "max_weight": 10000, "nodes": side * side})
        else:
            scale = max(2, round(math.log2(v)))
            out.append({"kind": "rmat", "scale": scale, "edge_factor": 8, "seed": seed + i, "max_weight": 255,
                        "nodes": 1 << scale})
    return out


def serving_specs() -> list[dict]:
    out = [{"kind": "road", "side": s, "seed": 1, "max_weight": 10000, "nodes": s * s} for s in (1024, 2048, 3072, 4096)]
    out += [{"kind": "rmat", "scale": s, "edge_factor": 8, "seed": 1, "max_weight": 255, "nodes": 1 << s}
            for s in (18, 20, 22, 23)]
    return out


def build(spec: dict, device: int = 0) -> DeviceGraph:
    if spec["kind"] == "road":
        return DeviceGraph.generate("road", device=device, seed=spec["seed"], side=spec["side"],
                                    max_weight=spec["max_weight"])
    if spec["kind"] == "rmat":
        return DeviceGraph.generate("rmat", device=device, seed=spec["seed"], scale=spec["scale"],
                                    edge_factor=spec["edge_factor"], max_weight=spec["max_weight"])
    return DeviceGraph.generate("grid", device=device, seed=spec["seed"], rows=spec["rows"], cols=spec["cols"],
                                max_weight=spec.get("max_weight", 1))


def name(spec: dict) -> str:
    if spec["kind"] == "road":
        return f"road{spec['side']}"
    if spec["kind"] == "rmat":
        return f"rmat{spec['scale']}"
    return f"grid{spec['rows']}x{spec['cols']}"
