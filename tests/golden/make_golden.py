"""Generates the golden fixtures of tests/golden from the reference's own CUDA
build (oracle/_ref/bfs and oracle/_ref/sssp, built by oracle/ref/Makefile from
the reference sources).  Needs a GPU; run from the repository root:

    python tests/golden/make_golden.py <out_dir>

For every case it writes the graph as .gr with this repository's writer,
runs the reference CLI exactly as a user would (`bfs [-s src] -o out g.gr`,
`sssp [-s src] [-d delta] -o out g.gr`, reference skelapp/skel.cu:88-137),
and stores
  - manifest.json: per case the graph recipe, the sha256 of the .gr file,
    the app/source/delta, the sha256 of the reference's output text and its
    'Total time' line;
  - values.npz: the parsed int32 values of every case (INF = INT_MAX).
The fixtures are then committed under tests/golden/.
"""

from __future__ import annotations

import hashlib
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import galoisgpu_b200 as gft  # noqa: E402
from graphs import hand_cases  # noqa: E402
from oracle import oracle as orc  # noqa: E402

REF = ROOT / "oracle" / "_ref"


def graph_cases():
    """(name, recipe, CSRGraph) -- recipes are re-executed by the tests."""
    out = []
    out.append(("grid256", {"kind": "grid", "rows": 256, "cols": 256, "seed": 0, "max_weight": 1},
                gft.CSRGraph.grid(256, 256, 0, 1)))
    out.append(("grid64x40w", {"kind": "grid", "rows": 64, "cols": 40, "seed": 3, "max_weight": 50},
                gft.CSRGraph.grid(64, 40, 3, 50)))
    out.append(("road128", {"kind": "road", "side": 128, "seed": 1}, gft.CSRGraph.road(128, seed=1)))
    out.append(("road200s7", {"kind": "road", "side": 200, "seed": 7}, gft.CSRGraph.road(200, seed=7)))
    out.append(("rmat12w", {"kind": "rmat", "scale": 12, "edge_factor": 16, "seed": 1, "max_weight": 255},
                gft.CSRGraph.rmat(12, 16, seed=1, max_weight=255)))
    out.append(("rmat14", {"kind": "rmat", "scale": 14, "edge_factor": 16, "seed": 2, "max_weight": 0},
                gft.CSRGraph.rmat(14, 16, seed=2)))
    for name, rs, dst, w in hand_cases():
        out.append((name, {"kind": "hand", "name": name}, gft.CSRGraph(rs, dst, w)))
    return out


def queries(name, g):
    """(app, src, delta, load_balance) tuples.  The reference cannot load a
    graph without edges (its device allocation assert fails,
    rt/src/csr_graph.cu:228-236), so such graphs get no reference queries."""
    if g.nedges == 0:
        return []
    srcs = sorted({0, g.nnodes // 2, g.nnodes - 1}) if g.nnodes < 5000 else ([0] + g.pick_sources(11, 2))
    qs = []
    for s in srcs:
        qs.append(("bfs", s, None, False))
        qs.append(("sssp", s, 10000, False))
        if name.startswith(("road", "rmat12w", "grid64")):
            qs.append(("sssp", s, 97, False))
    # The -l load-balanced, host-driven path (apps/bfs/kernel.cu:286-311).
    if name in ("rmat14", "star5000"):
        qs.append(("bfs", srcs[0], None, True))
    if name in ("road128", "rmat12w"):
        qs.append(("sssp", srcs[0], 10000, True))
    return qs


def run_ref(app, gr, src, delta, lb, out_txt):
    cmd = [str(REF / app), "-s", str(src), "-o", str(out_txt)]
    if lb:
        cmd.append("-l")
    if delta is not None:
        cmd += ["-d", str(delta)]
    cmd.append(str(gr))
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)} failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    total = [ln for ln in r.stderr.splitlines() if ln.startswith("Total time") and ln.endswith("ns")]
    return total[0] if total else ""


def main(out_dir: str) -> int:
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    manifest, values = {}, {}
    for name, recipe, g in graph_cases():
        gr = out / f"{name}.gr"
        g.write(gr)
        sha = hashlib.sha256(gr.read_bytes()).hexdigest()
        for app, src, delta, lb in queries(name, g):
            key = f"{name}.{app}.s{src}" + (f".d{delta}" if delta is not None else "") + (".l" if lb else "")
            txt = out / f"{key}.txt"
            total = run_ref(app, gr, src, delta, lb, txt)
            vals = orc.read_output(txt, g.nnodes)
            values[key] = vals
            manifest[key] = {
                "graph": name,
                "recipe": recipe,
                "gr_sha256": sha,
                "app": app,
                "src": src,
                "delta": delta,
                "load_balance": lb,
                "out_sha256": hashlib.sha256(txt.read_bytes()).hexdigest(),
                "ref_total_time": total,
            }
            txt.unlink()
            print(key, total, flush=True)
        gr.unlink()
    np.savez_compressed(out / "values.npz", **values)
    (out / "manifest.json").write_text(json.dumps(manifest, indent=1, sort_keys=True))
    print(f"{len(manifest)} cases written to {out}")
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    sys.exit(main(sys.argv[1]))
