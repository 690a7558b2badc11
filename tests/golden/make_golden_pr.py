"""Generates the PageRank golden fixtures of tests/golden from the
reference's own CUDA build (oracle/_ref/pr, built by oracle/ref/Makefile from
apps/pr of the reference sources).  Needs a GPU; run from the repository
root:

    python tests/golden/make_golden_pr.py <out_dir>

For every graph of make_golden.graph_cases() with at least one edge it writes
the graph as .gr and runs the reference CLI as a user would (`pr -o out
g.gr`, apps/pr/support.cu), twice, and stores
  - pr_manifest.json: per graph the recipe, the .gr sha256, the iteration
    count of each run ("PR took N iterations", apps/pr/kernel.cu:386) and the
    largest difference between the two runs' ranks;
  - pr_values.npz: the first run's ranks as printed ("%d %f", six decimals).
The reference accumulates float residuals with atomicAdd in the order the
GPU happens to run (apps/pr/kernel.cu:189,221), so its ranks are not
bit-reproducible; the run-to-run difference recorded here is the scale of
that noise.
"""

from __future__ import annotations

import hashlib
import json
import re
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import REF, graph_cases  # noqa: E402
from oracle import oracle as orc  # noqa: E402


def run_ref_pr(gr: Path, out_txt: Path) -> int:
    cmd = [str(REF / "pr"), "-o", str(out_txt), str(gr)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)} failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    m = re.search(r"PR took (\d+) iterations", r.stdout)
    if not m:
        raise RuntimeError(f"no iteration count in output:\n{r.stdout}")
    return int(m.group(1))


def main(out_dir: str) -> int:
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    manifest, values = {}, {}
    for name, recipe, g in graph_cases():
        if g.nedges == 0:
            continue
        gr = out / f"{name}.gr"
        g.write(gr)
        ranks, iters = [], []
        for run in range(2):
            txt = out / f"{name}.pr{run}.txt"
            iters.append(run_ref_pr(gr, txt))
            ranks.append(orc.read_pr_output(txt, g.nnodes))
            txt.unlink()
        if np.isnan(ranks[0]).any():
            raise RuntimeError(f"{name}: missing rank lines")
        key = f"{name}.pr"
        values[key] = ranks[0]
        manifest[key] = {
            "graph": name,
            "recipe": recipe,
            "gr_sha256": hashlib.sha256(gr.read_bytes()).hexdigest(),
            "app": "pr",
            "iterations_runs": iters,
            "max_abs_diff_between_runs": float(np.abs(ranks[0] - ranks[1]).max()),
            "rank_max": float(ranks[0].max()),
        }
        gr.unlink()
        print(key, iters, manifest[key]["max_abs_diff_between_runs"], flush=True)
    np.savez_compressed(out / "pr_values.npz", **values)
    (out / "pr_manifest.json").write_text(json.dumps(manifest, indent=1, sort_keys=True))
    print(f"{len(manifest)} cases written to {out}")
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    sys.exit(main(sys.argv[1]))
