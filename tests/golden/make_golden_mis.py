"""Generates the maximal-independent-set golden fixtures of tests/golden from
the reference's own CUDA build (oracle/_ref/mis, built by oracle/ref/Makefile
from apps/mis of the reference sources, with oracle/ref/mis_driver.cu running
its host-driven round loop).  Needs a GPU; run from the repository root:

    python tests/golden/make_golden_mis.py <out_dir>

For every graph of make_golden.graph_cases() with at least one edge, and two
graphs larger than the reference's priority-thread count (so that some
threads give priorities to several vertices), it writes the graph as .gr and
runs the reference CLI as a user would (`mis -o out g.gr`), twice, and stores
  - mis_manifest.json: per graph the recipe, the .gr sha256, the set size,
    the round count of each run ("Total steps: N") and whether the two runs
    wrote the same set;
  - mis_values.npz: the set as a membership bitmask (numpy packbits, bit
    order little: vertex v is bit v % 8 of byte v // 8).
The reference's priorities come from one xorshift128 stream per thread of
kernel_sizing's grid (apps/mis/kernel.cu:18-41, skelapp/skel.cu:37-43), so
they depend on the GPU's SM count; the manifest records the thread count.
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


def run_ref_mis(gr: Path, out_txt: Path) -> int:
    cmd = [str(REF / "mis"), "-o", str(out_txt), str(gr)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)} failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    m = re.search(r"Total steps: (\d+)", r.stdout)
    if not m:
        raise RuntimeError(f"no step count in output:\n{r.stdout}")
    return int(m.group(1))


def mis_cases():
    import galoisgpu_b200 as gft

    out = [c for c in graph_cases() if c[2].nedges > 0]
    out.append(("road600s3", {"kind": "road", "side": 600, "seed": 3}, gft.CSRGraph.road(600, seed=3)))
    out.append(("rmat19e8", {"kind": "rmat", "scale": 19, "edge_factor": 8, "seed": 4, "max_weight": 0},
                gft.CSRGraph.rmat(19, 8, seed=4)))
    return out


def main(out_dir: str) -> int:
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    nthreads = 8 * sms * 256
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    manifest, values = {}, {}
    for name, recipe, g in mis_cases():
        gr = out / f"{name}.gr"
        g.write(gr)
        sets, steps = [], []
        for run in range(2):
            txt = out / f"{name}.mis{run}.txt"
            steps.append(run_ref_mis(gr, txt))
            sets.append(np.flatnonzero(orc.read_mis_output(txt, g.nnodes)).astype(np.int32))
            txt.unlink()
        key = f"{name}.mis"
        mask = np.zeros(g.nnodes, dtype=bool)
        mask[sets[0]] = True
        values[key] = np.packbits(mask, bitorder="little")
        mine, my_steps = orc.mis(g.row_start, g.edge_dst, nthreads)
        manifest[key] = {
            "graph": name,
            "recipe": recipe,
            "nnodes": g.nnodes,
            "gr_sha256": hashlib.sha256(gr.read_bytes()).hexdigest(),
            "app": "mis",
            "prio_threads": nthreads,
            "set_size": int(len(sets[0])),
            "steps_runs": steps,
            "runs_identical": bool(np.array_equal(sets[0], sets[1])),
            "oracle_identical": bool(np.array_equal(np.flatnonzero(mine == 1), sets[0])),
            "oracle_steps": my_steps,
        }
        gr.unlink()
        print(key, steps, len(sets[0]), manifest[key]["runs_identical"], manifest[key]["oracle_identical"], flush=True)
    np.savez_compressed(out / "mis_values.npz", **values)
    (out / "mis_manifest.json").write_text(json.dumps(manifest, indent=1, sort_keys=True))
    print(f"{len(manifest)} cases written to {out}")
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    sys.exit(main(sys.argv[1]))
