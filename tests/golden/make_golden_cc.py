"""Generates the connected-components golden fixtures of tests/golden from
the reference's own CUDA build (oracle/_ref/cc, built by oracle/ref/Makefile
from apps/cc of the reference sources).  Needs a GPU; run from the
repository root:

    python tests/golden/make_golden_cc.py <out_dir>

For every graph of make_golden.graph_cases() with at least one edge (the
reference cannot load an edgeless graph) it writes the graph as .gr, runs
the reference CLI as a user would (`cc -o out g.gr`, apps/cc/README.md), and
stores
  - cc_manifest.json: per graph the recipe, the .gr sha256, the component
    count the reference printed ("components: N", apps/cc/kernel.cu:719),
    and the sha256 of its output text;
  - cc_values.npz: the partition, relabelled so every vertex carries the
    smallest vertex id of its component.
The reference's labels are the roots its racy hooks happen to leave
(apps/cc/kernel.cu:263,293,329), so the text differs between runs; the
partition and the count do not.  It is run twice per graph and both
partitions must agree before they are recorded.
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


def read_cc_output(path: Path, nnodes: int) -> np.ndarray:
    """Node lines of the reference's CC output ("%d %d\\n"; the per-edge
    lines start with a tab), apps/cc/support.cu:30-35."""
    lab = np.full(nnodes, -1, dtype=np.int64)
    with open(path) as f:
        for ln in f:
            if ln.startswith("\t"):
                continue
            i, v = ln.split()
            lab[int(i)] = int(v)
    if (lab < 0).any():
        raise ValueError(f"{path}: missing node lines")
    return lab.astype(np.int32)


def run_ref_cc(gr: Path, out_txt: Path) -> int:
    cmd = [str(REF / "cc"), "-o", str(out_txt), str(gr)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)} failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    m = re.search(r"components: (\d+)", r.stdout)
    if not m:
        raise RuntimeError(f"no component count in output:\n{r.stdout}")
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
        parts, shas, counts = [], [], []
        for run in range(2):
            txt = out / f"{name}.cc{run}.txt"
            counts.append(run_ref_cc(gr, txt))
            parts.append(orc.canonical_labels(read_cc_output(txt, g.nnodes)))
            shas.append(hashlib.sha256(txt.read_bytes()).hexdigest())
            txt.unlink()
        if counts[0] != counts[1] or not np.array_equal(parts[0], parts[1]):
            raise RuntimeError(f"{name}: the reference's two runs disagree on the partition")
        key = f"{name}.cc"
        values[key] = parts[0]
        manifest[key] = {
            "graph": name,
            "recipe": recipe,
            "gr_sha256": hashlib.sha256(gr.read_bytes()).hexdigest(),
            "app": "cc",
            "components": counts[0],
            "out_sha256_runs": shas,
        }
        gr.unlink()
        print(key, counts[0], "identical text" if shas[0] == shas[1] else "text differs between runs", flush=True)
    np.savez_compressed(out / "cc_values.npz", **values)
    (out / "cc_manifest.json").write_text(json.dumps(manifest, indent=1, sort_keys=True))
    print(f"{len(manifest)} cases written to {out}")
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    sys.exit(main(sys.argv[1]))
