"""Times the reference's own CUDA build (oracle/_ref, built by
oracle/ref/Makefile from the reference sources) on the full-size seeded
configurations, the way a user runs it: ``bfs|sssp -q -s <src> [-d delta]
<graph.gr>``, ``cc -q <graph.gr>``, ``pr -q <graph.gr>`` or ``mis -q
<graph.gr>``, one process per query, reading its
``Total time: N ns`` line
(reference skelapp/skel.cu:159-166; that time includes the worklist
allocations gg_main makes, apps/bfs/kernel.cu:389, apps/sssp/kernel.cu:475).
Kernel-only time comes from running this same script under
``ncu --metrics gpu__time_duration.sum -k regex:gg_main_pipe`` (for cc, every
kernel of the process: its driver is a host loop of launches; for pr the
init kernels and the persistent gg_main_pipe_1_gpu_gb; for mis gen_prio_gpu
and the round kernels).

Test/measurement infrastructure only: the input graphs are produced with this
repository's generator, and E_r comes from this repository's engine (whose
reach sets equal the reference's, checked with --check).

    python oracle/ref/run_ref_bench.py --config road4096 --sources 1 --check
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

import galoisgpu_b200 as gft  # noqa: E402
from oracle import oracle as orc  # noqa: E402

REF = ROOT / "oracle" / "_ref"
CONFIGS = {
    "grid256": dict(kind="grid", kw=dict(rows=256, cols=256, max_weight=1), seed=0, app="bfs", src_seed=None),
    "road4096": dict(kind="road", kw=dict(side=4096), seed=1, app="sssp", src_seed=1, delta=10000),
    "rmat24": dict(kind="rmat", kw=dict(scale=24, edge_factor=16), seed=1, app="bfs", src_seed=2),
    "road1024": dict(kind="road", kw=dict(side=1024), seed=1, app="sssp", src_seed=1, delta=10000),
    "rmat20": dict(kind="rmat", kw=dict(scale=20, edge_factor=16), seed=1, app="bfs", src_seed=2),
    "cc-rmat24": dict(kind="rmat", kw=dict(scale=24, edge_factor=16), seed=1, app="cc", src_seed=None),
    "cc-road4096": dict(kind="road", kw=dict(side=4096), seed=1, app="cc", src_seed=None),
    "pr-rmat24": dict(kind="rmat", kw=dict(scale=24, edge_factor=16), seed=1, app="pr", src_seed=None),
    "pr-road4096": dict(kind="road", kw=dict(side=4096), seed=1, app="pr", src_seed=None),
    "mis-rmat24": dict(kind="rmat", kw=dict(scale=24, edge_factor=16), seed=1, app="mis", src_seed=None),
    "mis-road4096": dict(kind="road", kw=dict(side=4096), seed=1, app="mis", src_seed=None),
}


def run_mis(a, c, dg, host, eng, gr: Path) -> int:
    """The reference's MIS (oracle/_ref/mis: its kernels through its host
    round loop) against this engine's: total time, rounds, and with --check
    whether the sets are identical."""
    mine = eng.mis(dg)
    cmd = [str(REF / "mis")]
    out = Path(a.workdir) / f"gft_{a.config}.mis.out"
    cmd += ["-o", str(out)] if a.check else ["-q"]
    t = time.time()
    r = subprocess.run(cmd + [str(gr)], capture_output=True, text=True, timeout=1800)
    wall = time.time() - t
    if r.returncode != 0:
        print(r.stdout, r.stderr, file=sys.stderr)
        return r.returncode
    m = re.search(r"Total time: (\d+) ns", r.stderr)
    ns = int(m.group(1)) if m else None
    steps = int(re.search(r"Total steps: (\d+)", r.stdout).group(1))
    rec = {"config": a.config, "app": "mis", "total_time_ns": ns, "steps": steps, "edges": dg.nedges,
           "gft_kernel_ms": mine["kernel_ms"], "gft_steps": mine["levels"], "gft_set_size": mine["vertices_reached"],
           "process_wall_s": wall}
    ok = steps == mine["levels"]
    if a.check:
        ref = orc.read_mis_output(out, host.nnodes)
        same = bool(np.array_equal(ref, mine["out"].cpu().numpy() == 1))
        rec["parity_vs_gft"] = "identical set" if same else "MISMATCH"
        ok = ok and same
        out.unlink()
    print(json.dumps(rec), flush=True)
    gr.unlink()
    return 0 if ok else 1


def run_pr(a, c, dg, host, eng, gr: Path) -> int:
    """The reference's PageRank to convergence against this engine's: total
    time, iterations, and with --check the largest rank difference (float
    atomics make neither side bit-reproducible)."""
    mine = eng.pr(dg)
    cmd = [str(REF / "pr")]
    out = Path(a.workdir) / f"gft_{a.config}.pr.out"
    cmd += ["-o", str(out)] if a.check else ["-q"]
    t = time.time()
    r = subprocess.run(cmd + [str(gr)], capture_output=True, text=True, timeout=1800)
    wall = time.time() - t
    if r.returncode != 0:
        print(r.stdout, r.stderr, file=sys.stderr)
        return r.returncode
    m = re.search(r"Total time: (\d+) ns", r.stderr)
    ns = int(m.group(1)) if m else None
    it = int(re.search(r"PR took (\d+) iterations", r.stdout).group(1))
    rec = {"config": a.config, "app": "pr", "total_time_ns": ns, "iterations": it, "edges": dg.nedges,
           "gft_kernel_ms": mine["kernel_ms"], "gft_iterations": mine["levels"],
           "gft_edges_pushed": mine["edges_scanned"], "process_wall_s": wall}
    if a.check:
        ref = orc.read_pr_output(out, host.nnodes)
        got = mine["out"].cpu().numpy()
        err = np.abs(got - ref) / np.maximum(1.0, np.abs(ref))
        rec["max_rel_diff_vs_gft"] = float(err.max())
        rec["vertices_over_1e-4"] = int(np.count_nonzero(err > 1e-4))
        out.unlink()
    print(json.dumps(rec), flush=True)
    gr.unlink()
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=sorted(CONFIGS), required=True)
    ap.add_argument("--sources", type=int, default=1)
    ap.add_argument("--delta", type=int, default=None)
    ap.add_argument("--workdir", default=os.environ.get("TMPDIR", tempfile.gettempdir()))
    ap.add_argument("--check", action="store_true", help="compare the reference output with this engine's")
    a = ap.parse_args(argv)
    c = CONFIGS[a.config]
    dg = gft.DeviceGraph.generate(c["kind"], seed=c["seed"], **c["kw"])
    host = dg.download()
    srcs = [0] if c["src_seed"] is None else host.pick_sources(c["src_seed"], a.sources)
    gr = Path(a.workdir) / f"gft_{a.config}.gr"
    t0 = time.time()
    host.write(gr)
    sha = hashlib.sha256(gr.read_bytes()).hexdigest()[:16]
    print(f"wrote {gr} ({gr.stat().st_size / 1e9:.2f} GB, sha256 {sha}) in {time.time() - t0:.1f}s",
          file=sys.stderr, flush=True)
    eng = gft.Engine(0)
    delta = a.delta or c.get("delta")
    results = []
    if c["app"] == "pr":
        return run_pr(a, c, dg, host, eng, gr)
    if c["app"] == "mis":
        return run_mis(a, c, dg, host, eng, gr)
    if c["app"] == "cc":
        # Component count only: the reference's CC output lists every edge
        # (apps/cc/support.cu:30-35), about 15 GB of text for RMAT-24.
        mine = eng.cc(dg)
        t = time.time()
        r = subprocess.run([str(REF / "cc"), "-q", str(gr)], capture_output=True, text=True, timeout=1800)
        wall = time.time() - t
        if r.returncode != 0:
            print(r.stdout, r.stderr, file=sys.stderr)
            return r.returncode
        m = re.search(r"Total time: (\d+) ns", r.stderr)
        ns = int(m.group(1)) if m else None
        comps = int(re.search(r"components: (\d+)", r.stdout).group(1))
        rec = {"config": a.config, "app": "cc", "total_time_ns": ns, "edges": dg.nedges,
               "gteps_total_time": dg.nedges / ns if ns else None, "components": comps,
               "components_gft": mine["components"], "gft_kernel_ms": mine["kernel_ms"],
               "parity_vs_gft": "same count" if comps == mine["components"] else "MISMATCH",
               "process_wall_s": wall}
        print(json.dumps(rec), flush=True)
        gr.unlink()
        return 0 if comps == mine["components"] else 1
    for i, s in enumerate(srcs):
        mine = (eng.sssp(dg, s, delta=delta) if c["app"] == "sssp" else eng.bfs(dg, s))["out"]
        v_r, e_r = gft.reach_stats(dg, mine)
        out = Path(a.workdir) / f"gft_{a.config}.s{s}.out"
        check = a.check and i == 0
        cmd = [str(REF / c["app"]), "-s", str(s)]
        if c["app"] == "sssp":
            cmd += ["-d", str(delta)]
        cmd += ["-o", str(out)] if check else ["-q"]
        cmd.append(str(gr))
        t = time.time()
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
        wall = time.time() - t
        if r.returncode != 0:
            print(r.stdout, r.stderr, file=sys.stderr)
            return r.returncode
        m = re.search(r"Total time: (\d+) ns", r.stderr)
        ns = int(m.group(1)) if m else None
        rec = {"config": a.config, "app": c["app"], "src": s, "delta": delta, "total_time_ns": ns,
               "gteps_total_time": e_r / ns if ns else None, "E_r": e_r, "V_r": v_r, "process_wall_s": wall}
        if check:
            ref = orc.read_output(out, host.nnodes)
            rec["parity_vs_gft"] = "bit-exact" if np.array_equal(ref, mine.cpu().numpy()) else "MISMATCH"
            out.unlink()
        results.append(rec)
        print(json.dumps(rec), flush=True)
    gr.unlink()
    return 0


if __name__ == "__main__":
    sys.exit(main())
