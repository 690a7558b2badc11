#!/usr/bin/env python
"""Benchmark of the B200 frontier-traversal engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gft|reference]
                    [--workload NAME]

A step is one single-source query over a resident seeded graph.  The
headline workload is SSSP on the 4096^2 road-like grid (16.8 M nodes, 5% of
edges deleted, 0.1% shortcuts, weights uniform [1, 10000], seed 1, source
drawn from the seed).  Its delta comes from the tuned parameters
(galoisgpu_b200/tuned_b200.json, 20000; the reference's default is 10000):
delta changes only the schedule, never the distances.  The metric is GTEPS =
E_r / t, E_r the sum of out-degrees of the reached vertices.  Rank 0 prints
one JSON line.

  value        device-resident throughput: K queries timed with CUDA events
               on the launching stream, max over ranks, all ranks' work summed
  e2e          the same queries through the C ABI host-buffer calls:
               every step's source in and all its nnodes results copied back
               to pinned host memory inside the timed region.  The value
               uses gft_sssp_host_many / gft_bfs_host_many, which copy a
               query's results back while the next query runs; e2e.one_call
               is one synchronous gft_sssp_host / gft_bfs_host call per step
  roofline     algorithmic bytes of the persistent traversal kernel (SSSP:
               12 E_r + 20 V_r, BFS: 8 E_r + 20 V_r) / its mean launch time,
               against the measured HBM copy bandwidth
  cpu_baseline the CPU oracle (serial Dijkstra / FIFO BFS, one core) on the
               same query, rank 0 at N = 1 only; also checks bit-exact parity
  reference_cuda  N = 1 only: the reference's own CUDA build for sm_100a
               (oracle/_ref, built from the reference sources) on the same
               graphs and sources in the same run: its kernel-only and
               `Total time`, GTEPS, the ratio to this engine, and bit-exact
               parity of every checked query against this engine's output
               (the headline source, 16 RMAT-24 sources, the 256^2 grid);
               --no-reference-build skips it
  secondary    N = 1 only: BFS on RMAT-24 (64 seeded sources, harmonic-mean
               GTEPS, all 64 checked against the CPU oracle) and on the 256^2
               grid; 512 batched SSSP queries; 256-source BFS on RMAT-24;
               serving 8 resident graphs under Poisson load; connected
               components, PageRank and maximal independent set on RMAT-24
               and the road grid (--workload cc-rmat-24, pr-road-4096,
               mis-rmat-24, ... runs one alone)

--impl reference runs the reference arm: the reference's own CUDA build
(oracle/_ref/{bfs,sssp}_multi) on the same seeded graph, sources and step
count, timed on this GPU (the reference has no CPU implementation of this
path).  It loads no part of this engine: the graph comes from
oracle/libgrgen.so.  Rank 0 only.

Multi-GPU: each rank is an independent replica (queries do not shard without
a per-level exchange), so scaling is weak and no collective touches the data
path; torch.distributed only carries the barrier and the max-over-ranks time.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # SSSP on the road-like grid: the configuration the headline metric is quoted on.
    "sssp-road-4096": dict(kind="road", side=4096, seed=1, app="sssp", delta=10000, nsrc=1, src_seed=1),
    # BFS on RMAT-24, 64 seeded non-isolated sources.
    "bfs-rmat-24": dict(kind="rmat", scale=24, edge_factor=16, seed=1, app="bfs", nsrc=64, src_seed=2),
    # BFS from node 0 on the 256^2 grid.
    "bfs-grid-256": dict(kind="grid", rows=256, cols=256, seed=0, app="bfs", nsrc=0, src_seed=0),
    # Smaller cases of the same kernels (profiling captures).
    "sssp-road-1024": dict(kind="road", side=1024, seed=1, app="sssp", delta=10000, nsrc=1, src_seed=1),
    "sssp-road-2048": dict(kind="road", side=2048, seed=1, app="sssp", delta=10000, nsrc=1, src_seed=1),
    "bfs-rmat-20": dict(kind="rmat", scale=20, edge_factor=16, seed=1, app="bfs", nsrc=8, src_seed=2),
}
HEADLINE = "sssp-road-4096"
TUNED = ROOT / "galoisgpu_b200" / "tuned_b200.json"


def tuned_for(gft, name: str, spec: dict):
    """(Tune, delta) from the committed autotuner results, else defaults."""
    try:
        t = json.loads(TUNED.read_text()).get(name)
    except Exception:
        t = None
    delta = spec.get("delta")
    if not t:
        return None, delta, None
    keys = ("block_threads", "blocks_per_sm", "hub_degree", "queue_tile", "warp_degree")
    if spec["app"] == "sssp":
        keys += ("fuse_budget",)
    tune = gft.Tune(**{k: t[k] for k in keys if k in t})
    if spec["app"] == "sssp" and "delta" in t:
        delta = t["delta"]
    return tune, delta, {k: t[k] for k in keys if k in t}
L2_BYTES = 126 * 2**20


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_id: str, fallback_id: str | None = None):
        self.lines: list[str] = []
        self.proc = None
        self._start(gpu_id)
        if not self.lines and fallback_id is not None:
            self._kill()
            self._start(fallback_id)

    def _kill(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.proc = None

    def _start(self, gpu_id: str):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", gpu_id],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return
        self.t = threading.Thread(target=self._read, args=(self.proc,), daemon=True)
        self.t.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 3:
            time.sleep(0.02)

    def _read(self, proc):
        for ln in proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(self.REASONS, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_id_for(dev: int) -> str:
    import torch

    try:
        return f"GPU-{torch.cuda.get_device_properties(dev).uuid}"
    except Exception:
        return str(dev)


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(workload: str, kernel: str) -> tuple[float | None, str | None]:
    """DRAM bytes per launch from the committed ncu summary, if any."""
    f = ROOT / "profiles" / "dram_traffic.txt"
    if not f.exists():
        return None, None
    for ln in f.read_text().splitlines():
        parts = ln.split()
        if len(parts) >= 3 and not ln.startswith("#") and parts[0] == workload and parts[1] == kernel:
            return float(parts[2]), " ".join(parts[3:]) or None
    return None, None


def algorithmic_bytes(app: str, v_r: int, e_r: int) -> int:
    """Bytes a traversal must move: per edge, its destination (+ weight for
    SSSP) and one probe of the destination's state; per reached vertex, its
    row_start pair, result write and queue push and pop.  For BFS, e_r is
    the edges actually examined: all reached edges top-down, fewer when
    bottom-up levels stop at the first parent found."""
    return (12 if app == "sssp" else 8) * e_r + 20 * v_r


def sources_for(spec: dict, host_graph) -> list[int]:
    if spec["nsrc"] == 0:
        return [0]
    return host_graph.pick_sources(spec["src_seed"], spec["nsrc"])


def make_device_graph(gft, spec: dict, device: int):
    if spec["kind"] == "road":
        return gft.DeviceGraph.generate("road", device=device, seed=spec["seed"], side=spec["side"])
    if spec["kind"] == "rmat":
        return gft.DeviceGraph.generate("rmat", device=device, seed=spec["seed"], scale=spec["scale"],
                                        edge_factor=spec["edge_factor"])
    return gft.DeviceGraph.generate("grid", device=device, seed=spec["seed"], rows=spec["rows"], cols=spec["cols"])


def make_host_graph(gft, spec: dict):
    if spec["kind"] == "road":
        return gft.CSRGraph.road(spec["side"], seed=spec["seed"])
    if spec["kind"] == "rmat":
        return gft.CSRGraph.rmat(spec["scale"], spec["edge_factor"], seed=spec["seed"])
    return gft.CSRGraph.grid(spec["rows"], spec["cols"], spec["seed"], 1)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_queries(gft, eng, dg, spec, sources, out, stream, tune=None, delta=None, stats=None):
    app = spec["app"]
    kms = []
    for s in sources:
        if app == "sssp":
            r = eng.sssp(dg, s, delta=delta, out=out, stream=stream, tune=tune)
        else:
            r = eng.bfs(dg, s, out=out, stream=stream, tune=tune)
        kms.append(r["kernel_ms"])
        if stats is not None:
            stats.append({k: r[k] for k in ("levels", "iterations", "edges_scanned", "grid_blocks", "block_threads")})
    return kms


def bench_workload(gft, name: str, steps: int, warmup: int, d, dev: int, headline: bool):
    import torch

    spec = WORKLOADS[name]
    app = spec["app"]
    t0 = time.time()
    dg = make_device_graph(gft, spec, dev)
    host = dg.download()
    sources = sources_for(spec, host)
    log(f"[{name}] graph {dg.nnodes} nodes {dg.nedges} edges, {len(sources)} sources, setup {time.time() - t0:.1f}s")
    eng = gft.Engine(dev)
    stream = torch.cuda.current_stream(dev)
    out = torch.empty(dg.nnodes, dtype=torch.int32, device=f"cuda:{dev}")
    tune, delta, tune_desc = tuned_for(gft, name, spec)

    # Per-source reach statistics (E_r, V_r) from the first run of each source.
    reach = {}
    qstats = []
    scanned = {}
    for s in sources:
        run_queries(gft, eng, dg, spec, [s], out, stream, tune, delta, qstats)
        reach[s] = gft.reach_stats(dg, out, stream)
        scanned[s] = qstats[-1]["edges_scanned"]
    step_src = [sources[i % len(sources)] for i in range(max(steps, len(sources)))]
    timed_src = step_src[:steps] if len(sources) <= steps else sources
    k = len(timed_src)

    run_queries(gft, eng, dg, spec, [sources[i % len(sources)] for i in range(warmup)], out, stream, tune, delta)
    clocks = ClockSampler(gpu_id_for(dev), str(dev)) if headline and d.rank == 0 else None
    d.barrier()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    kms = run_queries(gft, eng, dg, spec, timed_src, out, stream, tune, delta)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    d.barrier()
    clk = clocks.stop() if clocks else None
    local_ms = ev0.elapsed_time(ev1)
    total_ms = d.max(local_ms)
    e_sum = sum(reach[s][1] for s in timed_src)
    v_sum = sum(reach[s][0] for s in timed_src)
    value = d.world * e_sum / (total_ms * 1e6)
    # Harmonic mean of per-query GTEPS (Graph500 convention), kernel time.
    per_q = [reach[s][1] / (km * 1e6) for s, km in zip(timed_src, kms)]
    hmean = len(per_q) / sum(1.0 / x for x in per_q)
    kernel_ms = statistics.mean(kms)

    # End to end through the C ABI host-buffer calls: every step sends its
    # source to the device and brings all nnodes results back to pinned host
    # memory inside the timed region.  `e2e` uses the many-query call, which
    # copies a query's results back while the next query runs;
    # `e2e.one_call` makes one synchronous single-query call per step.
    h_out = torch.empty(dg.nnodes, dtype=torch.int32, pin_memory=True).numpy()
    k_e2e = max(3, min(k, 10))
    e2e_src = [timed_src[i % len(timed_src)] for i in range(k_e2e)]
    h_rows = torch.empty((k_e2e, dg.nnodes), dtype=torch.int32, pin_memory=True).numpy()

    def one_call(s):
        if app == "sssp":
            eng.sssp_host(dg, s, h_out, delta=delta, tune=tune)
        else:
            eng.bfs_host(dg, s, h_out, tune=tune)

    def many_call(srcs):
        if app == "sssp":
            eng.sssp_host_many(dg, srcs, h_rows, delta=delta, tune=tune)
        else:
            eng.bfs_host_many(dg, srcs, h_rows, tune=tune)

    for s in e2e_src[:2]:
        one_call(s)
    many_call(e2e_src[:2])
    e2e_edges = sum(reach[s][1] for s in e2e_src)
    d.barrier()
    t1 = time.perf_counter()
    for s in e2e_src:
        one_call(s)
    e2e_one_s = d.max(time.perf_counter() - t1)
    d.barrier()
    t1 = time.perf_counter()
    many_call(e2e_src)
    e2e_s = d.max(time.perf_counter() - t1)
    e2e_value = d.world * e2e_edges / (e2e_s * 1e9)
    e2e_one_value = d.world * e2e_edges / (e2e_one_s * 1e9)

    peak, peak_kind = measured_peaks()
    e_alg = e_sum if app == "sssp" else sum(min(reach[s][1], scanned[s]) for s in timed_src)
    alg_bytes = algorithmic_bytes(app, v_sum, e_alg) / k
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    kname = f"{app}_persistent"
    if qstats and qstats[0]["grid_blocks"] == 1:
        # Small graphs run on one CTA: BFS on a uniform-degree graph of at
        # most 2^17 vertices takes the thread-per-vertex kernel.
        max_deg = int(np.diff(host.row_start.astype(np.int64)).max(initial=0))
        kname = ("sssp_single_cta" if app == "sssp" else
                 "bfs_cta_lanes" if dg.nnodes <= 1 << 17 and max_deg <= 32 else "bfs_single_cta")
        tune_desc = {"launch": "one CTA of 1024 threads (graphs of <= 2^17 vertices and <= 2^19 edges)",
                     "kernel": kname}
    traffic, traffic_src = profile_traffic(name, kname)
    res = {
        "name": name,
        "app": app,
        "nodes": dg.nnodes,
        "edges": dg.nedges,
        "sources": timed_src if len(timed_src) <= 4 else f"{len(set(timed_src))} seeded (seed {spec['src_seed']})",
        "k": k,
        "total_ms": total_ms,
        "value": value,
        "gteps_hmean_kernel": hmean,
        # Graph500 convention for symmetric graphs (every generated graph
        # here): each undirected edge counted once, E_r / 2.
        "gteps_graph500": value / 2,
        "kernel_ms_mean": kernel_ms,
        "e_r_per_query": e_sum / k,
        "v_r_per_query": v_sum / k,
        "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": 4, "d2h_bytes_per_step": dg.nnodes * 4,
                "steps": k_e2e, "call": f"gft_{app}_host_many (copy back overlaps the next query)",
                "one_call": {"value": e2e_one_value, "call": f"gft_{app}_host, one synchronous call per step"}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "alg_bytes_per_launch": alg_bytes,
                     "kernel": kname, "traffic_source": traffic_src},
        "clocks": clk,
        "graph_bytes": (dg.nnodes + 1) * 4 + dg.nedges * (8 if dg.weighted else 4),
        "weighted": bool(dg.weighted),
        "tuning": tune_desc,
        "tune": tune,
        "delta": delta,
        "query_stats": qstats[:4],
        "host": host,
        "out_last": out,
        "timed_src": timed_src,
        "kms": kms,
        "reach": reach,
    }
    eng.close()
    return res, dg


def cpu_baseline(orc, spec, host, src, reach, gpu_out=None) -> dict:
    """The oracle's query on one host core.  A query of under 0.1 s is
    repeated for about a second and its median taken, so that a
    sub-millisecond baseline is not one noisy sample."""
    def run():
        if spec["app"] == "sssp":
            return orc.sssp(host.row_start, host.edge_dst, host.edge_data, src)
        return orc.bfs(host.row_start, host.edge_dst, src)

    t = time.perf_counter()
    ref = run()
    dt = time.perf_counter() - t
    times = [dt]
    if dt < 0.1:
        t_end = time.perf_counter() + 1.0
        while time.perf_counter() < t_end and len(times) < 5000:
            t = time.perf_counter()
            run()
            times.append(time.perf_counter() - t)
        dt = statistics.median(times[1:])
    e_r = reach[src][1]
    algo = "binary-heap Dijkstra" if spec["app"] == "sssp" else "FIFO BFS"
    sample = (f"one full {spec['app'].upper()} query from source {src} ({algo}, {dt:.1f} s)" if len(times) == 1 else
              f"the median of {len(times) - 1} full {spec['app'].upper()} queries from source {src} ({algo}, "
              f"{dt * 1e3:.3f} ms each; min {min(times[1:]) * 1e3:.3f} ms)")
    res = {"value": e_r / dt / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port", "sample": sample}
    parity = None
    if gpu_out is not None:
        parity = "bit-exact" if np.array_equal(ref, gpu_out) else "MISMATCH"
    return res, parity


def our_arm(args) -> int:
    import torch

    import galoisgpu_b200 as gft

    from galoisgpu_b200.replicas import ReplicaGroup

    d = ReplicaGroup()
    dev = d.local if d.world > 1 else 0
    torch.cuda.set_device(dev)
    name = args.workload
    spec = WORKLOADS[name]
    res, dg = bench_workload(gft, name, args.steps, args.warmup, d, dev, headline=True)

    line = {
        "metric": "GTEPS per query",
        "value": res["value"],
        "unit": "GTEPS",
        "n_gpus": d.world,
        "steps": res["k"],
        "warmup": args.warmup,
        "ms_per_step": res["total_ms"] / res["k"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic: seeded graph generated on the device (SplitMix64 streams), same graph on every rank",
        "config": workload_config(name, spec, res["nodes"], res["edges"], res["weighted"], res["timed_src"],
                                  res["e_r_per_query"], res["v_r_per_query"], d.world),
        "detail": {
            "kernel_ms_mean": res["kernel_ms_mean"],
            "gteps_hmean_kernel": res["gteps_hmean_kernel"],
            "gteps_graph500": res["gteps_graph500"],
            **({"delta": res["delta"]} if spec["app"] == "sssp" else {}),
            "tuning": res["tuning"] or "engine defaults",
            "query_stats": res["query_stats"],
        },
        "e2e": res["e2e"],
        "gpu_launches": res["k"],
        "roofline": res["roofline"],
        "clocks": res["clocks"],
    }
    if d.rank == 0 and d.world == 1:
        from oracle import oracle as orc

        src = res["timed_src"][0]
        gpu_ref = None
        # Recompute the first source on the GPU for the parity check.
        eng = gft.Engine(dev)
        out = (eng.sssp(dg, src, delta=spec["delta"]) if spec["app"] == "sssp" else eng.bfs(dg, src))["out"]
        gpu_ref = out.cpu().numpy()
        eng.close()
        cb, parity = cpu_baseline(orc, spec, res["host"], src, res["reach"], gpu_ref)
        line["cpu_baseline"] = cb
        line["parity"] = {"vs_oracle": parity, "source": src}
        # The reference's own CUDA build on the same graph and source, in this run.
        ref_blocks = {}
        if not args.no_reference_build:
            try:
                ref_blocks[name] = reference_build_block(
                    gft, name, spec, res["host"], dg, dev, [src], res["delta"], _kms_by_source(res), res["reach"],
                    repeat=5, our_e2e_gteps=res["e2e"]["value"], tune=res["tune"])
            except Exception as ex:
                ref_blocks[name] = {"error": repr(ex)}
            line["parity"]["vs_reference_build"] = ref_blocks[name].get("parity_vs_reference_build")
            line["parity"]["sources_checked"] = {name: ref_blocks[name].get("sources_checked", 0)}
        if not args.no_secondary:
            sec = {}
            for sname in ("bfs-rmat-24", "bfs-grid-256"):
                if sname == name:
                    continue
                try:
                    dg.free()
                    torch.cuda.empty_cache()
                    r2, dg2 = bench_workload(gft, sname, 64 if sname == "bfs-rmat-24" else args.steps, 3, d, dev,
                                             headline=False)
                    s2 = r2["timed_src"][0]
                    spec2 = WORKLOADS[sname]
                    cb2, par2 = cpu_baseline(orc, spec2, r2["host"], s2, r2["reach"],
                                             _rerun(gft, dg2, spec2, s2, dev))
                    sec[sname] = {
                        "tuning": r2["tuning"], "query_stats": r2["query_stats"][:2],
                        "value": r2["value"], "unit": "GTEPS", "gteps_hmean_kernel": r2["gteps_hmean_kernel"],
                        "gteps_graph500": r2["gteps_graph500"],
                        "kernel_ms_mean": r2["kernel_ms_mean"], "queries": r2["k"], "nodes": r2["nodes"],
                        "edges": r2["edges"], "E_r_per_query": r2["e_r_per_query"], "e2e": r2["e2e"],
                        "roofline": r2["roofline"], "cpu_baseline": cb2, "parity_vs_oracle": par2,
                    }
                    srcs2 = sorted(set(r2["timed_src"]), key=r2["timed_src"].index)
                    if len(srcs2) > 1:
                        # Every timed source against the CPU oracle, on all host threads.
                        sec[sname]["parity_vs_oracle_all_sources"] = oracle_parity_many(
                            orc, spec2, r2["host"], _digests(gft, dg2, spec2, srcs2, dev, r2["tune"]),
                            max(1, min(16, _cores())))
                    if sname == "bfs-rmat-24":
                        try:
                            sec["ingest-rmat-24"] = bench_ingest(gft, sname, r2["host"], dev)
                        except Exception as ex:
                            sec["ingest-rmat-24"] = {"error": repr(ex)}
                    if not args.no_reference_build:
                        try:
                            ref_blocks[sname] = reference_build_block(
                                gft, sname, spec2, r2["host"], dg2, dev, srcs2[:16], None, _kms_by_source(r2),
                                r2["reach"], repeat=2 if len(srcs2) > 1 else 5,
                                our_e2e_gteps=r2["e2e"]["value"], tune=r2["tune"])
                        except Exception as ex:
                            ref_blocks[sname] = {"error": repr(ex)}
                        line["parity"]["sources_checked"][sname] = ref_blocks[sname].get("sources_checked", 0)
                    dg2.free()
                except Exception as ex:  # keep the headline line even if a secondary fails
                    sec[sname] = {"error": repr(ex)}
            try:
                torch.cuda.empty_cache()
                sec["batch-sssp-512"] = bench_batch(gft, dev)
            except Exception as ex:
                sec["batch-sssp-512"] = {"error": repr(ex)}
            try:
                torch.cuda.empty_cache()
                sec["msbfs-rmat24-256"] = bench_msbfs(gft, dev)
            except Exception as ex:
                sec["msbfs-rmat24-256"] = {"error": repr(ex)}
            try:
                torch.cuda.empty_cache()
                sec["serve-8-graphs"] = bench_serve(gft, dev)
            except Exception as ex:
                sec["serve-8-graphs"] = {"error": repr(ex)}
            for mname in MIS_WORKLOADS:
                try:
                    torch.cuda.empty_cache()
                    sec[mname] = bench_mis(gft, orc, mname, dev)
                except Exception as ex:
                    sec[mname] = {"error": repr(ex)}
            for pname in PR_SECONDARY:
                try:
                    torch.cuda.empty_cache()
                    sec[pname] = bench_pr(gft, orc, pname, dev)
                except Exception as ex:
                    sec[pname] = {"error": repr(ex)}
            for cname in CC_WORKLOADS:
                try:
                    torch.cuda.empty_cache()
                    sec[cname] = bench_cc(gft, orc, cname, dev)
                except Exception as ex:
                    sec[cname] = {"error": repr(ex)}
            line["secondary"] = sec
        if ref_blocks:
            line["reference_cuda"] = ref_blocks
    if d.rank == 0:
        print(json.dumps(line), flush=True)
    d.barrier()
    d.close()
    return 0


CC_WORKLOADS = {
    "cc-rmat-24": dict(kind="rmat", scale=24, edge_factor=16, seed=1),
    "cc-road-4096": dict(kind="road", side=4096, seed=1),
}


def bench_cc(gft, orc, name: str, dev: int, steps: int = 10, warmup: int = 3) -> dict:
    """Connected components (apps/cc on this engine) on a full-size seeded
    graph: GTEPS = all E directed edges / kernel time, end to end with the
    labels copied to pinned host memory, the oracle's union-find on one core
    of the host as CPU baseline, and bit-exact parity of the labels."""
    import torch

    spec = {**CC_WORKLOADS[name], "app": "cc"}
    dg = make_device_graph(gft, spec, dev)
    host = dg.download()
    eng = gft.Engine(dev)
    out = torch.empty(dg.nnodes, dtype=torch.int32, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        r = eng.cc(dg, out=out, stream=stream)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    kms = []
    for _ in range(steps):
        r = eng.cc(dg, out=out, stream=stream)
        kms.append(r["kernel_ms"])
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    total_ms = ev0.elapsed_time(ev1)
    kernel_ms = statistics.mean(kms)
    h_out = torch.empty(dg.nnodes, dtype=torch.int32, pin_memory=True).numpy()
    eng.cc_host(dg, h_out)
    t1 = time.perf_counter()
    for _ in range(steps):
        eng.cc_host(dg, h_out)
    e2e_s = (time.perf_counter() - t1) / steps
    t2 = time.perf_counter()
    want, comps = orc.cc(host.row_start, host.edge_dst)
    cpu_s = time.perf_counter() - t2
    peak, peak_kind = measured_peaks()
    # Bytes a union-find pass must move: each directed edge's destination
    # (4 B), two label reads per joined edge (8 B), and per vertex its
    # row_start pair, the initial label, and the final read and write (16 B).
    alg = 4 * dg.nedges + 8 * r["edges_scanned"] + 16 * dg.nnodes
    res = {
        "metric": "GTEPS (all edges)", "value": dg.nedges / (total_ms / steps * 1e6), "unit": "GTEPS",
        "kernel_ms_mean": kernel_ms, "steps": steps, "warmup": warmup, "nodes": dg.nnodes, "edges": dg.nedges,
        "edges_joined": r["edges_scanned"], "components": r["components"],
        "e2e": {"value": dg.nedges / (e2e_s * 1e9), "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": dg.nnodes * 4},
        "roofline": {"bound": "hbm", "achieved": alg / (kernel_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (kernel_ms * 1e-3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg, "kernel": "cc_hook"},
        "cpu_baseline": {"value": dg.nedges / cpu_s / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
                         "sample": f"one union-find pass over all edges ({cpu_s:.1f} s)"},
        "parity_vs_oracle": "bit-exact" if np.array_equal(h_out, want) and comps == r["components"] else "MISMATCH",
    }
    log(f"[{name}] {res['value']:.1f} GTEPS, kernel {kernel_ms:.3f} ms, {r['components']} components, "
        f"parity {res['parity_vs_oracle']}")
    eng.close()
    dg.free()
    return res


MIS_WORKLOADS = {
    "mis-rmat-24": dict(kind="rmat", scale=24, edge_factor=16, seed=1),
    "mis-road-4096": dict(kind="road", side=4096, seed=1),
}


def bench_mis(gft, orc, name: str, dev: int, steps: int = 10, warmup: int = 3) -> dict:
    """Maximal independent set (apps/mis on this engine) on a full-size seeded
    graph with the reference's priorities on this device: GTEPS = all E
    directed edges / kernel time, end to end with the states copied to
    pinned host memory, the oracle's rounds on one host core as CPU
    baseline, and bit-exact parity of the set and the round count."""
    import torch

    spec = {**MIS_WORKLOADS[name], "app": "mis"}
    dg = make_device_graph(gft, spec, dev)
    host = dg.download()
    eng = gft.Engine(dev)
    out = torch.empty(dg.nnodes, dtype=torch.int32, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        r = eng.mis(dg, out=out, stream=stream)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    kms = []
    for _ in range(steps):
        r = eng.mis(dg, out=out, stream=stream)
        kms.append(r["kernel_ms"])
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    total_ms = ev0.elapsed_time(ev1)
    kernel_ms = statistics.mean(kms)
    h_out = torch.empty(dg.nnodes, dtype=torch.int32, pin_memory=True).numpy()
    eng.mis_host(dg, h_out)
    t1 = time.perf_counter()
    for _ in range(steps):
        eng.mis_host(dg, h_out)
    e2e_s = (time.perf_counter() - t1) / steps
    prio_threads = 8 * torch.cuda.get_device_properties(dev).multi_processor_count * 256
    t2 = time.perf_counter()
    want, want_steps = orc.mis(host.row_start, host.edge_dst, prio_threads)
    cpu_s = time.perf_counter() - t2
    peak, peak_kind = measured_peaks()
    # Bytes the rounds must move: per neighbour tested its id and packed
    # word (12 B); per worklist entry and pass the entry, the vertex's own
    # word and its row pair (20 B, two passes); per vertex the priority
    # word and worklist entry written at the start and the word read and
    # state written at the end (24 B).
    alg = 12 * r["edges_scanned"] + 40 * r["pushes"] + 24 * dg.nnodes
    res = {
        "metric": "GTEPS (all edges)", "value": dg.nedges / (total_ms / steps * 1e6), "unit": "GTEPS",
        "kernel_ms_mean": kernel_ms, "steps": steps, "warmup": warmup, "nodes": dg.nnodes, "edges": dg.nedges,
        "rounds": r["levels"], "set_size": r["vertices_reached"], "neighbours_tested": r["edges_scanned"],
        "worklist_entries": r["pushes"], "prio_threads": prio_threads,
        "e2e": {"value": dg.nedges / (e2e_s * 1e9), "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": dg.nnodes * 4},
        "roofline": {"bound": "hbm", "achieved": alg / (kernel_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (kernel_ms * 1e-3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg, "kernel": "mis_persistent"},
        "cpu_baseline": {"value": dg.nedges / cpu_s / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
                         "sample": f"the oracle's full MIS ({want_steps} rounds, {cpu_s:.1f} s)"},
        "parity_vs_oracle": "bit-exact" if np.array_equal(h_out, want) and want_steps == r["levels"] else "MISMATCH",
    }
    log(f"[{name}] {res['value']:.1f} GTEPS, kernel {kernel_ms:.3f} ms, {r['levels']} rounds, "
        f"set {r['vertices_reached']}, parity {res['parity_vs_oracle']}")
    eng.close()
    dg.free()
    return res


PR_WORKLOADS = {
    "pr-rmat-24": dict(kind="rmat", scale=24, edge_factor=16, seed=1),
    "pr-road-4096": dict(kind="road", side=4096, seed=1),
    "pr-rmat-20": dict(kind="rmat", scale=20, edge_factor=16, seed=1),  # profiling case
}
PR_SECONDARY = ("pr-rmat-24", "pr-road-4096")


def bench_pr(gft, orc, name: str, dev: int, steps: int = 5, warmup: int = 3, cpu_seconds: float = 10.0) -> dict:
    """PageRank by residual push (apps/pr on this engine) to convergence on a
    full-size seeded graph: GTEPS = edges pushed / kernel time, end to end
    with the ranks copied to pinned host memory, and the oracle on one host
    core, capped at the iterations that fit in about cpu_seconds (its
    per-edge rate is the CPU baseline; the ranks are checked against the
    oracle in the tests, at sizes the oracle finishes in seconds)."""
    import torch

    spec = {**PR_WORKLOADS[name], "app": "pr"}
    dg = make_device_graph(gft, spec, dev)
    eng = gft.Engine(dev)
    out = torch.empty(dg.nnodes, dtype=torch.float32, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        r = eng.pr(dg, out=out, stream=stream)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    runs = [eng.pr(dg, out=out, stream=stream) for _ in range(steps)]
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    total_ms = ev0.elapsed_time(ev1) / steps
    kernel_ms = statistics.mean(x["kernel_ms"] for x in runs)
    pushed = statistics.mean(x["edges_scanned"] for x in runs)
    h_out = torch.empty(dg.nnodes, dtype=torch.float32, pin_memory=True).numpy()
    t1 = time.perf_counter()
    for _ in range(steps):
        eng.pr_host(dg, h_out)
    e2e_s = (time.perf_counter() - t1) / steps
    host = dg.download()
    cpu = {}
    iters = 1
    while True:  # grow the capped oracle run until it takes about cpu_seconds
        t2 = time.perf_counter()
        orc.pr(host.row_start, host.edge_dst, max_iterations=iters, stats=cpu)
        dt = time.perf_counter() - t2
        if dt * 2 > cpu_seconds or iters >= runs[0]["levels"]:
            break
        iters *= 2
    peak, peak_kind = measured_peaks()
    pops = statistics.mean(x["pushes"] for x in runs)
    # Bytes a push step must move per edge pushed: its destination (4 B), the
    # residual read-modify-write (8 B); per worklist entry popped: the entry,
    # the residual exchange, the rank update and the row pair (20 B).
    alg = 12 * pushed + 20 * pops
    res = {
        "metric": "GTEPS (edges pushed)", "value": pushed / (total_ms * 1e6), "unit": "GTEPS",
        "kernel_ms_mean": kernel_ms, "iterations": runs[0]["levels"], "edges_pushed": pushed, "pops": pops,
        "steps": steps,
        "warmup": warmup, "nodes": dg.nnodes, "edges": dg.nedges,
        "e2e": {"value": pushed / (e2e_s * 1e9), "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": dg.nnodes * 4},
        "roofline": {"bound": "hbm", "achieved": alg / (kernel_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (kernel_ms * 1e-3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg, "kernel": "pr_persistent"},
        "cpu_baseline": {"value": cpu["edges_pushed"] / dt / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
                         "sample": f"the oracle's first {iters} iterations ({cpu['edges_pushed']} edges pushed, "
                                   f"{dt:.1f} s)"},
    }
    log(f"[{name}] {res['value']:.1f} GTEPS, kernel {kernel_ms:.3f} ms, {runs[0]['levels']} iterations")
    eng.close()
    dg.free()
    return res


def _pct(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, max(0, math.ceil(q * len(xs)) - 1))]


def bench_batch(gft, dev: int, n_queries: int = 512, reps: int = 3, delta: int = 40000) -> dict:
    """C4: n SSSP queries over n seeded graphs (log-uniform sizes, half road,
    half R-MAT) in one persistent launch replayed as a CUDA graph, against
    the same queries launched one at a time on the same engine."""
    import torch

    from galoisgpu_b200 import workloads as wl

    specs = wl.batch_specs(n_queries)
    t0 = time.time()
    graphs = [wl.build(sp, dev) for sp in specs]
    srcs = [g.pick_sources(sp["seed"], 1)[0] for g, sp in zip(graphs, specs)]
    setup_s = time.time() - t0
    eng = gft.Engine(dev)
    stream = torch.cuda.current_stream(dev)
    queries = [{"graph": g, "app": "sssp", "src": s, "delta": delta} for g, s in zip(graphs, srcs)]
    # Batch launch shapes tried (CTA size, CTAs per large query, size from
    # which a query gets a CTA group); the fastest is reported.
    shapes = [(512, 8, 1 << 18), (512, 16, 1 << 18), (256, 16, 1 << 17), (256, 32, 1 << 18), (512, 1, 1 << 30)]
    tried = []
    best = None
    for blk, grp, gmin in shapes:
        b = gft.Batch(eng, queries, tune=gft.Tune(block_threads=blk, group_blocks=grp, group_min_nodes=gmin))
        st = b.run(stream)  # warm-up; every query must succeed
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        for _ in range(reps):
            b.submit(stream)
        ev1.record(stream)
        st = b.wait()
        ms = ev0.elapsed_time(ev1) / reps
        tried.append({"block_threads": blk, "group_blocks": grp, "group_min_nodes": gmin, "ms": ms})
        log(f"[batch] block {blk} group {grp} min {gmin}: {ms:.1f} ms")
        if best is None or ms < best[0]:
            if best is not None:
                best[1].close()
            best = (ms, b, st, tried[-1])
        else:
            b.close()
    batch_ms, b, st, shape = best
    edges = sum(q["edges_scanned"] for q in b.queries)
    # One query at a time through the same engine (grid-wide kernel per query).
    out = torch.empty(max(g.nnodes for g in graphs), dtype=torch.int32, device=f"cuda:{dev}")
    mismatches = 0
    single_ms = []
    for q in queries:
        g = q["graph"]
        o = out[: g.nnodes]
        r = eng.sssp(g, q["src"], delta=delta, out=o)
        single_ms.append(r["kernel_ms"])
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    cum = []
    for i, q in enumerate(queries):
        g = q["graph"]
        o = out[: g.nnodes]
        eng.sssp(g, q["src"], delta=delta, out=o)
        cum.append((time.perf_counter() - t1) * 1e3)
        if not torch.equal(o, b.queries[i]["out"]):
            mismatches += 1
    single_total_s = time.perf_counter() - t1
    b.close()
    eng.close()
    res = {
        "queries": n_queries,
        "graphs": {"nodes_min": min(sp["nodes"] for sp in specs), "nodes_max": max(sp["nodes"] for sp in specs),
                   "nodes_total": sum(g.nnodes for g in graphs), "edges_total": sum(g.nedges for g in graphs),
                   "setup_s": setup_s},
        "delta": delta,
        "batch": {"ms_per_launch": batch_ms, "queries_per_s": n_queries / (batch_ms * 1e-3),
                  "p50_ms": batch_ms, "p99_ms": batch_ms, "busy_ms": st["busy_ms"],
                  "grid": f"{st['grid_blocks']} x {st['block_threads']}", "scratch_bytes": st["scratch_bytes"],
                  "edges_scanned": edges, "cuda_graph_replay": True, "shape": shape, "shapes_tried": tried},
        "one_at_a_time": {"total_s": single_total_s, "queries_per_s": n_queries / single_total_s,
                          "p50_ms": _pct(cum, 0.5), "p99_ms": _pct(cum, 0.99),
                          "kernel_ms_sum": sum(single_ms)},
        "parity_batch_vs_single": "bit-exact" if mismatches == 0 else f"{mismatches} MISMATCHES",
        "note": "closed batch submitted at t=0: a query's latency is its completion time, so a batch's p50 = p99 = "
                "its launch time and one-at-a-time p50/p99 are cumulative completion times",
    }
    res["speedup_qps"] = res["batch"]["queries_per_s"] / res["one_at_a_time"]["queries_per_s"]
    for g in graphs:
        g.free()
    return res


def bench_msbfs(gft, dev: int, k: int = 256, reps: int = 3, max_levels: int = 16) -> dict:
    """256-source BFS on RMAT-24 in one launch (bitset multi-source BFS,
    direction-optimising per level), against the same 256 queries as
    single-source launches of the same engine."""
    import torch

    spec = WORKLOADS["bfs-rmat-24"]
    dg = make_device_graph(gft, spec, dev)
    srcs = dg.pick_sources(spec["src_seed"], k)
    eng = gft.Engine(dev)
    tune, _, tune_desc = tuned_for(gft, "bfs-rmat-24", spec)
    plane_bytes = gft.load().gft_msbfs_plane_bytes(dg.nnodes, k)
    planes = torch.empty(max_levels * plane_bytes // 4, dtype=torch.int32, device=f"cuda:{dev}")
    r = eng.msbfs(dg, srcs, max_levels=max_levels, symmetric=True, planes=planes)  # warm-up
    ms = []
    for _ in range(reps):
        r = eng.msbfs(dg, srcs, max_levels=max_levels, symmetric=True, planes=planes)
        ms.append(r["kernel_ms"])
    t_ms = statistics.median(ms)
    # Single-source queries of the same engine, and parity on a sample.
    out = torch.empty(dg.nnodes, dtype=torch.int32, device=f"cuda:{dev}")
    e_r_total, single_ms, mismatches = 0, [], 0
    check = set(range(0, k, 17)) | {k - 1}
    for i, s in enumerate(srcs):
        rr = eng.bfs(dg, s, out=out, tune=tune)
        single_ms.append(rr["kernel_ms"])
        e_r_total += gft.reach_stats(dg, out)[1]
        if i in check and not torch.equal(r["levels_of"](i), out):
            mismatches += 1
    eng.close()
    del planes
    dg.free()
    return {
        "sources": k,
        "levels": r["levels"],
        "msbfs_ms": t_ms,
        "queries_per_s": k / (t_ms * 1e-3),
        "gteps_aggregate": e_r_total / (t_ms * 1e6),
        "one_at_a_time": {"ms_total": sum(single_ms), "queries_per_s": k / (sum(single_ms) * 1e-3),
                          "tuning": tune_desc},
        "speedup_qps": sum(single_ms) / t_ms,
        "parity_vs_single": "bit-exact" if mismatches == 0 else f"{mismatches} MISMATCHES",
        "parity_sources_checked": len(check),
        "note": "kernel time of one msbfs launch (bitsets, top-down/bottom-up per level) vs the sum of 256 "
                "single-query kernel times",
    }


def bench_serve(gft, dev: int, rates=(200, 500, 1000, 3000, 10000, 50000),
                p99_targets=(10.0, 20.0, 50.0, 100.0, 200.0, 500.0), delta: int = 40000) -> dict:
    """C5: Poisson BFS/SSSP requests with random non-isolated sources over
    resident graphs, at offered rates from 200 to 50,000 requests/s, against
    - the resident serving kernel (one persistent launch; requests through a
      mapped ring; teams of lanes drafted on the device, gft_serve resident=1),
    - the lane server (one launch per lane micro-batch, resident=0), and
    - the same engine serving one request at a time with the whole GPU
      (max_batch 1, one lane, one group of every resident CTA).
    Three mixes: the configured one (50/50 BFS/SSSP over the 8 graphs), a
    BFS-only one over the same graphs, and 50/50 over the three smallest
    graphs (road 1024^2, RMAT-18, RMAT-20).  Each sweep offers every rate
    (arrivals wait for a free output buffer and are counted as throttled);
    for each p99 target the result gives the best throughput each server
    sustained within it."""
    import torch

    from galoisgpu_b200 import workloads as wl
    from galoisgpu_b200.serve import Server, poisson_run

    specs = wl.serving_specs()
    t0 = time.time()
    graphs = [wl.build(sp, dev) for sp in specs]
    sources = [g.pick_sources(7 + i, 256) for i, g in enumerate(graphs)]
    # Output buffers: each in-flight request owns one; about 1.5 GB per graph.
    pools = [[torch.empty(g.nnodes, dtype=torch.int32, device=f"cuda:{dev}")
              for _ in range(max(4, min(256, int(1.5e9 // (4 * g.nnodes)))))] for g in graphs]
    torch.cuda.synchronize(dev)
    setup_s = time.time() - t0
    eng = gft.Engine(dev)
    small = [i for i, sp in enumerate(specs) if sp["nodes"] <= 1 << 20]

    def sweep(srv, tag, idx, bfs_fraction):
        out = []
        for r in rates:
            n = int(min(1500, max(300, r * 0.5)))
            res = poisson_run(srv, [graphs[i] for i in idx], [sources[i] for i in idx], [pools[i] for i in idx],
                              rate=r, n_requests=n, seed=7, delta=delta, bfs_fraction=bfs_fraction)
            out.append(res)
            log(f"[{tag}] rate {r}: {res['achieved_qps']:.0f} q/s p50 {res['p50_ms']:.2f} ms "
                f"p99 {res['p99_ms']:.2f} ms width {res['mean_width']:.1f} throttled {res['throttled_arrivals']}")
        return out

    def best_under(rs, p99):
        ok = [x["achieved_qps"] for x in rs if x["p99_ms"] is not None and x["p99_ms"] <= p99 and x["failures"] == 0]
        return max(ok) if ok else 0.0

    servers = {
        "resident": dict(resident=1, lane_blocks=8, lane_arena_bytes=1600 << 20),
        "lanes": {},
        "one_at_a_time": dict(lanes=1, max_batch=1, group_min_nodes=1, group_blocks=10**6),
    }
    mixes = {
        "mix": (list(range(len(specs))), 0.5, ("resident", "lanes", "one_at_a_time")),
        "bfs_only": (list(range(len(specs))), 1.0, ("resident", "one_at_a_time")),
        "small_graphs": (small, 0.5, ("resident", "one_at_a_time")),
    }
    result = {"graphs": [wl.name(sp) for sp in specs], "nodes_total": sum(sp["nodes"] for sp in specs),
              "setup_s": setup_s, "delta": delta, "offered_rates": list(rates)}
    for mname, (idx, bfs_fraction, names) in mixes.items():
        runs = {}
        for sname in names:
            srv = Server(eng, **servers[sname])
            runs[sname] = sweep(srv, f"{mname} {sname}", idx, bfs_fraction)
            srv.close()
        equal = []
        for t in p99_targets:
            base = best_under(runs["one_at_a_time"], t)
            row = {"p99_ms": t, "one_at_a_time_qps": base}
            for sname in names:
                if sname != "one_at_a_time":
                    q = best_under(runs[sname], t)
                    row[f"{sname}_qps"] = q
                    row[f"{sname}_speedup"] = (q / base) if base else None
            equal.append(row)
        result[mname] = {
            "graphs": [wl.name(specs[i]) for i in idx], "bfs_fraction": bfs_fraction, "runs": runs,
            "at_equal_p99": equal,
            "peak_qps": {k: max(x["achieved_qps"] for x in v) for k, v in runs.items()},
        }
        log(f"[{mname}] peak q/s " + ", ".join(f"{k} {v:.0f}" for k, v in result[mname]["peak_qps"].items()))
    eng.close()
    del pools
    for g in graphs:
        g.free()
    return result


def _kms_by_source(res) -> dict:
    """Median kernel time of each timed source of a bench_workload result."""
    by: dict = {}
    for s, km in zip(res["timed_src"], res["kms"]):
        by.setdefault(s, []).append(km)
    return {s: statistics.median(v) for s, v in by.items()}


def _cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _digests(gft, dg, spec, sources, dev, tune=None) -> dict:
    """sha256 of this engine's result for every source."""
    import hashlib

    import torch

    eng = gft.Engine(dev)
    out = torch.empty(dg.nnodes, dtype=torch.int32, device=f"cuda:{dev}")
    dig = {}
    for s in sources:
        if spec["app"] == "sssp":
            eng.sssp(dg, s, delta=spec["delta"], out=out, tune=tune)
        else:
            eng.bfs(dg, s, out=out, tune=tune)
        dig[s] = hashlib.sha256(out.cpu().numpy().tobytes()).hexdigest()
    eng.close()
    return dig


def _rerun(gft, dg, spec, src, dev):
    eng = gft.Engine(dev)
    out = (eng.sssp(dg, src, delta=spec["delta"]) if spec["app"] == "sssp" else eng.bfs(dg, src))["out"]
    eng.close()
    return out.cpu().numpy()


# ---------------------------------------------------------------------------
# the reference's own CUDA build (oracle/_ref, compiled for sm_100a from the
# reference sources by oracle/ref/Makefile)
# ---------------------------------------------------------------------------
REF_BUILD = ROOT / "oracle" / "_ref"
_REF_QUERY = re.compile(r"oracle-ref-query source (\d+) total_ns (\d+) kernel_ms ([0-9.]+)")


def run_reference_build(app: str, gr_path, sources, delta=None, repeat: int = 1, dump_dir=None,
                        timeout: float = 1200.0):
    """Runs the reference's BFS or SSSP (its gg_main, kernels and worklists,
    apps/bfs/kernel.cu:380-393, apps/sssp/kernel.cu:455-480) once per source
    and repetition in one process (oracle/_ref/{bfs,sssp}_multi, see
    oracle/ref/multi_driver.cu), the way skel.cu runs one query: the graph
    read by the reference's own reader, `-d delta` for SSSP.  Returns one
    dict per call in call order: source, total_ns (the reference's timer
    around gg_main, skelapp/skel.cu:55-66, worklist allocations included)
    and kernel_ms (CUDA events around every kernel the call launched)."""
    exe = REF_BUILD / f"{app}_multi"
    if not exe.exists():
        raise FileNotFoundError(f"{exe} is not built (make -C oracle/ref)")
    env = dict(os.environ, GFT_REF_SOURCES=",".join(str(int(x)) for x in sources), GFT_REF_REPEAT=str(repeat))
    if dump_dir is not None:
        env["GFT_REF_DUMP"] = str(dump_dir)
    cmd = [str(exe), "-q", "-s", str(int(sources[0]))]
    if app == "sssp":
        cmd += ["-d", str(int(delta))]
    cmd.append(str(gr_path))
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{exe.name} exited {r.returncode}: {r.stderr[-1500:]}")
    calls = [{"source": int(m[1]), "total_ns": int(m[2]), "kernel_ms": float(m[3])}
             for m in _REF_QUERY.finditer(r.stderr)]
    if len(calls) != len(sources) * repeat:
        raise RuntimeError(f"{exe.name}: {len(calls)} query lines for {len(sources) * repeat} calls")
    return calls


def _hmean(xs):
    return len(xs) / sum(1.0 / x for x in xs) if xs else None


def reference_build_block(gft, name: str, spec: dict, host, dg, dev: int, sources, our_delta, our_kms: dict,
                          reach: dict, repeat: int, our_e2e_gteps=None, tune=None) -> dict:
    """The reference's own sm_100a build on the same graph (written as .gr
    and read by the reference's reader) and the same sources, in this run:
    its kernel-only and `Total time`, GTEPS from the same E_r, the ratio to
    this engine, and bit-exact parity of every query's result (its
    node_data against this engine's output for the same source).  The
    reference runs SSSP with its default delta (10000, apps/sssp/support.cu:10);
    distances do not depend on delta.  Calls of
    the first repetition are cold (the process's first gg_main also sets up
    the drivers' barriers), so with repeat > 1 the times are the later
    repetitions'."""
    app = spec["app"]
    tmp = Path(tempfile.mkdtemp(prefix="gft_refbuild_"))
    try:
        gr = tmp / f"{name}.gr"
        host.write(gr)
        dump = tmp / "dump"
        dump.mkdir()
        t = time.time()
        calls = run_reference_build(app, gr, sources, delta=spec.get("delta"), repeat=repeat, dump_dir=dump)
        wall = time.time() - t
        warm = calls[len(sources):] if repeat > 1 else calls
        eng = gft.Engine(dev)
        mismatches = []
        import torch

        out = torch.empty(dg.nnodes, dtype=torch.int32, device=f"cuda:{dev}")
        for s in sources:
            if app == "sssp":
                eng.sssp(dg, s, delta=our_delta, out=out, tune=tune)
            else:
                eng.bfs(dg, s, out=out, tune=tune)
            ref = np.fromfile(dump / f"{s}.i32", dtype=np.int32)
            if ref.shape[0] != dg.nnodes or not np.array_equal(ref, out.cpu().numpy()):
                mismatches.append(int(s))
        eng.close()
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    by_src: dict = {}
    for c in warm:
        by_src.setdefault(c["source"], []).append(c)
    ref_k = {s: statistics.median(x["kernel_ms"] for x in cs) for s, cs in by_src.items()}
    ref_t = {s: statistics.median(x["total_ns"] for x in cs) / 1e6 for s, cs in by_src.items()}
    e_r = {s: reach[s][1] for s in sources}
    ref_gteps = _hmean([e_r[s] / (ref_k[s] * 1e6) for s in sources])
    ref_total_gteps = _hmean([e_r[s] / (ref_t[s] * 1e6) for s in sources])
    ours = _hmean([e_r[s] / (our_kms[s] * 1e6) for s in sources if s in our_kms])
    res = {
        "binary": f"oracle/_ref/{app}_multi (the reference's gg_main, kernels and worklists, compiled for sm_100a)",
        "sources": len(sources),
        "calls": len(calls),
        "kernel_ms_mean": statistics.mean(ref_k.values()),
        "total_ms_mean": statistics.mean(ref_t.values()),
        "gteps_kernel": ref_gteps,
        "gteps_total_time": ref_total_gteps,
        "this_engine_gteps_kernel": ours,
        "speedup_kernel": (ours / ref_gteps) if ours and ref_gteps else None,
        "parity_vs_reference_build": "bit-exact" if not mismatches else f"{len(mismatches)} MISMATCHES {mismatches[:8]}",
        "sources_checked": len(sources),
        "process_wall_s": wall,
        "note": "kernel_ms: CUDA events around every kernel of a gg_main call (init, worklist set-up, the persistent "
                "driver); total_ms: the reference's own timer around gg_main, its worklist cudaMallocs included "
                "(padded by the harness, oracle/ref/launch_wrap.cu); GTEPS as the harmonic mean over sources",
    }
    if our_e2e_gteps is not None and ref_total_gteps:
        res["this_engine_e2e_gteps"] = our_e2e_gteps
        res["speedup_e2e_vs_total_time"] = our_e2e_gteps / ref_total_gteps
    log(f"[{name}] reference build: kernel {res['kernel_ms_mean']:.3f} ms ({ref_gteps:.2f} GTEPS), total "
        f"{res['total_ms_mean']:.1f} ms; this engine {ours:.2f} GTEPS; parity {res['parity_vs_reference_build']}")
    return res


def _drop_file_cache(path) -> bool:
    """Evicts one file's pages from the page cache (fsync, then
    POSIX_FADV_DONTNEED on that file only), so the next read comes from the
    storage device."""
    try:
        fd = os.open(str(path), os.O_RDONLY)
        try:
            os.fsync(fd)
            os.posix_fadvise(fd, 0, 0, os.POSIX_FADV_DONTNEED)
        finally:
            os.close(fd)
        return True
    except (OSError, AttributeError):
        return False


def bench_ingest(gft, name: str, host, dev: int, reps: int = 3) -> dict:
    """.gr ingest of a full-size graph: this engine's gft_graph_load_gr
    (parallel chunked reads into pinned staging, overlapped with the H2D
    copies, destinations checked on the device) against the reference's own
    CSRGraph::read + copy_to_gpu (oracle/_ref/ingest: a serial per-edge
    parse loop over an mmap, then synchronous pageable copies,
    rt/src/csr_graph.cu:152-261), both from the page cache right after the
    file was written (warm) and after the file's pages were dropped (cold).
    GB/s = file bytes / (parse + upload) time."""
    tmp = Path(tempfile.mkdtemp(prefix="gft_ingest_"))
    try:
        gr = tmp / f"{name}.gr"
        host.write(gr)
        size = gr.stat().st_size
        res = {"file_bytes": size, "nodes": host.nnodes, "edges": host.nedges}

        def ours():
            t = time.perf_counter()
            d = gft.DeviceGraph.load_gr(gr, device=dev)
            dt = time.perf_counter() - t
            d.free()
            return dt

        def theirs():
            exe = REF_BUILD / "ingest"
            r = subprocess.run([str(exe), str(gr)], capture_output=True, text=True, timeout=600)
            if r.returncode != 0:
                raise RuntimeError(f"ingest exited {r.returncode}: {r.stderr[-500:]}")
            m = re.search(r"oracle-ref-ingest read_ns (\d+) upload_ns (\d+)", r.stderr)
            return int(m[1]) / 1e9, int(m[2]) / 1e9

        ours()  # first call pins the staging buffers
        warm = min(ours() for _ in range(reps))
        res["gft_warm"] = {"s": warm, "gbs": size / warm / 1e9}
        if (REF_BUILD / "ingest").exists():
            rr, ru = theirs()
            res["reference_warm"] = {"read_s": rr, "upload_s": ru, "s": rr + ru, "gbs": size / (rr + ru) / 1e9}
            res["speedup_warm"] = (rr + ru) / warm
        if _drop_file_cache(gr):
            cold = ours()
            res["gft_cold"] = {"s": cold, "gbs": size / cold / 1e9}
            if (REF_BUILD / "ingest").exists() and _drop_file_cache(gr):
                rr, ru = theirs()
                res["reference_cold"] = {"read_s": rr, "upload_s": ru, "s": rr + ru, "gbs": size / (rr + ru) / 1e9}
                res["speedup_cold"] = (rr + ru) / cold
        log(f"[ingest {name}] {size / 1e9:.2f} GB: gft {res['gft_warm']['gbs']:.1f} GB/s warm"
            + (f", reference {res['reference_warm']['gbs']:.2f} GB/s" if "reference_warm" in res else "")
            + (f"; cold gft {res['gft_cold']['gbs']:.1f} GB/s" if "gft_cold" in res else "")
            + (f", reference {res['reference_cold']['gbs']:.2f} GB/s" if "reference_cold" in res else ""))
        return res
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def oracle_parity_many(orc, spec, host, gpu_digests: dict, threads: int) -> dict:
    """Every source's result from this engine (as a digest) against the CPU
    oracle's, the oracle queries spread over host threads."""
    import hashlib

    def one(s):
        if spec["app"] == "sssp":
            ref = orc.sssp(host.row_start, host.edge_dst, host.edge_data, s)
        else:
            ref = orc.bfs(host.row_start, host.edge_dst, s)
        return s, hashlib.sha256(ref.tobytes()).hexdigest() == gpu_digests[s]

    t = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(one, list(gpu_digests)))
    bad = [s for s, ok in res if not ok]
    return {"sources_checked": len(res), "result": "bit-exact" if not bad else f"{len(bad)} MISMATCHES {bad[:8]}",
            "threads": threads, "wall_s": time.perf_counter() - t}


# ---------------------------------------------------------------------------
# reference arm: the reference's own CUDA build on this GPU
# ---------------------------------------------------------------------------
def workload_config(name: str, spec: dict, nnodes: int, nedges: int, weighted: bool, timed_src, e_r: float,
                    v_r: float, world: int) -> dict:
    """The workload description both arms print (identical for the same
    workload, graph and sources)."""
    graph_bytes = (nnodes + 1) * 4 + nedges * (8 if weighted else 4)
    return {
        "workload": name,
        "app": spec["app"],
        "graph": {k: v for k, v in spec.items() if k not in ("app", "nsrc", "src_seed", "delta")},
        **({"reference_default_delta": spec["delta"]} if "delta" in spec else {}),
        "nodes": nnodes,
        "edges": nedges,
        "sources": list(timed_src) if len(timed_src) <= 4 else f"{len(set(timed_src))} seeded (seed {spec['src_seed']})",
        "E_r_per_query": e_r,
        "V_r_per_query": v_r,
        "l2": ("inputs larger than L2 (graph %.2f GB > 126 MB), no flush" % (graph_bytes / 1e9))
        if graph_bytes > L2_BYTES else "graph smaller than L2 (resident between steps)",
        "parallelism": f"replicas x{world}",
    }


def _visible_gpu() -> str:
    v = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0].strip()
    return v or "0"


def reference_arm(args) -> int:
    """The reference's own BFS/SSSP, compiled for sm_100a from its sources
    (oracle/_ref, oracle/ref/Makefile), on the same seeded graph, sources and
    step count as the engine's arm.  The graph comes from oracle/libgrgen.so
    (the engine's generators built without the engine library) and is
    written as .gr for the reference's own reader.  One process runs the
    reference's gg_main once per step (oracle/ref/multi_driver.cu): `value`
    is E_r over the summed device time of each call's kernels, `e2e` E_r
    over the reference's own timer around gg_main (its worklist allocations
    included).  Rank 0 only; other ranks exit at once."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    name = args.workload
    spec = WORKLOADS.get(name)
    exe = REF_BUILD / f"{spec['app']}_multi" if spec else None
    if spec is None or not exe.exists():
        why = (f"no reference build for workload {name}" if spec is None else
               f"{exe.relative_to(ROOT)} is not built (make -C oracle/ref needs the reference sources)")
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return 0
    from oracle import grgen
    from oracle import oracle as orc

    kw = {k: v for k, v in spec.items() if k not in ("kind", "seed", "app", "nsrc", "src_seed", "delta")}
    if spec["kind"] == "grid":
        kw["max_weight"] = 1
    t0 = time.time()
    host = grgen.generate(spec["kind"], spec["seed"], **kw)
    sources = [0] if spec["nsrc"] == 0 else host.pick_sources(spec["src_seed"], spec["nsrc"])
    step_src = [sources[i % len(sources)] for i in range(max(args.steps, len(sources)))]
    timed_src = step_src[:args.steps] if len(sources) <= args.steps else sources
    warm_src = [sources[i % len(sources)] for i in range(args.warmup)]
    distinct = sorted(set(timed_src), key=timed_src.index)
    tmp = Path(tempfile.mkdtemp(prefix="gft_refarm_"))
    try:
        gr = tmp / f"{name}.gr"
        host.write_gr(gr)
        log(f"[reference] {name}: graph {host.nnodes} nodes {host.nedges} edges written in {time.time() - t0:.1f}s")
        dump = tmp / "dump"
        dump.mkdir()
        try:
            # First pass: one call per distinct source, results dumped for E_r.
            run_reference_build(spec["app"], gr, distinct, delta=spec.get("delta"), dump_dir=dump)
            reach = {}
            for s in distinct:
                val = np.fromfile(dump / f"{s}.i32", dtype=np.int32)
                reach[s] = orc.reach_stats(host.row_start, val)
            clocks = ClockSampler(_visible_gpu())
            calls = run_reference_build(spec["app"], gr, warm_src + list(timed_src), delta=spec.get("delta"))
            clk = clocks.stop()
        except (RuntimeError, OSError, subprocess.TimeoutExpired) as ex:
            # The reference build could not run here (no usable GPU, say).
            why = " ".join(str(ex).split())[:300]
            print(json.dumps({"impl": "reference", "unavailable": f"the reference build did not run: {why}"}),
                  flush=True)
            host.close()
            return 0
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    timed = calls[len(warm_src):]
    kms = [c["kernel_ms"] for c in timed]
    tot = [c["total_ns"] / 1e6 for c in timed]
    e_sum = sum(reach[c["source"]][1] for c in timed)
    v_sum = sum(reach[c["source"]][0] for c in timed)
    k = len(timed)
    value = e_sum / (sum(kms) * 1e6)
    e2e_value = e_sum / (sum(tot) * 1e6)
    per_q = [reach[c["source"]][1] / (c["kernel_ms"] * 1e6) for c in timed]
    line = {
        "impl": "reference",
        "metric": "GTEPS per query",
        "value": value,
        "unit": "GTEPS",
        "n_gpus": args.gpus,
        "steps": k,
        "warmup": args.warmup,
        "ms_per_step": statistics.mean(kms),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic: the same seeded graph and sources as the gft arm (oracle/libgrgen.so), written as .gr and "
                "read by the reference's own reader",
        "config": workload_config(name, spec, host.nnodes, host.nedges, host.edge_data is not None, timed_src,
                                  e_sum / k, v_sum / k, 1),
        "detail": {
            "binary": f"oracle/_ref/{spec['app']}_multi: the reference's gg_main, kernels and worklists "
                      "(apps/{bfs,sssp}/kernel.cu) compiled for sm_100a; one process, one gg_main call per step",
            **({"delta": spec["delta"]} if spec["app"] == "sssp" else {}),
            "kernel_ms_mean": statistics.mean(kms),
            "total_time_ms_mean": statistics.mean(tot),
            "gteps_hmean_kernel": len(per_q) / sum(1.0 / x for x in per_q),
            "launch": "the reference's own sizing: kernel_sizing (8 CTAs of 256 per SM), persistent driver at "
                      "min(blocks, SMs x residency), launched cooperatively by the harness",
        },
        "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "E_r over the reference's own timer around gg_main (skelapp/skel.cu:55-66): its worklist "
                        "cudaMallocs, init kernels and the traversal; the graph is already on the device and the "
                        "result stays there, as in the reference's CLI"},
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": 1, "kind": "reference",
                         "sample": f"{k} {spec['app'].upper()} queries of the reference's own CUDA build on this "
                                   "B200 (the reference has no CPU implementation of this path), driven by one host "
                                   "thread"},
        "gpu_launches": None,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    host.close()
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("gft", "reference"), default="gft")
    ap.add_argument("--workload",
                    choices=sorted(WORKLOADS) + sorted(CC_WORKLOADS) + sorted(PR_WORKLOADS) + sorted(MIS_WORKLOADS)
                    + ["serve-8-graphs", "batch-sssp-512", "msbfs-rmat24-256"],
                    default=HEADLINE, help="a traversal workload (the headline by default), or a connected-components, "
                                           "PageRank or maximal-independent-set one")
    ap.add_argument("--no-secondary", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--no-reference-build", action="store_true",
                    help="skip running the reference's own CUDA build (oracle/_ref) beside this engine")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload in CC_WORKLOADS or args.workload in PR_WORKLOADS or args.workload in MIS_WORKLOADS:
        return cc_arm(args)
    if args.workload in ("serve-8-graphs", "batch-sssp-512", "msbfs-rmat24-256"):
        return many_arm(args)
    return our_arm(args)


def many_arm(args) -> int:
    """One of the many-query workloads (serving, batching, multi-source BFS)
    alone on one GPU, as a JSON line."""
    import torch

    import galoisgpu_b200 as gft

    torch.cuda.set_device(0)
    fn = {"serve-8-graphs": bench_serve, "batch-sssp-512": bench_batch, "msbfs-rmat24-256": bench_msbfs}[args.workload]
    r = fn(gft, 0)
    print(json.dumps({"workload": args.workload, "n_gpus": 1, "data": "synthetic: seeded graphs generated on the device",
                      **r}), flush=True)
    return 0


def cc_arm(args) -> int:
    """One connected-components, PageRank or maximal-independent-set
    workload on one GPU, as a JSON line."""
    import torch

    import galoisgpu_b200 as gft
    from oracle import oracle as orc

    torch.cuda.set_device(0)
    is_pr, is_mis = args.workload in PR_WORKLOADS, args.workload in MIS_WORKLOADS
    fn, table = (bench_pr, PR_WORKLOADS) if is_pr else (bench_mis, MIS_WORKLOADS) if is_mis else (bench_cc, CC_WORKLOADS)
    r = fn(gft, orc, args.workload, 0, steps=args.steps, warmup=args.warmup)
    line = {**r, "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if is_pr else "u32",
            "data": "synthetic: seeded graph generated on the device (SplitMix64 streams)",
            "config": {"workload": args.workload, **table[args.workload]}}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
