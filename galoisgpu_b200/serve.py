"""Serving: a request loop over resident graphs with continuous batching
(the gft_serve_* C ABI), plus a Poisson load generator that reports
throughput and p50/p99 latency.

The server splits the device's CTAs into lanes (streams).  A large query
runs alone as one CTA group over a fair share of the free lanes (the whole
device when the server is idle, one lane under load); small queries are
packed into micro-batches on one lane, one CTA each.  Requests that arrive
while others are on the GPU start as soon as a lane and scratch memory are
free.  See include/gft.h.
"""

from __future__ import annotations

import ctypes as C
import math
import random
import threading
import time

from ._lib import Completion, Query, ServeConfig, check, load
from .graph import DEFAULT_DELTA, DeviceGraph, Engine


class Server:
    def __init__(self, engine: Engine, **cfg):
        c = ServeConfig()
        check(load().gft_serve_config_default(C.byref(c)))
        for k, v in cfg.items():
            if not hasattr(c, k):
                raise TypeError(f"unknown serving option {k!r}")
            setattr(c, k, v)
        self.config = {name: getattr(c, name) for name, _ in ServeConfig._fields_}
        h = C.c_void_p()
        check(load().gft_serve_open(engine._h, C.byref(c), C.byref(h)))
        self._h = h
        self._q = Query()

    def enqueue(self, graph: DeviceGraph, app: str, src: int, out, delta: int = DEFAULT_DELTA, parent=None) -> int:
        """Admits one request; `out` (int32 device tensor of graph.nnodes) must
        stay alive until the request's completion is polled.  With
        resident=1 the request is ordered with no stream: any pending work
        that writes `out` must have finished first."""
        q = self._q
        q.graph = graph.handle
        q.app = 1 if app == "sssp" else 0
        q.src = src
        q.delta = delta if app == "sssp" else 0
        q.d_out = out.data_ptr()
        q.d_parent = parent.data_ptr() if parent is not None else None
        t = C.c_uint64()
        check(load().gft_serve_enqueue(self._h, C.byref(q), C.byref(t)))
        return t.value

    def poll(self, max_items: int = 4096, wait_us: int = 0) -> list[dict]:
        buf = (Completion * max_items)()
        n = C.c_uint32()
        check(load().gft_serve_poll(self._h, buf, max_items, C.byref(n), wait_us))
        return [{name: getattr(buf[i], name) for name, _ in Completion._fields_} for i in range(n.value)]

    def stats(self) -> dict:
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(load().gft_serve_stats(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"in_flight": a.value, "batches": b.value, "queries": c.value}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            check(load().gft_serve_close(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _pct(xs, q):
    if not xs:
        return None
    xs = sorted(xs)
    return xs[min(len(xs) - 1, max(0, math.ceil(q * len(xs)) - 1))]


def poisson_run(server: Server, graphs: list[DeviceGraph], sources: list[list[int]], pools: list[list], rate: float,
                n_requests: int, seed: int = 7, bfs_fraction: float = 0.5, delta: int = 40000) -> dict:
    """Offers `n_requests` Poisson arrivals at `rate` per second, uniformly
    over `graphs` (BFS with probability bfs_fraction, else SSSP) from the
    given source lists.  Each request needs a free output buffer from its
    graph's pool; when none is free the arrival waits (counted as
    throttled).  Returns achieved throughput and latency percentiles."""
    rng = random.Random(seed)
    free = [list(range(len(p))) for p in pools]
    lock = threading.Lock()
    busy = {}  # ticket -> (graph index, buffer index)
    lat, qms, lanes, bsz, width, slow = [], [], {}, [], [], []
    failures = 0
    done = [0]
    stop = [False]

    def collector():
        nonlocal failures
        last = time.perf_counter()
        while not stop[0] or done[0] < n_requests:
            if time.perf_counter() - last > 300:
                raise TimeoutError(f"poisson_run: no completion for 300 s ({done[0]} of {n_requests} done)")
            for c in server.poll(4096, 2000):
                last = time.perf_counter()
                with lock:
                    gi, bi, app = busy.pop(c["ticket"])
                    free[gi].append(bi)
                slow.append((c["latency_ms"], gi, app, c["width"], c["queue_ms"]))
                if c["status"] != 0:
                    failures += 1
                lat.append(c["latency_ms"])
                qms.append(c["queue_ms"])
                lanes[c["lane"]] = lanes.get(c["lane"], 0) + 1
                bsz.append(c["batch_size"])
                width.append(c["width"])
                done[0] += 1
            if stop[0] and done[0] >= n_requests:
                break

    errors = []

    def collector_guarded():
        try:
            collector()
        except Exception as ex:  # surfaced below instead of hanging the join
            errors.append(ex)

    th = threading.Thread(target=collector_guarded, daemon=True)
    th.start()
    throttled = 0
    t0 = time.perf_counter()
    t_next = 0.0
    for _ in range(n_requests):
        t_next += rng.expovariate(rate)
        gi = rng.randrange(len(graphs))
        app = "bfs" if rng.random() < bfs_fraction else "sssp"
        src = rng.choice(sources[gi])
        while time.perf_counter() - t0 < t_next:
            pass
        waited = False
        while True:
            with lock:
                if free[gi]:
                    bi = free[gi].pop()
                    break
            waited = True
            time.sleep(20e-6)
        throttled += waited
        with lock:  # the collector may see the completion before enqueue returns
            t = server.enqueue(graphs[gi], app, src, pools[gi][bi], delta=delta)
            busy[t] = (gi, bi, app)
    offered_s = time.perf_counter() - t0
    stop[0] = True
    th.join(timeout=600)
    if errors:
        raise errors[0]
    elapsed = time.perf_counter() - t0
    return {
        "offered_rate": rate,
        "requests": n_requests,
        "achieved_qps": n_requests / elapsed,
        "offer_s": offered_s,
        "p50_ms": _pct(lat, 0.5),
        "p99_ms": _pct(lat, 0.99),
        "queue_p50_ms": _pct(qms, 0.5),
        "mean_batch": sum(bsz) / max(1, len(bsz)),
        "mean_width": sum(width) / max(1, len(width)),
        "lanes": lanes,
        "throttled_arrivals": throttled,
        "failures": failures,
        # The slowest requests: (latency ms, graph index, app, team width, queue ms).
        "slowest": sorted(slow, reverse=True)[:5],
    }
