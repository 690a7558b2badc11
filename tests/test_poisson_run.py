"""galoisgpu_b200.serve.poisson_run, the load generator behind the serving
numbers, against a stand-in server on the CPU: every request completes once,
no output buffer is handed to two requests in flight, arrivals that find
their graph's buffers all busy are counted as throttled, and the reported
latency percentiles are the server's."""

import threading
import time

import pytest


class _FakeServer:
    """Completes each request `service_ms` after its enqueue, in order;
    records which buffers are in flight."""

    def __init__(self, service_ms: float, fail_every: int = 0):
        self.service = service_ms / 1e3
        self.fail_every = fail_every
        self.lock = threading.Lock()
        self.pending = []  # (due, ticket, buffer id, enqueue time)
        self.in_flight = set()
        self.max_in_flight = 0
        self.reused = False
        self.next = 0

    def enqueue(self, graph, app, src, out, delta=0):
        with self.lock:
            t = self.next
            self.next += 1
            if id(out) in self.in_flight:
                self.reused = True
            self.in_flight.add(id(out))
            self.max_in_flight = max(self.max_in_flight, len(self.in_flight))
            now = time.perf_counter()
            self.pending.append((now + self.service, t, id(out), now))
            return t

    def poll(self, max_n, wait_us):
        end = time.perf_counter() + wait_us / 1e6
        while True:
            now = time.perf_counter()
            with self.lock:
                ready = [p for p in self.pending if p[0] <= now][:max_n]
                for p in ready:
                    self.pending.remove(p)
                    self.in_flight.discard(p[2])
            if ready or now >= end:
                break
            time.sleep(50e-6)
        return [{"ticket": t, "status": 1 if self.fail_every and (t + 1) % self.fail_every == 0 else 0,
                 "latency_ms": (now - t0) * 1e3, "queue_ms": 0.0, "lane": 1 + t % 3, "batch_size": 1, "width": 2}
                for _, t, _, t0 in ready]


class _G:
    nnodes = 4


def test_every_request_completes_once_with_its_own_buffer():
    from galoisgpu_b200.serve import poisson_run

    srv = _FakeServer(service_ms=2.0, fail_every=50)
    pools = [[object() for _ in range(4)], [object() for _ in range(4)]]
    r = poisson_run(srv, [_G(), _G()], [[0, 1], [2]], pools, rate=2000, n_requests=300)
    assert r["requests"] == 300 and not srv.pending
    assert not srv.reused and srv.max_in_flight <= 8
    assert r["failures"] == 6
    assert 2.0 <= r["p50_ms"] <= r["p99_ms"] < 50
    assert sum(r["lanes"].values()) == 300 and r["mean_width"] == 2
    assert r["slowest"][0][0] >= r["p99_ms"]


def test_a_small_pool_throttles_arrivals():
    from galoisgpu_b200.serve import poisson_run

    srv = _FakeServer(service_ms=5.0)
    r = poisson_run(srv, [_G()], [[0]], [[object()]], rate=5000, n_requests=60)
    assert srv.max_in_flight == 1 and not srv.reused
    assert r["throttled_arrivals"] > 30
    assert r["achieved_qps"] < 250  # one buffer, 5 ms each
