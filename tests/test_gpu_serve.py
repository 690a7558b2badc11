"""Serving with continuous batching: every result of a request served in a
mix of concurrent requests equals the same query run alone (bit for bit),
requests really are batched and overlapped, and admission errors are
statuses."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def drain(srv, n: int, deadline_s: float = 120.0) -> dict:
    """Polls until n completions arrived; fails (instead of waiting forever)
    when one is lost."""
    got = {}
    t_end = time.monotonic() + deadline_s
    while len(got) < n:
        assert time.monotonic() < t_end, f"only {len(got)} of {n} completions within {deadline_s} s"
        for c in srv.poll(256, 100000):
            got[c["ticket"]] = c
    return got


def test_mix_equals_alone(gft, engine):
    import torch

    from galoisgpu_b200.serve import Server

    hosts = [gft.CSRGraph.road(60, seed=21), gft.CSRGraph.road(200, seed=22), gft.CSRGraph.rmat(11, 8, seed=23, max_weight=255),
             gft.CSRGraph.rmat(14, 8, seed=24, max_weight=255), gft.CSRGraph.grid(30, 30, 0, 7)]
    devs = [h.copy_to_gpu() for h in hosts]
    # Queries on the 2^14- and 40,000-vertex graphs run on CTA groups (except
    # BFS on the sparse road graph), the rest on one CTA each.
    srv = Server(engine, max_batch=16, group_min_nodes=1 << 14, group_blocks=8, lane_arena_bytes=64 << 20)
    reqs = []
    for i in range(120):
        gi = i % len(devs)
        src = hosts[gi].pick_sources(300 + i, 1)[0]
        app = "sssp" if i % 3 else "bfs"
        out = torch.full((devs[gi].nnodes,), -5, dtype=torch.int32, device="cuda")
        t = srv.enqueue(devs[gi], app, src, out, delta=[100, 40000][i % 2])
        reqs.append((t, gi, app, src, out, [100, 40000][i % 2]))
    got = drain(srv, len(reqs))
    st = srv.stats()
    srv.close()
    assert all(c["status"] == 0 for c in got.values())
    assert max(c["batch_size"] for c in got.values()) > 1, "requests were never batched"
    assert len({c["lane"] for c in got.values()}) > 1, "micro-batches never overlapped on several lanes"
    assert st["batches"] < st["queries"]
    for t, gi, app, src, out, delta in reqs:
        alone = (engine.sssp(devs[gi], src, delta=delta) if app == "sssp" else engine.bfs(devs[gi], src))["out"]
        np.testing.assert_array_equal(out.cpu().numpy(), alone.cpu().numpy())


def test_idle_server_gives_a_heavy_request_the_device(gft, engine):
    import torch

    from galoisgpu_b200.serve import Server

    h = gft.CSRGraph.road(200, seed=5)
    d = h.copy_to_gpu()
    srv = Server(engine, group_min_nodes=1 << 12, group_blocks=8, lane_arena_bytes=64 << 20)
    out = torch.empty(d.nnodes, dtype=torch.int32, device="cuda")
    srv.enqueue(d, "sssp", 3, out, delta=1000)
    got = list(drain(srv, 1).values())
    srv.close()
    assert got[0]["status"] == 0 and got[0]["width"] > 1
    np.testing.assert_array_equal(out.cpu().numpy(), engine.sssp(d, 3, delta=1000)["out"].cpu().numpy())


def test_admission_errors(gft, engine):
    import torch

    from galoisgpu_b200.serve import Server

    h = gft.CSRGraph.road(300, seed=3)
    d = h.copy_to_gpu()
    srv = Server(engine, lanes=1, lane_arena_bytes=1 << 16)
    out = torch.empty(d.nnodes, dtype=torch.int32, device="cuda")
    with pytest.raises(gft.GftError) as ei:
        srv.enqueue(d, "sssp", 0, out)
    assert ei.value.status_name == "GFT_ERR_OOM"
    with pytest.raises(gft.GftError) as ei:
        srv.enqueue(d, "bfs", d.nnodes, out)
    assert ei.value.status_name == "GFT_ERR_INVALID_ARG"
    srv.close()


def test_poisson_load_smoke(gft, engine):
    import torch

    from galoisgpu_b200.serve import Server, poisson_run

    hosts = [gft.CSRGraph.road(100, seed=31), gft.CSRGraph.rmat(12, 8, seed=32, max_weight=255)]
    devs = [h.copy_to_gpu() for h in hosts]
    srcs = [h.pick_sources(5, 64) for h in hosts]
    pools = [[torch.empty(d.nnodes, dtype=torch.int32, device="cuda") for _ in range(32)] for d in devs]
    srv = Server(engine, lanes=2, max_batch=64)
    r = poisson_run(srv, devs, srcs, pools, rate=2000, n_requests=400)
    srv.close()
    assert r["failures"] == 0 and r["requests"] == 400
    assert r["p99_ms"] is not None and r["p99_ms"] >= r["p50_ms"] > 0


def test_wide_pool_for_skewed_sssp(gft, engine):
    """SSSP on a skewed graph of at least wide_min_edges edges runs on the
    reserved wide pool (lane 1 onwards, many lanes at once), everything else
    on the shared lanes; every result equals the query run alone."""
    import torch

    from galoisgpu_b200.serve import Server

    rm = gft.CSRGraph.rmat(13, 8, seed=41, max_weight=255)
    rd = gft.CSRGraph.road(90, seed=42)
    devs = [rm.copy_to_gpu(), rd.copy_to_gpu()]
    srv = Server(engine, group_min_nodes=1 << 10, group_blocks=8, lane_arena_bytes=64 << 20, wide_min_edges=1)
    reqs = []
    for i in range(48):
        gi, app = i % 2, ("sssp" if i % 3 else "bfs")
        host = (rm, rd)[gi]
        src = host.pick_sources(500 + i, 1)[0]
        out = torch.full((devs[gi].nnodes,), -5, dtype=torch.int32, device="cuda")
        reqs.append((srv.enqueue(devs[gi], app, src, out, delta=300), gi, app, src, out))
    got = drain(srv, len(reqs))
    srv.close()
    wide = [got[t] for t, gi, app, _, _ in reqs if gi == 0 and app == "sssp"]
    assert wide and all(c["lane"] == 1 and c["width"] >= 2 for c in wide)
    others = [got[t] for t, gi, app, _, _ in reqs if not (gi == 0 and app == "sssp")]
    assert all(c["lane"] > 1 for c in others), "shared requests never start on the wide pool"
    for t, gi, app, src, out in reqs:
        assert got[t]["status"] == 0
        alone = (engine.sssp(devs[gi], src, delta=300) if app == "sssp" else engine.bfs(devs[gi], src))["out"]
        np.testing.assert_array_equal(out.cpu().numpy(), alone.cpu().numpy())


# ---------------------------------------------------------------------------
# Resident mode: one persistent kernel, requests through a mapped ring, teams
# of lanes drafted on the device.
# ---------------------------------------------------------------------------
def test_resident_mix_equals_alone(gft, engine):
    import torch

    from galoisgpu_b200.serve import Server

    hosts = [gft.CSRGraph.road(60, seed=21), gft.CSRGraph.road(200, seed=22),
             gft.CSRGraph.rmat(11, 8, seed=23, max_weight=255), gft.CSRGraph.rmat(14, 8, seed=24, max_weight=255),
             gft.CSRGraph.grid(30, 30, 0, 7)]
    devs = [h.copy_to_gpu() for h in hosts]
    # Resident requests are ordered with no stream: the outputs' fills must
    # be finished before the requests are enqueued.
    plan = []
    for i in range(160):
        gi = i % len(devs)
        src = hosts[gi].pick_sources(300 + i, 1)[0]
        out = torch.full((devs[gi].nnodes,), -5, dtype=torch.int32, device="cuda")
        plan.append((gi, "sssp" if i % 3 else "bfs", src, out, [100, 40000][i % 2]))
    torch.cuda.synchronize()
    srv = Server(engine, resident=1, lane_blocks=8, lane_arena_bytes=64 << 20)
    reqs = [(srv.enqueue(devs[gi], app, src, out, delta=d), gi, app, src, out, d) for gi, app, src, out, d in plan]
    got = drain(srv, len(reqs))
    st = srv.stats()
    srv.close()
    assert all(c["status"] == 0 for c in got.values()), [c["status"] for c in got.values() if c["status"]]
    assert len({c["lane"] for c in got.values()}) > 1, "requests never ran on several teams at once"
    assert st["batches"] < st["queries"], "one kernel launch per request: the kernel did not stay resident"
    for t, gi, app, src, out, delta in reqs:
        alone = (engine.sssp(devs[gi], src, delta=delta) if app == "sssp" else engine.bfs(devs[gi], src))["out"]
        np.testing.assert_array_equal(out.cpu().numpy(), alone.cpu().numpy())


def test_resident_idle_server_gives_a_request_every_lane_and_relaunches(gft, engine):
    import torch

    from galoisgpu_b200.serve import Server

    h = gft.CSRGraph.road(300, seed=5)
    d = h.copy_to_gpu()
    srv = Server(engine, resident=1, lane_blocks=8, lane_arena_bytes=64 << 20, idle_exit_us=1000)
    outs, widths = [], []
    for k in range(2):
        out = torch.empty(d.nnodes, dtype=torch.int32, device="cuda")
        srv.enqueue(d, "sssp", 3 + k, out, delta=1000)
        c = list(drain(srv, 1).values())[0]
        assert c["status"] == 0, c
        widths.append(c["width"])
        outs.append(out)
        time.sleep(0.05)  # longer than idle_exit_us: the kernel ends and the next request launches it again
    st = srv.stats()
    srv.close()
    # Alone on an idle server, each request gets every lane.
    assert widths[0] > 1 and widths[0] == widths[1], widths
    assert st["batches"] == 2, st
    for k, out in enumerate(outs):
        np.testing.assert_array_equal(out.cpu().numpy(), engine.sssp(d, 3 + k, delta=1000)["out"].cpu().numpy())


def test_resident_close_finishes_admitted_requests(gft, engine):
    import torch

    from galoisgpu_b200.serve import Server

    h = gft.CSRGraph.rmat(13, 8, seed=41, max_weight=255)
    d = h.copy_to_gpu()
    srv = Server(engine, resident=1, lane_arena_bytes=64 << 20)
    srcs = h.pick_sources(9, 24)
    outs = [torch.full((d.nnodes,), -5, dtype=torch.int32, device="cuda") for _ in srcs]
    torch.cuda.synchronize()  # the fills finish before the requests reach the resident kernel
    for s, o in zip(srcs, outs):
        srv.enqueue(d, "bfs", s, o)
    srv.close()
    for s, o in zip(srcs, outs):
        np.testing.assert_array_equal(o.cpu().numpy(), engine.bfs(d, s)["out"].cpu().numpy())


def test_resident_admission_errors(gft, engine):
    import torch

    from galoisgpu_b200.serve import Server

    h = gft.CSRGraph.road(300, seed=3)
    d = h.copy_to_gpu()
    srv = Server(engine, resident=1, lane_arena_bytes=1 << 16)
    out = torch.empty(d.nnodes, dtype=torch.int32, device="cuda")
    with pytest.raises(gft.GftError) as ei:
        srv.enqueue(d, "sssp", 0, out)
    assert ei.value.status_name == "GFT_ERR_OOM"
    with pytest.raises(gft.GftError) as ei:
        srv.enqueue(d, "bfs", d.nnodes, out)
    assert ei.value.status_name == "GFT_ERR_INVALID_ARG"
    srv.close()
