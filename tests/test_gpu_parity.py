"""GPU parity: libgft BFS / SSSP (through the C ABI) against the CPU oracle,
bit for bit, plus parent-tree validity, on hand graphs and seeded synthetic
graphs at sizes the oracle finishes in seconds."""

import numpy as np
import pytest

from graphs import hand_cases

pytestmark = pytest.mark.gpu

TUNES = [
    dict(),  # small graphs run on one CTA, larger ones on the whole grid
    dict(block_threads=256, blocks_per_sm=4, max_blocks=1 << 30),  # always the grid
    dict(block_threads=1024, blocks_per_sm=1, max_blocks=1 << 30),
    dict(hub_degree=32, max_blocks=1 << 30),  # every vertex of degree >= 32 goes through the grid-wide hub phase
    dict(max_blocks=1, hub_degree=32),  # always one CTA
    dict(queue_tile=64, warp_degree=8, max_blocks=1 << 30),  # small push buffers, warps from degree 8
    dict(block_threads=512, queue_tile=256, warp_degree=128, max_blocks=1 << 30),  # edge lists < 128 flattened
]
TUNE_IDS = ["auto", "grid256x4", "grid1024x1", "grid-hub32", "one-cta", "tile64-warp8", "tile256-warp128"]


def _sources(n):
    return sorted({0, n // 2, n - 1})


def _run_bfs(gft, engine, dg, src, tune=None):
    import torch

    par = torch.empty(dg.nnodes, dtype=torch.int32, device="cuda")
    r = engine.bfs(dg, src, parent=par, tune=gft.Tune(**tune) if tune else None)
    return r["out"].cpu().numpy(), r["parent"].cpu().numpy().view(np.uint32), r


def _run_sssp(gft, engine, dg, src, delta, tune=None):
    import torch

    par = torch.empty(dg.nnodes, dtype=torch.int32, device="cuda")
    r = engine.sssp(dg, src, delta=delta, parent=par, tune=gft.Tune(**tune) if tune else None)
    return r["out"].cpu().numpy(), r["parent"].cpu().numpy().view(np.uint32), r


@pytest.mark.parametrize("case", hand_cases(), ids=lambda c: c[0])
def test_hand_graphs_bfs_sssp(gft, orc, engine, case):
    name, rs, dst, w = case
    g = gft.CSRGraph(rs, dst, w)
    dg = g.copy_to_gpu()
    for src in _sources(g.nnodes):
        want = orc.bfs(rs, dst, src)
        got, par, _ = _run_bfs(gft, engine, dg, src)
        np.testing.assert_array_equal(got, want)
        assert orc.check_tree(rs, dst, None, src, got, par) == 0
        for delta in (1, 7, 10000):
            want = orc.sssp(rs, dst, w, src)
            got, par, _ = _run_sssp(gft, engine, dg, src, delta)
            np.testing.assert_array_equal(got, want)
            if w is not None and (w > 0).all():
                assert orc.check_tree(rs, dst, w, src, got, par) == 0


@pytest.mark.parametrize("tune", TUNES, ids=lambda t: ",".join(f"{k}={v}" for k, v in t.items()) or "default")
def test_grid_bfs_closed_form(gft, orc, engine, tune):
    g = gft.CSRGraph.grid(256, 256)
    dg = g.copy_to_gpu()
    got, par, st = _run_bfs(gft, engine, dg, 0, tune)
    r, c = np.divmod(np.arange(g.nnodes), 256)
    np.testing.assert_array_equal(got, (r + c).astype(np.int32))
    assert orc.check_tree(g.row_start, g.edge_dst, None, 0, got, par) == 0
    assert st["levels"] == 511


@pytest.mark.parametrize("tune", TUNES, ids=lambda t: ",".join(f"{k}={v}" for k, v in t.items()) or "default")
def test_rmat_bfs_sssp(gft, orc, engine, tune):
    g = gft.CSRGraph.rmat(16, 16, seed=3, max_weight=255)
    dg = g.copy_to_gpu()
    for src in g.pick_sources(2, 3):
        want = orc.bfs(g.row_start, g.edge_dst, src)
        got, par, _ = _run_bfs(gft, engine, dg, src, tune)
        np.testing.assert_array_equal(got, want)
        assert orc.check_tree(g.row_start, g.edge_dst, None, src, got, par) == 0
        want = orc.sssp(g.row_start, g.edge_dst, g.edge_data, src)
        for delta in (16, 255, 10000):
            got, par, _ = _run_sssp(gft, engine, dg, src, delta, tune)
            np.testing.assert_array_equal(got, want)
            assert orc.check_tree(g.row_start, g.edge_dst, g.edge_data, src, got, par) == 0


@pytest.mark.parametrize("side", [362, 363], ids=["bitmap-in-shared", "bitmap-in-global"])
def test_one_cta_bfs_either_side_of_the_shared_bitmap_limit(gft, orc, engine, side):
    """A one-CTA BFS keeps its visited bitmap in shared memory for graphs of
    at most 2^17 vertices (362^2 = 131,044) and in global memory above
    (363^2 = 131,769); levels and parent trees match the oracle on both
    sides, top-down and with the direction switch."""
    g = gft.CSRGraph.road(side, seed=7)
    dg = g.copy_to_gpu()
    for src in g.pick_sources(8, 2):
        want = orc.bfs(g.row_start, g.edge_dst, src)
        for tune in (dict(max_blocks=1), dict(max_blocks=1, direction=1)):
            got, par, _ = _run_bfs(gft, engine, dg, src, tune)
            np.testing.assert_array_equal(got, want)
            assert orc.check_tree(g.row_start, g.edge_dst, None, src, got, par) == 0


def test_one_cta_bfs_frontier_beyond_the_shared_queue_head(gft, orc, engine):
    """Small uniform-degree graphs run a thread per frontier vertex on one
    CTA, with the first 8,192 entries of each frontier queue in shared
    memory and the rest in global memory.  A random graph of 120,000
    vertices and degree <= 32 has levels of tens of thousands of vertices,
    so both parts of the queue carry vertices; levels and parents stay
    exact."""
    rng = np.random.default_rng(12)
    n, m = 120_000, 240_000
    u = rng.integers(0, n, m, dtype=np.int64)
    v = rng.integers(0, n, m, dtype=np.int64)
    keep = u != v
    a = np.concatenate([u[keep], v[keep]])
    b = np.concatenate([v[keep], u[keep]])
    key = np.unique(a * n + b)
    src_of, dst = (key // n).astype(np.uint32), (key % n).astype(np.uint32)
    rs = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum(np.bincount(src_of, minlength=n), out=rs[1:])
    assert int(np.diff(rs.astype(np.int64)).max()) <= 32 and len(dst) <= 1 << 19
    g = gft.CSRGraph(rs, dst, None)
    dg = g.copy_to_gpu()
    for src in g.pick_sources(13, 2):
        want = orc.bfs(rs, dst, src)
        reached = want != np.iinfo(np.int32).max
        assert np.bincount(want[reached]).max() > 16384
        for tune in (None, dict(max_blocks=1)):
            got, par, r = _run_bfs(gft, engine, dg, src, tune)
            np.testing.assert_array_equal(got, want)
            assert orc.check_tree(rs, dst, None, src, got, par) == 0
            assert r["grid_blocks"] == 1
            assert r["vertices_reached"] == int(reached.sum()) - 1  # the source is not counted


def test_one_cta_bfs_on_graphs_with_odd_cycles(gft, orc, engine):
    """Random graphs of degree <= 4 (the one-CTA kernel's per-vertex slot
    path; 131,000 vertices take the 1024-thread CTA) and <= 9 (some
    vertices through the CSR), full of odd cycles, so that a level's
    vertices also claim one another's neighbours: levels, the level count
    and the reached count equal the oracle's, and parent trees are valid,
    with and without the parent output."""
    import torch

    rng = np.random.default_rng(31)
    for n, cap in ((30_000, 4), (50_000, 9), (131_000, 4)):
        u = rng.integers(0, n, 3 * n)
        v = rng.integers(0, n, 3 * n)
        key = np.unique(np.concatenate([u * n + v, v * n + u]))
        key = key[key // n != key % n]
        src_of, dst = key // n, key % n
        deg = np.bincount(src_of, minlength=n)
        first = np.concatenate([[0], np.cumsum(deg)[:-1]])
        rank = np.arange(len(key)) - first[src_of]
        keep = rank < cap
        pairs = set(zip(src_of[keep].tolist(), dst[keep].tolist()))
        sym = np.array(sorted(p for p in pairs if (p[1], p[0]) in pairs), dtype=np.int64)
        rs = np.zeros(n + 1, dtype=np.uint32)
        np.cumsum(np.bincount(sym[:, 0], minlength=n), out=rs[1:])
        g = gft.CSRGraph(rs, sym[:, 1].astype(np.uint32), None)
        dg = g.copy_to_gpu()
        for src in g.pick_sources(5, 3):
            want = orc.bfs(g.row_start, g.edge_dst, src)
            got, par, r = _run_bfs(gft, engine, dg, src)
            np.testing.assert_array_equal(got, want)
            assert orc.check_tree(g.row_start, g.edge_dst, None, src, got, par) == 0
            assert r["grid_blocks"] == 1
            reached = want != np.iinfo(np.int32).max
            assert r["levels"] == int(want[reached].max()) + 1
            assert r["vertices_reached"] == int(reached.sum()) - 1
            out = torch.empty(dg.nnodes, dtype=torch.int32, device="cuda")
            np.testing.assert_array_equal(engine.bfs(dg, src, out=out)["out"].cpu().numpy(), want)


def _wrap(gft, rs, dst):
    """A device graph over caller-owned device arrays (no copy, no BFS slots)."""
    import ctypes as C

    import torch

    d_rs = torch.from_numpy(rs.astype(np.int32)).cuda()
    d_dst = torch.from_numpy(dst.astype(np.int32)).cuda()
    h = C.c_void_p()
    assert gft.load().gft_graph_wrap(0, len(rs) - 1, len(dst), C.c_void_p(d_rs.data_ptr()),
                                     C.c_void_p(d_dst.data_ptr()), None, C.byref(h)) == 0
    return gft.DeviceGraph(h, 0), (d_rs, d_dst)


def test_one_cta_bfs_on_a_wrapped_graph(gft, orc, engine):
    """A wrapped graph has no per-vertex slots, so the one-CTA kernel reads
    every vertex through the CSR: a grid (degree <= 4) and a random graph
    of degree <= 12 give the oracle's levels and valid parent trees."""
    rng = np.random.default_rng(4)
    grid = gft.CSRGraph.grid(90, 110, 0, 1)
    n = 20_000
    u = rng.integers(0, n, 50_000)
    v = rng.integers(0, n, 50_000)
    key = np.unique(np.concatenate([u * n + v, v * n + u]))
    key = key[key // n != key % n]
    src_of, dst = key // n, (key % n).astype(np.uint32)
    deg = np.bincount(src_of, minlength=n)
    first = np.concatenate([[0], np.cumsum(deg)[:-1]])
    keep = np.arange(len(key)) - first[src_of] < 12  # at most 12 edges a vertex
    src_of, dst = src_of[keep], dst[keep]
    rs = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum(np.bincount(src_of, minlength=n), out=rs[1:])
    for g_rs, g_dst in ((grid.row_start, grid.edge_dst), (rs, dst)):
        dg, keep_alive = _wrap(gft, g_rs, g_dst)
        for src in (0, len(g_rs) // 2):
            want = orc.bfs(g_rs, g_dst, src)
            got, par, r = _run_bfs(gft, engine, dg, src)
            np.testing.assert_array_equal(got, want)
            assert orc.check_tree(g_rs, g_dst, None, src, got, par) == 0
            assert r["grid_blocks"] == 1
        dg.free()


def test_one_cta_bfs_reports_a_destination_outside_the_graph(gft, engine):
    """An edge leaving the graph (only possible in wrapped, caller-owned
    arrays) ends the one-CTA BFS with GFT_ERR_FORMAT, not a stray write."""
    g = gft.CSRGraph.grid(40, 40, 0, 1)
    dst = g.edge_dst.copy()
    dst[len(dst) // 2] = g.nnodes + 5
    dg, keep_alive = _wrap(gft, g.row_start, dst)
    with pytest.raises(gft.GftError) as ei:
        engine.bfs(dg, 0)
    assert ei.value.status_name == "GFT_ERR_FORMAT"
    dg.free()


def test_road_sssp(gft, orc, engine):
    g = gft.CSRGraph.road(512, seed=1)
    dg = g.copy_to_gpu()
    for src in g.pick_sources(1, 2):
        want = orc.sssp(g.row_start, g.edge_dst, g.edge_data, src)
        for delta in (1000, 10000, 100000):
            got, par, st = _run_sssp(gft, engine, dg, src, delta)
            np.testing.assert_array_equal(got, want)
            assert orc.check_tree(g.row_start, g.edge_dst, g.edge_data, src, got, par) == 0


@pytest.mark.parametrize("cta_small", [2**32 - 1, 64, 2048, 1 << 22], ids=["never", "64", "2048", "all"])
def test_sssp_small_iterations_on_one_cta(gft, orc, engine, cta_small):
    """Grid launches hand runs of small iterations to the first CTA and take
    the loop state back at a grid barrier: distances and the parent tree
    stay exact whether that never happens, happens for tiny piles only, or
    for every iteration (hubs of degree >= 32 included)."""
    for g, hub in ((gft.CSRGraph.road(400, seed=31), 0), (gft.CSRGraph.rmat(16, 16, seed=32, max_weight=255), 32),
                   (gft.CSRGraph.grid(12, 4000, 2, 50), 0)):
        dg = g.copy_to_gpu()
        tune = dict(max_blocks=1 << 30, cta_small=cta_small, hub_degree=hub)
        for src in g.pick_sources(33, 2):
            want = orc.sssp(g.row_start, g.edge_dst, g.edge_data, src)
            for delta in (100, 10000):
                got, par, _ = _run_sssp(gft, engine, dg, src, delta, tune)
                np.testing.assert_array_equal(got, want)
                assert orc.check_tree(g.row_start, g.edge_dst, g.edge_data, src, got, par) == 0


@pytest.mark.parametrize("fuse", [32, 256, 1 << 20], ids=["fuse32", "fuse256", "fuse-unbounded"])
@pytest.mark.parametrize("mode", [dict(max_blocks=1 << 30), dict(max_blocks=1), dict(max_blocks=1 << 30, hub_degree=32)],
                         ids=["grid", "one-cta", "grid-hub32"])
def test_sssp_bucket_fusion(gft, orc, engine, fuse, mode):
    """Warps that expand the near vertices they found in the same iteration
    (claimed by swapping the near tag, so later improvements queue them
    again) give the same distances and a valid parent tree."""
    for g in (gft.CSRGraph.road(400, seed=41), gft.CSRGraph.rmat(16, 16, seed=42, max_weight=255),
              gft.CSRGraph.grid(12, 4000, 3, 50)):
        dg = g.copy_to_gpu()
        for src in g.pick_sources(43, 2):
            want = orc.sssp(g.row_start, g.edge_dst, g.edge_data, src)
            for delta in (100, 10000):
                got, par, _ = _run_sssp(gft, engine, dg, src, delta, dict(mode, fuse_budget=fuse))
                np.testing.assert_array_equal(got, want)
                assert orc.check_tree(g.row_start, g.edge_dst, g.edge_data, src, got, par) == 0


def test_unweighted_sssp_is_zero_weight(gft, orc, engine):
    """An unweighted .gr has weight 0 everywhere (calloc'd edge_data in the
    reference), so every reached vertex has distance 0."""
    g = gft.CSRGraph.rmat(12, 8, seed=5)
    dg = g.copy_to_gpu()
    src = g.pick_sources(1, 1)[0]
    got, _, _ = _run_sssp(gft, engine, dg, src, 10000)
    np.testing.assert_array_equal(got, orc.sssp(g.row_start, g.edge_dst, None, src))


@pytest.mark.parametrize(
    "kind,kw,host",
    [
        ("grid", dict(rows=100, cols=37, max_weight=1), lambda g: g.CSRGraph.grid(100, 37, 1, 1)),
        ("road", dict(side=300), lambda g: g.CSRGraph.road(300, seed=1)),
        ("rmat", dict(scale=14, edge_factor=16, max_weight=255), lambda g: g.CSRGraph.rmat(14, 16, seed=1, max_weight=255)),
        ("rmat", dict(scale=12, edge_factor=8), lambda g: g.CSRGraph.rmat(12, 8, seed=1)),
    ],
)
def test_device_generator_matches_host(gft, kind, kw, host):
    dg = gft.DeviceGraph.generate(kind, seed=1, **kw)
    a = dg.download()
    b = host(gft)
    np.testing.assert_array_equal(a.row_start, b.row_start)
    np.testing.assert_array_equal(a.edge_dst, b.edge_dst)
    if b.edge_data is None:
        assert a.edge_data is None
    else:
        np.testing.assert_array_equal(a.edge_data, b.edge_data)


def test_host_api_matches_device_api(gft, orc, engine):
    g = gft.CSRGraph.road(128, seed=4)
    dg = g.copy_to_gpu()
    out = np.empty(g.nnodes, dtype=np.int32)
    par = np.empty(g.nnodes, dtype=np.uint32)
    engine.sssp_host(dg, 5, out, parent=par)
    np.testing.assert_array_equal(out, orc.sssp(g.row_start, g.edge_dst, g.edge_data, 5))
    assert orc.check_tree(g.row_start, g.edge_dst, g.edge_data, 5, out, par) == 0
    engine.bfs_host(dg, 5, out, parent=par)
    np.testing.assert_array_equal(out, orc.bfs(g.row_start, g.edge_dst, 5))
    assert orc.check_tree(g.row_start, g.edge_dst, None, 5, out, par) == 0


@pytest.mark.parametrize("app", ["bfs", "sssp"])
def test_host_many_rows_equal_single_queries(gft, orc, engine, app):
    """The many-query host calls copy each query's results back while the
    next query runs, through two device buffers: every row equals the oracle
    (and so the single-query host call), in pinned and pageable memory, for
    five sources (both buffers reused), on the grid and on one CTA; no
    sources is a no-op, and a bad source fails before anything runs."""
    import torch

    for g in (gft.CSRGraph.road(700, seed=6), gft.CSRGraph.road(100, seed=6)):
        dg = g.copy_to_gpu()
        srcs = g.pick_sources(21, 5)
        want = [orc.sssp(g.row_start, g.edge_dst, g.edge_data, s) if app == "sssp" else
                orc.bfs(g.row_start, g.edge_dst, s) for s in srcs]
        run = engine.sssp_host_many if app == "sssp" else engine.bfs_host_many
        pinned = torch.empty((len(srcs), g.nnodes), dtype=torch.int32, pin_memory=True).numpy()
        for out in (pinned, np.empty((len(srcs), g.nnodes), dtype=np.int32)):
            out.fill(-7)
            st = run(dg, srcs, out)
            assert len(st) == len(srcs)
            for i in range(len(srcs)):
                np.testing.assert_array_equal(out[i], want[i])
                assert st[i]["levels"] > 0 and st[i]["kernel_ms"] > 0
        assert run(dg, [], pinned[:0]) == []
        pinned.fill(-7)
        with pytest.raises(gft.GftError, match="INVALID_ARG"):
            run(dg, [srcs[0], g.nnodes], pinned)
        assert (pinned == -7).all()


def test_barrier_timeout_is_reported_and_engine_recovers(gft, orc, engine):
    """One CTA never arrives at the first grid barrier (test hook); the other
    CTAs' bounded waits expire, the call returns GFT_ERR_TIMEOUT and the
    context stays usable."""
    g = gft.CSRGraph.grid(64, 64)
    dg = g.copy_to_gpu()
    with pytest.raises(gft.GftError) as ei:
        engine.bfs(dg, 0, tune=gft.Tune(timeout_ms=200, test_skip_block=1))
    assert ei.value.status_name == "GFT_ERR_TIMEOUT"
    with pytest.raises(gft.GftError) as ei:
        engine.sssp(dg, 0, tune=gft.Tune(timeout_ms=200, test_skip_block=0))
    assert ei.value.status_name == "GFT_ERR_TIMEOUT"
    r = engine.bfs(dg, 0)
    np.testing.assert_array_equal(r["out"].cpu().numpy(), orc.bfs(g.row_start, g.edge_dst, 0))


def test_queue_tile_must_be_built(gft, engine):
    """Queue tiles are 64, 128 or 256 entries a warp; SSSP at 1024 threads
    takes at most 128 (its near and far buffers share 48 KB of static
    shared memory).  Anything else is GFT_ERR_INVALID_ARG, not a launch."""
    g = gft.CSRGraph.rmat(12, 8, seed=3, max_weight=255)
    dg = g.copy_to_gpu()
    for app, tune in (("bfs", dict(queue_tile=96)), ("sssp", dict(block_threads=1024, queue_tile=256)),
                      ("sssp", dict(queue_tile=512))):
        t = gft.Tune(max_blocks=1 << 30, **tune)
        with pytest.raises(gft.GftError) as ei:
            engine.sssp(dg, 0, tune=t) if app == "sssp" else engine.bfs(dg, 0, tune=t)
        assert ei.value.status_name == "GFT_ERR_INVALID_ARG"
    ok = engine.sssp(dg, 0, tune=gft.Tune(block_threads=1024, queue_tile=128, max_blocks=1 << 30))
    assert ok["out"].cpu().numpy()[0] == 0


def test_invalid_arguments(gft, engine):
    g = gft.CSRGraph.grid(8, 8)
    dg = g.copy_to_gpu()
    with pytest.raises(gft.GftError, match="INVALID_ARG"):
        engine.bfs(dg, 64)
    with pytest.raises(gft.GftError, match="INVALID_ARG"):
        engine.sssp(dg, 0, delta=0)
    with pytest.raises(gft.GftError, match="INVALID_ARG"):
        engine.bfs(dg, 0, tune=gft.Tune(block_threads=300))


@pytest.mark.parametrize("tune", TUNES, ids=TUNE_IDS)
def test_direction_optimising_bfs(gft, orc, engine, tune):
    """On a graph marked symmetric, BFS runs bottom-up levels when the
    frontier is large: levels equal the oracle's and the top-down-only run's,
    parents form a valid BFS tree, and far fewer edges are examined."""
    g = gft.CSRGraph.rmat(17, 16, seed=11)
    assert g.symmetric
    dg = g.copy_to_gpu()
    assert dg.symmetric
    for src in g.pick_sources(4, 3):
        want = orc.bfs(g.row_start, g.edge_dst, src)
        got, par, r = _run_bfs(gft, engine, dg, src, tune)
        np.testing.assert_array_equal(got, want)
        assert orc.check_tree(g.row_start, g.edge_dst, None, src, got, par) == 0
        td, _, r_td = _run_bfs(gft, engine, dg, src, {**tune, "direction": 1})
        np.testing.assert_array_equal(td, want)
        assert r["edges_scanned"] < r_td["edges_scanned"] / 2


def test_direction_optimising_needs_the_symmetry_mark(gft, orc, engine):
    """A directed graph is never traversed bottom-up: an unmarked upload stays
    top-down, and the mark is the caller's to set."""
    rs = np.array([0, 1, 2, 3, 3], dtype=np.uint32)  # 0 -> 1 -> 2 -> 3, one way
    dst = np.array([1, 2, 3], dtype=np.uint32)
    g = gft.CSRGraph(rs, dst, None)
    assert not g.symmetric
    dg = g.copy_to_gpu()
    assert not dg.symmetric
    for src in range(4):
        got, par, _ = _run_bfs(gft, engine, dg, src)
        np.testing.assert_array_equal(got, orc.bfs(rs, dst, src))
    dg.symmetric = True
    assert dg.symmetric


def test_grid_and_road_bfs_with_static_chunks(gft, orc, engine):
    """Low-degree graphs split large frontiers into one static chunk per
    warp; levels and parents stay exact."""
    for g in (gft.CSRGraph.grid(700, 700, 0, 1), gft.CSRGraph.road(600, seed=4)):
        dg = g.copy_to_gpu()
        for src in g.pick_sources(9, 2):
            got, par, _ = _run_bfs(gft, engine, dg, src)
            np.testing.assert_array_equal(got, orc.bfs(g.row_start, g.edge_dst, src))
            assert orc.check_tree(g.row_start, g.edge_dst, None, src, got, par) == 0


def test_direction_optimising_on_a_uniform_low_diameter_graph(gft, orc, engine):
    """A random graph of small, even degree takes the uniform-degree path of
    the direction switch (no degree loads) and still runs bottom-up."""
    rng = np.random.default_rng(5)
    n, m = 200_000, 800_000
    u = rng.integers(0, n, m, dtype=np.int64)
    v = rng.integers(0, n, m, dtype=np.int64)
    keep = u != v
    a = np.concatenate([u[keep], v[keep]])
    b = np.concatenate([v[keep], u[keep]])
    key = np.unique(a * n + b)
    src_of, dst = (key // n).astype(np.uint32), (key % n).astype(np.uint32)
    rs = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum(np.bincount(src_of, minlength=n), out=rs[1:])
    g = gft.CSRGraph(rs, dst, None)
    assert int(np.diff(rs.astype(np.int64)).max()) <= 32
    dg = g.copy_to_gpu()
    dg.symmetric = True
    for src in g.pick_sources(3, 2):
        want = orc.bfs(rs, dst, src)
        got, par, r = _run_bfs(gft, engine, dg, src)
        np.testing.assert_array_equal(got, want)
        assert orc.check_tree(rs, dst, None, src, got, par) == 0
        _, _, r_td = _run_bfs(gft, engine, dg, src, {"direction": 1})
        assert r["edges_scanned"] < r_td["edges_scanned"]
