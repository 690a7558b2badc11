"""Batched queries (one CTA per query, CUDA-graph replay) give the same
results as single queries and as the CPU oracle."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mix(gft):
    graphs = [
        gft.CSRGraph.road(40, seed=11),
        gft.CSRGraph.road(150, seed=12),
        gft.CSRGraph.rmat(10, 8, seed=13, max_weight=255),
        gft.CSRGraph.rmat(13, 8, seed=14, max_weight=255),
        gft.CSRGraph.grid(1, 50, 0, 3),
        gft.CSRGraph.rmat(12, 16, seed=15),
    ]
    return graphs, [g.copy_to_gpu() for g in graphs]


@pytest.mark.parametrize("block,group,gmin", [(256, 0, 0), (512, 0, 0), (1024, 0, 0), (128, 1, 0),
                                              (512, 4, 2000), (256, 8, 1), (1024, 2, 5000)])
def test_batch_matches_oracle_and_replays(gft, orc, engine, block, group, gmin):
    """group > 1 with a small gmin puts large queries on CTA groups (phase 1
    of the batch kernel, cooperative launch); group 1 runs all on one CTA."""
    import torch

    hosts, devs = _mix(gft)
    queries, want = [], []
    for i, (h, d) in enumerate(zip(hosts, devs)):
        for k, src in enumerate(h.pick_sources(100 + i, 2)):
            app = "sssp" if (i + k) % 2 == 0 else "bfs"
            queries.append({"graph": d, "app": app, "src": src, "delta": [50, 1000, 20000][(i + k) % 3]})
            want.append(orc.sssp(h.row_start, h.edge_dst, h.edge_data, src) if app == "sssp"
                        else orc.bfs(h.row_start, h.edge_dst, src))
    b = gft.Batch(engine, queries, tune=gft.Tune(block_threads=block, group_blocks=group, group_min_nodes=gmin))
    for rep in range(2):  # CUDA-graph replay
        for q in b.queries:
            q["out"].fill_(-7)
        st = b.run()
        assert st["queries"] == len(queries)
        for q, w in zip(b.queries, want):
            assert q["status"] == 0
            np.testing.assert_array_equal(q["out"].cpu().numpy(), w)
    b.close()


def test_batch_set_source_and_bfs_parent(gft, orc, engine):
    import torch

    h = gft.CSRGraph.rmat(12, 8, seed=3)
    d = h.copy_to_gpu()
    par = torch.empty(h.nnodes, dtype=torch.int32, device="cuda")
    b = gft.Batch(engine, [{"graph": d, "app": "bfs", "src": 0, "parent": par}])
    for src in h.pick_sources(9, 3):
        b.set_source(0, src)
        b.run()
        got = b.queries[0]["out"].cpu().numpy()
        np.testing.assert_array_equal(got, orc.bfs(h.row_start, h.edge_dst, src))
        assert orc.check_tree(h.row_start, h.edge_dst, None, src, got, par.cpu().numpy().view(np.uint32)) == 0
    b.close()


def test_batch_same_as_single_query(gft, engine):
    h = gft.CSRGraph.road(300, seed=5)
    d = h.copy_to_gpu()
    srcs = h.pick_sources(5, 8)
    b = gft.Batch(engine, [{"graph": d, "app": "sssp", "src": s, "delta": 40000} for s in srcs])
    b.run()
    for q, s in zip(b.queries, srcs):
        single = engine.sssp(d, s, delta=40000)["out"]
        np.testing.assert_array_equal(q["out"].cpu().numpy(), single.cpu().numpy())
    b.close()


def test_batch_rejects_bad_queries(gft, engine):
    h = gft.CSRGraph.grid(4, 4)
    d = h.copy_to_gpu()
    with pytest.raises(gft.GftError):
        gft.Batch(engine, [{"graph": d, "app": "bfs", "src": 16}])
    with pytest.raises(gft.GftError):
        gft.Batch(engine, [{"graph": d, "app": "sssp", "src": 0, "delta": 0}])
    with pytest.raises(gft.GftError):
        gft.Batch(engine, [{"graph": d, "app": "bfs", "src": 0}], tune=gft.Tune(block_threads=100))
