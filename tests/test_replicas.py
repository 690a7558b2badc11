"""Multi-rank host logic on CPU: two gloo ranks on 127.0.0.1."""

import os
import socket
import subprocess
import sys
import textwrap
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


WORKER = textwrap.dedent("""
    import json, os, sys
    sys.path.insert(0, sys.argv[1])
    from galoisgpu_b200.replicas import ReplicaGroup, shard
    g = ReplicaGroup(backend="gloo", timeout_s=60)
    items = list(range(10))
    mine = shard(items, g.rank, g.world)
    # rank r "processes" its items in (r + 1) seconds
    rate = g.throughput(len(mine), float(g.rank + 1))
    g.barrier()
    out = {"rank": g.rank, "world": g.world, "mine": mine, "rate": rate, "max": g.max(g.rank * 10.0),
           "sum": g.sum(1.0)}
    print(json.dumps(out), flush=True)
    g.close()
""")


def test_two_gloo_ranks(tmp_path):
    import json

    script = tmp_path / "w.py"
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script), str(ROOT)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    outs.sort(key=lambda d: d["rank"])
    assert outs[0]["mine"] == [0, 2, 4, 6, 8] and outs[1]["mine"] == [1, 3, 5, 7, 9]
    for d in outs:
        assert d["world"] == 2
        assert d["rate"] == 10 / 2.0  # all units over the slowest rank's time
        assert d["max"] == 10.0 and d["sum"] == 2.0


def test_single_process_is_identity():
    sys.path.insert(0, str(ROOT))
    from galoisgpu_b200.replicas import ReplicaGroup, shard

    g = ReplicaGroup()
    assert g.world == 1 and g.max(3.0) == 3.0 and g.sum(2.0) == 2.0
    assert g.throughput(10, 2.0) == 5.0
    g.barrier()
    assert shard(range(5), 0, 1) == [0, 1, 2, 3, 4]
