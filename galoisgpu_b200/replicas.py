"""Multi-GPU plumbing for independent replicas.

Single BFS/SSSP queries do not shard without a per-level exchange of remote
frontier vertices, so multi-GPU runs use one process per GPU, each an
independent replica over its own copy of the graph; batched and served
queries are sharded across replicas.  No collective touches the data path:
torch.distributed (NCCL on GPUs, gloo on CPU) carries only the barrier that
brackets a timed region, the max-over-ranks of elapsed times and sums of
counters.
"""

from __future__ import annotations

import datetime
import os


def shard(items, rank: int, world: int) -> list:
    """Round-robin share of `items` owned by `rank`."""
    return list(items)[rank::world]


class ReplicaGroup:
    """Rank/world from the torchrun environment; a process group only when
    world > 1."""

    def __init__(self, backend: str | None = None, timeout_s: int = 300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = None
        if self.world > 1:
            import torch
            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = torch.device("cuda", self.local)
                kw["device_id"] = self.device
            else:
                self.device = torch.device("cpu")
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def _tensor(self, values, dtype):
        import torch

        return torch.tensor(values, dtype=dtype, device=self.device)

    def barrier(self) -> None:
        if self.dist:
            import torch

            t = self._tensor([0.0], torch.float64)
            self.dist.all_reduce(t)
            if t.is_cuda:
                torch.cuda.synchronize(t.device)

    def max(self, x: float) -> float:
        if not self.dist:
            return x
        import torch

        t = self._tensor([x], torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return x
        import torch

        t = self._tensor([x], torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def throughput(self, units_local: float, seconds_local: float) -> float:
        """Whole-job rate: all ranks' units over the slowest rank's time."""
        return self.sum(units_local) / self.max(seconds_local)

    def close(self) -> None:
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None
