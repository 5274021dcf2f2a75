"""Replica plumbing for one process per GPU.

The reconstruction path exchanges nothing between GPUs: each rank decodes its
own images (or serves its own request stream), and the only collectives are
the timing reductions of a benchmark -- the maximum of the ranks' times and
the sum of their pixels.  Ranks come from the torchrun environment (RANK,
LOCAL_RANK, WORLD_SIZE, MASTER_ADDR/PORT); NCCL on GPUs, gloo on CPU.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import List, Sequence, TypeVar

T = TypeVar("T")


@dataclass
class Replicas:
    world: int = 1
    rank: int = 0
    local: int = 0
    backend: str = ""

    def _tensor(self, value: float):
        import torch
        device = "cuda" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(value)], dtype=torch.float64, device=device)

    def max(self, value: float) -> float:
        """The maximum of `value` over ranks (every rank calls it)."""
        if self.world == 1:
            return float(value)
        import torch.distributed as dist
        t = self._tensor(value)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, value: float) -> float:
        """The sum of `value` over ranks (every rank calls it)."""
        if self.world == 1:
            return float(value)
        import torch.distributed as dist
        t = self._tensor(value)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def barrier(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def close(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            if dist.is_initialized():
                dist.destroy_process_group()


def init(backend: str | None = None, timeout_s: float = 120.0) -> Replicas:
    """Join the process group of a torchrun launch (a single replica when
    WORLD_SIZE is unset or 1)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    r = Replicas(world, rank, local, "")
    if world > 1:
        import torch
        import torch.distributed as dist
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
        r.backend = backend
    return r


def shard(items: Sequence[T], rank: int, world: int) -> List[T]:
    """The items of one rank when a fixed set is split over ranks (round
    robin, so that sizes mix evenly)."""
    return [it for k, it in enumerate(items) if k % world == rank]
