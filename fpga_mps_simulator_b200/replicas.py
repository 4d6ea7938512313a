"""Replica plumbing for runs on several GPUs of one node.

The two-site update has no exchange step, so N GPUs run N independent
replicas (one process per GPU, launched by ``torch.distributed.run``): each
rank advances its own circuits (seed + rank), timing is the maximum over
ranks, and the whole-job throughput is world * units / max seconds.  The
only collectives are the barrier around the timed region and the MAX
reduction of the timings -- no collective on the data path.
"""
from __future__ import annotations

import os
from datetime import timedelta
from typing import Optional

import torch
import torch.distributed as dist

__all__ = ["Replicas"]


class Replicas:
    """Rank bookkeeping from the torchrun environment (RANK, WORLD_SIZE, LOCAL_RANK)."""

    def __init__(self, backend: Optional[str] = None, device: Optional[torch.device] = None,
                 timeout_s: float = 300.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        self.device = device if device is not None else (
            torch.device("cuda", self.local_rank) if self.backend == "nccl" else torch.device("cpu"))
        self._own = False
        if self.world > 1 and not dist.is_initialized():
            kw = {"timeout": timedelta(seconds=timeout_s)}
            if self.backend == "nccl":
                kw["device_id"] = self.device
            dist.init_process_group(self.backend, **kw)
            self._own = True

    def seed(self, base: int) -> int:
        """Each replica's own seed."""
        return int(base) + self.rank

    def barrier(self) -> None:
        if self.world > 1:
            dist.barrier()

    def max(self, x: float) -> float:
        """Maximum of a per-rank float over all ranks (the job's timing)."""
        if self.world == 1:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, units_per_rank: float, seconds: float) -> float:
        """Whole-job units per second: every rank processed units_per_rank in at most max(seconds)."""
        return self.world * float(units_per_rank) / self.max(seconds)

    def close(self) -> None:
        if self._own and dist.is_initialized():
            dist.barrier()
            dist.destroy_process_group()
            self._own = False
