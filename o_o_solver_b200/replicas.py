"""Replicas over the GPUs of one node. Neither the statics nor the modes path shards (the top separators of one model
hold most of its flops), so with N GPUs every rank runs its own copy of the workload, one process per GPU, and the
only collectives are a barrier and the slowest rank's time. The rank, world size and rendezvous come from the
environment torch.distributed.run sets (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_ADDR, MASTER_PORT)."""

from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0, device=None):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            kwargs = {"device_id": device} if backend == "nccl" and device is not None else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kwargs)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def slowest(self, seconds: float) -> float:
        """The largest of every rank's value (the job's time is its slowest replica's)."""
        if self.dist is None:
            return float(seconds)
        import torch

        on = self.device if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(seconds)], dtype=torch.float64, device=on)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def total(self, count: float) -> float:
        """The sum of every rank's value (the units all replicas processed)."""
        if self.dist is None:
            return float(count)
        import torch

        on = self.device if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(count)], dtype=torch.float64, device=on)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
