"""One process per GPU running independent replicas of the spectrometer.

Streams, channels and integrations are independent, so ranks exchange no
data: the process group carries only the barriers around the timed region
and the max-over-ranks of the measured time (the job's time is the slowest
rank's).  Rank, world size and rendezvous come from the torchrun
environment (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_ADDR, MASTER_PORT).
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _tensor(self, x: float):
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        return torch.tensor([x], dtype=torch.float64, device=dev)

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """Max of x over ranks (every rank gets it)."""
        if self.dist is None:
            return x
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, units_per_rank: float, seconds: float) -> float:
        """Whole-job rate: units of all ranks over the slowest rank's time."""
        return units_per_rank * self.world / self.max(seconds)

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
