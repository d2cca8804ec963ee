"""Replica serving across GPUs: one process per GPU, every rank holding its own
copy of the resident scenes and serving its own seeded job stream (weak
scaling).  The data path has no collective; torch.distributed only reduces the
measurements: the slowest rank's time, the sum of rays, and every job latency
gathered on rank 0 for the global percentiles."""
from __future__ import annotations

import datetime
import os
from typing import List

import numpy as np

from . import scenes


def env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def rank_stream(rank: int, n_jobs: int = 512, seed: int = 4) -> List[scenes.Job]:
    """The job stream a rank serves: the seeded stream with seed + rank."""
    return scenes.job_stream(n_jobs, seed=seed + rank)


class Group:
    """Reductions of per-rank measurements (NCCL on GPUs, gloo on CPU)."""

    def __init__(self, world: int, backend: str = "nccl", timeout_s: int = 120):
        self.world = world
        self.device = "cpu"
        if world > 1:
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            if not dist.is_initialized():
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
            self.device = "cuda" if backend == "nccl" else "cpu"

    def _reduce(self, x: float, op) -> float:
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return x if self.world == 1 else self._reduce(x, self.dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return x if self.world == 1 else self._reduce(x, self.dist.ReduceOp.SUM)

    def gather(self, values: List[float]) -> List[float]:
        """All ranks' values, concatenated in rank order (on every rank)."""
        if self.world == 1:
            return list(values)
        import torch
        n = torch.tensor([len(values)], dtype=torch.int64, device=self.device)
        sizes = [torch.zeros_like(n) for _ in range(self.world)]
        self.dist.all_gather(sizes, n)
        m = int(max(int(s.item()) for s in sizes))
        buf = torch.zeros(m, dtype=torch.float64, device=self.device)
        buf[:len(values)] = torch.tensor(values, dtype=torch.float64)
        outs = [torch.zeros_like(buf) for _ in range(self.world)]
        self.dist.all_gather(outs, buf)
        res = []
        for s, o in zip(sizes, outs):
            res += o[:int(s.item())].cpu().tolist()
        return res

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def close(self):
        if self.world > 1 and self.dist.is_initialized():
            self.dist.destroy_process_group()


def percentile(values, q):
    return float(np.percentile(np.asarray(values), q)) if len(values) else None
