"""Multi-GPU plumbing for independent work (batches of lines, serving
requests): one process per GPU, the lines partitioned across the ranks, no
data-path collective; the only communication is the timing barrier and the
max over ranks.  NCCL on GPUs, gloo on CPU (the multi-process tests)."""
from __future__ import annotations

import os
from datetime import timedelta

import numpy as np


def partition_lines(lengths, world: int):
    """Splits lines stored back to back into `world` contiguous runs of about
    equal points (HBM bytes and transform work both grow with the points),
    so that each rank owns one contiguous range of the buffers.  Returns a
    list of (first line, end line) per rank; every line belongs to exactly
    one rank, and a rank may own no line when there are fewer lines than
    ranks."""
    lengths = np.asarray(lengths, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be at least 1")
    n = len(lengths)
    if n == 0:
        return [(0, 0)] * world
    ends = np.cumsum(lengths)
    total = int(ends[-1])
    cuts = [0]
    for r in range(1, world):
        # first line whose end passes r/world of the points
        c = int(np.searchsorted(ends, total * r / world, side="left")) + 1
        cuts.append(min(max(c, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


class Replicas:
    def __init__(self, backend: str | None = None, timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            self.backend = backend
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            self._dist = dist

    def _device(self):
        import torch
        return torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, value: float) -> float:
        """Max of a per-rank value (times: the job is as slow as its slowest rank)."""
        if self._dist is None:
            return value
        import torch
        t = torch.tensor([value], dtype=torch.float64, device=self._device())
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, value: float) -> float:
        if self._dist is None:
            return value
        import torch
        t = torch.tensor([value], dtype=torch.float64, device=self._device())
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def aggregate_rate(self, units_per_rank: float, seconds: float) -> float:
        """Whole-job throughput: every rank's units over the slowest rank's time."""
        return self.sum(units_per_rank) / self.max(seconds)

    def close(self) -> None:
        if self._dist is not None:
            self.barrier()
            self._dist.destroy_process_group()
            self._dist = None
