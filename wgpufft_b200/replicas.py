"""Replica plumbing for multi-GPU runs of independent work (batches, mixed
lines, serving requests): one process per GPU, no data-path collective; the
only communication is the timing barrier and the max over ranks.  NCCL on
GPUs, gloo on CPU (the multi-process tests)."""
from __future__ import annotations

import os
from datetime import timedelta


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
