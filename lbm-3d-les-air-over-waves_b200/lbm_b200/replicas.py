"""Replicas across GPUs: one independent domain per rank, no data-path
collective.

The step does not shard here (each solve runs on one GPU), so a
multi-GPU run is N independent replicas: each rank advances its own domain
(seed offset by the rank), and the only collectives are a barrier around the
timed region and a max of the ranks' timings.  Launched one process per GPU
by torch.distributed.run; the same code runs with the gloo backend on CPU
for tests.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str | None = None, timeout_s: float = 300.0):
        import torch

        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        self.backend = backend
        if backend == "nccl":
            torch.cuda.set_device(self.local)
            self.device = torch.device("cuda", self.local)
        else:
            self.device = torch.device("cpu")
        if self.world > 1:
            import torch.distributed as dist

            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl":
                kw["device_id"] = self.device
            dist.init_process_group(backend, **kw)
            self.dist = dist

    def seed(self, base: int) -> int:
        """Seed of this rank's replica."""
        return base + self.rank

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, values):
        """Element-wise max over ranks (timings: the job is as slow as its slowest rank)."""
        import torch

        t = torch.tensor(list(values), dtype=torch.float64, device=self.device)
        if self.dist is not None:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return t.tolist()

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
