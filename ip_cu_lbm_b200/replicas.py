"""Replica orchestration for several GPUs of one node.

The per-step path has no exchange step: each rank advances its own
independent simulation (one process per GPU, launched by torchrun), so no
collective touches simulation data. torch.distributed carries only the
plumbing: a barrier around the timed region and a max over ranks of the
elapsed time. NCCL on GPUs; gloo serves the same calls on CPU (tests).
"""
from __future__ import annotations

import datetime
import os


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


class Replicas:
    def __init__(self, backend="nccl", timeout_s=120):
        self.rank, self.world = env_int("RANK", 0), env_int("WORLD_SIZE", 1)
        self.local = env_int("LOCAL_RANK", 0)
        self.backend = backend
        self.dist = None
        if backend == "nccl":
            import torch

            torch.cuda.set_device(self.local)
        if self.world > 1:
            import torch
            import torch.distributed as dist

            kw = {}
            if backend == "nccl":
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def barrier(self):
        """Device synchronize, barrier, synchronize (the timing bracket)."""
        if self.backend == "nccl":
            import torch

            torch.cuda.synchronize()
        if self.dist is not None:
            self.dist.barrier()
        if self.backend == "nccl":
            import torch

            torch.cuda.synchronize()

    def max(self, v: float) -> float:
        if self.dist is None:
            return float(v)
        import torch

        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def aggregate(self, units_per_rank: float, seconds_max: float) -> float:
        """Whole-job throughput: all ranks' units over the slowest rank's time."""
        return self.world * units_per_rank / seconds_max

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
