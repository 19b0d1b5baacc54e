"""Replica plumbing for multi-GPU runs: one process per GPU, independent
products (no collective on the data path), a barrier around timed regions
and the maximum over ranks of device times.

Products are independent requests and a ModUp inside one product would need
an all-to-all per switch, so multi-GPU throughput is request-level data
parallel: every rank holds its own keys and operands and runs its own
products; the process group only synchronises timing.
"""
from __future__ import annotations

import os
from datetime import timedelta


def dist_env():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """The process group of a replica run (NCCL on GPUs, gloo on CPU)."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0):
        import torch
        self.torch = torch
        self.world, self.rank, self.local = dist_env()
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self.dist = dist
        self.timeout = timedelta(seconds=timeout_s)
        self.device = (torch.device("cuda", self.local) if backend == "nccl"
                       else torch.device("cpu"))

    def sync_device(self):
        if self.device.type == "cuda":
            self.torch.cuda.synchronize()

    def barrier(self):
        """Device work drained, then every rank at the same point."""
        self.sync_device()
        if self.dist is not None:
            if self.backend == "gloo":
                # bounded: raises naming the ranks that did not arrive
                self.dist.monitored_barrier(timeout=self.timeout)
            else:
                self.dist.barrier()
        self.sync_device()

    def max_over_ranks(self, x: float) -> float:
        if self.dist is None:
            return float(x)
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, units_per_rank: float, seconds_per_rank: float) -> float:
        """Whole-job units per second: every rank's units over the slowest
        rank's time."""
        return self.world * units_per_rank / self.max_over_ranks(seconds_per_rank)

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
