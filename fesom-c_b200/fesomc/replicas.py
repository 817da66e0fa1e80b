"""Multi-GPU runs of the time step: replicas only.

The whole mesh lives on one GPU, so the time step does not shard and has no
exchange step.  Running on N GPUs means N independent meshes, one process per
GPU (launched by torchrun), joined only for a barrier around the timed region
and the maximum of the per-rank times.  The whole-job rate is the units all
ranks processed divided by that maximum.
"""
import os
from datetime import timedelta


def dist_env():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """Process group of the replicas (NCCL on GPUs, gloo for CPU tests)."""

    def __init__(self, world_size, backend="nccl", timeout_s=120):
        self.ws = world_size
        self.dist = None
        self.device = "cuda" if backend == "nccl" else "cpu"
        if world_size > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x):
        """Maximum of a per-rank float over all ranks."""
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def whole_job_rate(units_per_step, steps, world_size, seconds):
    """Units all replicas processed per second of the slowest replica."""
    return units_per_step * steps * world_size / seconds
