"""Replica plumbing of the N-GPU benchmark: one process per GPU, each running
an independent solve (the path does not shard: pulse instances and requests
are independent), torch.distributed only for the barrier around the timed
region and for the maximum of the per-rank device times.

The launcher (torchrun) sets RANK, WORLD_SIZE and LOCAL_RANK; a plain run is
rank 0 of 1 and touches no process group.
"""
import datetime
import os


def dist_env():
    """(rank, world size, local rank) from the launcher's environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ReplicaGroup:
    """Process group of the replicas (backend "nccl" on GPUs, "gloo" on CPU).

    device: where the reduction tensors live ("cuda:<local>" or "cpu"). The
    timeout bounds every collective, so ranks that wait for a rank that died
    end with an error instead of hanging."""

    def __init__(self, backend="nccl", device="cpu", timeout_s=120):
        import torch

        self.torch = torch
        self.rank, self.world, self.local = dist_env()
        self.device = device
        self.active = self.world > 1
        if self.active:
            torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def barrier(self):
        if self.device.startswith("cuda"):
            self.torch.cuda.synchronize()
        if self.active:
            self.torch.distributed.barrier()

    def max(self, x):
        """Maximum of x over the ranks (x itself on a single rank)."""
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        if self.active:
            self.torch.distributed.all_reduce(t, op=self.torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.active:
            self.torch.distributed.destroy_process_group()
            self.active = False


def whole_job_rate(world, units_per_step, steps, max_seconds):
    """Units of all ranks per second: every rank processes units_per_step per
    step (weak scaling), timed by the slowest rank."""
    return world * units_per_step * steps / max_seconds
