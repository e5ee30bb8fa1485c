"""Replicas on several GPUs of one node: one process per GPU, independent simulations, no collective on the data path.

The reference scales out with a Slurm job array of one-GPU jobs (slurm/submit_all.sh:21,36-38): instances share
nothing. Here the ranks of one torchrun job play those jobs: each runs its own lattices (its share of a sweep or a
request stream) and the only collectives are the timing ones — a barrier around the timed region and the maximum
of the ranks' durations, so that a whole-job rate is (units all ranks processed) / (slowest rank's time).
"""
import os
from datetime import timedelta

import torch
import torch.distributed as dist


class Replicas:
    """Rank / world from the torchrun environment; backend "nccl" on GPUs, "gloo" for host-only use."""

    def __init__(self, backend="nccl", timeout_s=120, device=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device if device is not None else torch.device("cpu")
        self.owned = False
        if self.world > 1 and not dist.is_initialized():
            kw = {"device_id": self.device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            self.owned = True

    def barrier(self):
        if self.world > 1:
            dist.barrier()

    def max(self, x):
        """The largest value over ranks (a duration: the whole job ends when its slowest rank does)."""
        if self.world == 1:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if self.world == 1:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def rate(self, units, seconds):
        """Whole-job rate: the units every rank processed over the slowest rank's time."""
        return self.sum(units) / max(self.max(seconds), 1e-300)

    def gather(self, obj):
        """Every rank's `obj` (a picklable host value), in rank order, on every rank."""
        if self.world == 1:
            return [obj]
        out = [None] * self.world
        dist.all_gather_object(out, obj)
        return out

    def share(self, items):
        """This rank's share of a list of independent items (round robin, so sizes spread evenly)."""
        return list(items)[self.rank::self.world]

    def close(self):
        if self.owned and dist.is_initialized():
            dist.destroy_process_group()
            self.owned = False
