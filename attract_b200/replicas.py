"""Replica plumbing for running the minimiser on N GPUs of one node.

Poses are independent, so N GPUs run N replicas of a workload (one process
per GPU, launched by torchrun) with no collective on the data path: the only
communication is a barrier around timed regions and the max over ranks of a
device-measured time.  The process group uses NCCL on GPUs and gloo on CPU
(the multi-process tests).
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta

import torch
import torch.distributed as dist


@dataclass
class Ranks:
    rank: int
    world: int
    local: int
    device: torch.device

    @property
    def leader(self) -> bool:
        return self.rank == 0


def init(backend: str | None = None, timeout_s: float = 300.0) -> Ranks:
    """Read RANK / WORLD_SIZE / LOCAL_RANK (torchrun), pick this rank's device
    and, for more than one rank, join the process group (a short timeout, so
    that ranks waiting on a dead peer end with an error)."""
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
        device = torch.device("cuda", local)
    else:
        device = torch.device("cpu")
    if world > 1 and not dist.is_initialized():
        kw = dict(timeout=timedelta(seconds=timeout_s))
        if backend == "nccl":
            kw["device_id"] = device
        dist.init_process_group(backend, **kw)
    return Ranks(rank, world, local, device)


def barrier(r: Ranks):
    if r.world > 1:
        dist.barrier()


def max_over_ranks(r: Ranks, value: float) -> float:
    """The largest ``value`` over all ranks (every rank gets it)."""
    if r.world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=r.device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def finish(r: Ranks):
    if r.world > 1 and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
