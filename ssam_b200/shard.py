"""One process per GPU: rank plumbing for runs over several GPUs.

The stencil path shards by independent units -- whole grids, batches of
grids, batches of Poisson right-hand sides -- so ranks exchange nothing on
the data path.  What they share is the clock: every timed region is
bracketed by barriers and the reported time is the maximum over ranks (a
one-double all-reduce outside the data path).  torchrun (or any launcher
that sets RANK / WORLD_SIZE / LOCAL_RANK / MASTER_ADDR / MASTER_PORT) starts
the processes; NCCL is the backend on GPUs, gloo on the CPU (tests).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    rank: int
    world: int
    local: int


def ranks() -> Ranks:
    """This process's rank, the world size and its local rank (GPU index)."""
    return Ranks(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                 int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0, device=None) -> Ranks:
    """Join the process group when there is more than one rank.  The short
    timeout makes ranks that wait for a missing peer fail instead of hang."""
    import torch.distributed as dist
    r = ranks()
    if r.world > 1 and not dist.is_initialized():
        kw = {"device_id": device} if backend == "nccl" and device is not None else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return r


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (the time of the slowest rank)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def partition(n_units: int, rank: int, world: int) -> range:
    """Contiguous share of n_units independent units for `rank` (sizes differ
    by at most one), for runs that split a fixed amount of work."""
    base, extra = divmod(n_units, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def weak_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job rate when every rank processes the same amount of work and
    the job takes as long as its slowest rank."""
    return units_per_rank * world / seconds_max


def finish() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
