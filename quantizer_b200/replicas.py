"""Replica bookkeeping of runs over several GPUs of one node.

A leapfrog step of one simulation has no exchange step that this library
distributes, so a multi-GPU run is N independent replicas, one process per GPU
(launched by torch.distributed.run): each rank steps its own simulation (its own
seed), no data-path collective runs, and the only collective is the reduction of
the timings: the whole job's time is the slowest rank's, its throughput the
units all ranks processed over that time.
"""
from __future__ import annotations

import datetime
import os


def env() -> tuple[int, int, int]:
    """(world, rank, local rank) from the launcher's environment (1, 0, 0 alone)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0) -> None:
    """Joins the process group when there is more than one rank; a short timeout
    makes a rank that never arrives an error for the others."""
    import torch.distributed as dist
    world, _, _ = env()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def finish() -> None:
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()


def seed_for(rank: int, base: int = 1) -> int:
    """The initial-condition seed of a rank's replica."""
    return base + rank


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over the ranks (the value itself alone)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, steps: int, ms_max: float, world: int) -> float:
    """Units of all ranks per second of the slowest rank's time."""
    return world * units_per_rank * steps / (ms_max / 1e3)
