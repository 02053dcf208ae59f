"""Replica runs on several GPUs: one process per GPU, independent columns.

The hourly step has no exchange between cells (every array is per cell), so
N GPUs run N independent replicas with no data-path collective.  What the
ranks share is only the bookkeeping of a measurement: who they are, the seed
each replica's columns come from, a barrier around the timed region, and the
maximum of the timings over ranks (the job is as slow as its slowest rank).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class World:
    rank: int
    size: int
    local: int

    @property
    def multi(self) -> bool:
        return self.size > 1


def world_from_env() -> World:
    """Rank, world size and local rank as torchrun sets them (1 process by default)."""
    return World(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                 int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's columns: each replica advances its own cells."""
    return int(base) + int(rank)


def init(world: World, backend: str, device=None, timeout_s: int = 120):
    """Join the process group (short timeout, so ranks that wait on a dead peer fail)."""
    if not world.multi:
        return
    import torch.distributed as dist
    kw = dict(timeout=datetime.timedelta(seconds=timeout_s))
    if device is not None and backend == "nccl":
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)


def barrier(world: World):
    if world.multi:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world: World, values, device="cpu"):
    """Element-wise maximum over ranks of a list of floats (the job's timings)."""
    values = [float(v) for v in values]
    if not world.multi:
        return values
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def finish(world: World):
    if world.multi:
        import torch.distributed as dist
        dist.destroy_process_group()
