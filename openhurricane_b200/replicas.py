"""Replica bookkeeping for runs on several GPUs of one node.

Cells are independent within a chemistry step, so the path does not shard
over a collective: every rank integrates its own cells (its own replica of a
workload, or its own slice of a mesh) and the ranks meet only to agree on
timing. These helpers are that agreement, written against
torch.distributed so they run on NCCL between GPUs and on gloo in CPU tests.
"""
from __future__ import annotations

import os
from typing import List, Sequence, Tuple

import torch


def env_ranks() -> Tuple[int, int, int]:
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def cell_slice(ncells: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous [begin, end) cell range of `rank` when a mesh's cells are
    split over `world` ranks (sizes differ by at most one)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank / world size")
    base, extra = divmod(ncells, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def max_over_ranks(values: Sequence[float], device=None) -> List[float]:
    """Element-wise maximum over all ranks (identity without a process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def sum_over_ranks(values: Sequence[float], device=None) -> List[float]:
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu()]


def whole_job_rate(units_per_rank: Sequence[float], ms_max: float) -> float:
    """Throughput of the whole job: all ranks' units over the slowest rank's time."""
    return float(sum(units_per_rank)) / (ms_max * 1e-3)
