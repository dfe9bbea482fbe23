"""Rank plumbing shared by the benchmark and the sharded assembly: one
process per GPU, ranks from the torchrun environment, timings reduced as the
maximum over ranks (a multi-rank step ends when its slowest rank ends)."""
from __future__ import annotations

import os


def rank_env() -> tuple:
    """(rank, world, local_rank) from RANK / WORLD_SIZE / LOCAL_RANK."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(values, device=None) -> list:
    """Element-wise maximum of a list of floats over all ranks (identity
    without an initialised process group). ``device`` is where the reduction
    tensor lives: a CUDA device for NCCL, None (CPU) for gloo."""
    import torch
    import torch.distributed as dist

    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def sum_over_ranks(values, device=None) -> list:
    """Element-wise sum of a list of floats over all ranks."""
    import torch
    import torch.distributed as dist

    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.cpu()]
