"""Bookkeeping of replica runs on N GPUs (one process per GPU, no collective on the
data path): timings are the maximum over ranks, throughput is the work of all
ranks divided by the slowest rank's time."""
from __future__ import annotations

import torch
import torch.distributed as dist


def world_size():
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def max_over_ranks(values, device=None):
    """Element-wise maximum over all ranks of a list of floats (identity on one rank)."""
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def whole_job_rate(world, steps_per_rank, max_ms):
    """Steps per second of the whole job: every rank ran steps_per_rank steps."""
    return world * steps_per_rank / (max_ms * 1e-3)
