"""One process per GPU: the multi-rank host logic of the benchmark and of
batched sampling.

Chains and replicas are independent, so ranks share no data: each rank
builds its own systems from a rank-offset seed, runs them on its GPU, and
only the timing is combined — the slowest rank's time (max) and the units
of all ranks (sum).  The process group comes from the usual torchrun
environment (RANK, WORLD_SIZE, MASTER_ADDR/PORT); NCCL on GPUs, gloo where
the host logic is tested without one.
"""
from __future__ import annotations

import datetime
import os

import torch


def rank_info():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def rank_seed(base, rank):
    """Seed of rank `rank`'s systems: disjoint streams for every rank."""
    return int(base) + 1000 * int(rank)


def init(backend="nccl", timeout_s=120):
    """Process group with a short timeout, so a rank that dies ends the
    others' next collective with an error instead of a hang."""
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def reduce_timing(ms, units, device="cpu"):
    """(max over ranks of ms, sum over ranks of units).  Every rank must
    call it (same collective steps on every rank)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms), float(units)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())
