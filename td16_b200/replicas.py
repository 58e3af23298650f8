"""Replica bookkeeping for multi-GPU runs.

The search shards by instance: every rank searches its own seeded batch and
no data crosses between GPUs.  The only collective is host-side reporting:
the job time is the maximum over ranks and the counts are summed.
"""
from __future__ import annotations


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s batch; instance i of it uses splitmix64(seed ^ i)."""
    return int(seed) ^ (int(rank) << 40)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(values, dist=None, device=None):
    values = [float(v) for v in values]
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return values
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t)
    return [float(v) for v in t.tolist()]
