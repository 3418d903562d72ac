"""Multi-GPU layout of the benchmark: one process per GPU, independent
work per rank, no collective on the data path.

The unit of work is an independent energy+gradient evaluation.  Every rank
evaluates its own conformation(s) (weak scaling); ranks meet only to take
the maximum of their device times, so the whole-job throughput is
world * units_per_rank / max_rank_time.
"""
from __future__ import annotations


def rank_seed(base_seed: int, rank: int) -> int:
    """Seed of the conformation a rank evaluates (rank 0 uses the base
    seed, so a 1-GPU run measures the same system as rank 0 of N)."""
    return base_seed + rank


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Maximum of a per-rank float over all ranks (identity for world 1)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(units_per_rank: int, max_seconds: float, world: int) -> float:
    """Whole-job units per second."""
    return world * units_per_rank / max_seconds
