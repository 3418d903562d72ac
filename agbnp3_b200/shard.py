"""Multi-GPU layouts, one process per GPU.

Independent work per rank (the benchmark's layout): the unit of work is an
independent energy+gradient evaluation; every rank evaluates its own
conformation(s) (weak scaling) and ranks meet only to take the maximum of
their device times, so the whole-job throughput is
world * units_per_rank / max_rank_time.

One instance over all ranks (row sharding, `shard_instance`): every rank
holds the whole instance and evaluates its share of the pair-pass work
items; the partial sums are added over the ranks by NCCL inside each
evaluation (agbnp3_shard).
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


def shard_instance(inst, group=None, make_id=None):
    """Row-shard `inst` (an agbnp3_b200.Instance holding the same system on
    every rank) over the ranks of the torch.distributed process group:
    rank 0 makes the NCCL unique id (make_id, default
    agbnp3_b200.shard_unique_id), every rank receives it over the group
    (any backend) and joins the communicator as its own rank.  Collective:
    every rank of the group calls it.  Returns (rank, world)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if make_id is None:
        from agbnp3_b200 import shard_unique_id as make_id
    box = [make_id() if rank == 0 else None]
    dist.broadcast_object_list(box, src=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
    inst.shard(rank, world, box[0])
    return rank, world
