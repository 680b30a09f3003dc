"""Replica execution across ranks.

A single graph's clustering does not shard (every sweep needs the global
cluster volumes and every neighbour's label), so multi-GPU runs are independent
replicas: one graph (or one seed of a trial set) per rank, no data-path
collective.  The only exchange is the final reduction of per-rank timings (max)
and, for trial sets, the selection of the best clustering (max objective), the
way app/cluster_main.cpp:189-204 keeps the best of its trials.
"""
from __future__ import annotations


def replica_seed(base_seed: int, rank: int) -> int:
    """Seed of rank `rank`'s replica (distinct, deterministic)."""
    return int(base_seed) + int(rank)


def max_over_ranks(values, device=None):
    """Element-wise max of a list of floats over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def best_trial(objective: float, device=None):
    """(rank holding the best objective, best objective); ties go to the lowest rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return 0, float(objective)
    world = dist.get_world_size()
    t = torch.zeros(world, dtype=torch.float64, device=device)
    t[dist.get_rank()] = objective
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    best = float(t.max())
    rank = int((t == best).nonzero()[0])
    return rank, best
