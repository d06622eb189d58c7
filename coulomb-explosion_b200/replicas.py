"""Replica sharding for several GPUs (one process per GPU).

Explosions are independent, so the N-GPU form of the path has no data exchange:
rank r of W integrates sims [r*S, (r+1)*S) of one counter-based Philox
population (sim s is the same geometry on every rank and in a one-GPU run), and
the only collective is the max over ranks of each rank's device time.
"""
from __future__ import annotations


def shard(rank: int, world: int, sims_per_rank: int) -> tuple[int, int]:
    """(first_sim, count) of this rank's slice of the population."""
    if not (0 <= rank < world) or sims_per_rank < 0:
        raise ValueError("rank must be in [0, world) and sims_per_rank >= 0")
    return rank * sims_per_rank, sims_per_rank


def max_over_ranks(value: float, device="cpu") -> float:
    """Max of a per-rank scalar over the process group (identity without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, sims_per_rank: int, steps: int, max_ms: float) -> float:
    """Whole-job explosions/s: every rank's sims over the slowest rank's time."""
    return world * sims_per_rank * steps / (max_ms / 1e3)
