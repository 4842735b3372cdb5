"""Multi-GPU placement of independent orbits (one process per GPU).

Orbits are independent (each species x met draw x right-hand side has its own
factors), so N GPUs run N disjoint shares of the work with no collective on
the data path; the only collectives are the timing barrier and the maximum
of the per-rank elapsed times.
"""
from __future__ import annotations

from typing import List


def orbits_for_rank(n_total: int, rank: int, world: int) -> List[int]:
    """Round-robin share of orbit indices 0..n_total-1 for one rank."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    return list(range(rank, n_total, world))


def met_draw_seed(base: int, rank: int, draw: int) -> int:
    """Seed of a rank's met draw (disjoint across ranks for any world size)."""
    return base + 1000 * (rank * 64 + draw)


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar over the default process group (or the value)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
