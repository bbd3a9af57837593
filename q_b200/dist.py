"""Multi-GPU plumbing: one process per GPU, whole systems per rank.

The MD systems of a campaign (lambda windows, replicas, spheres) are
independent, so ranks share no per-step data: each rank steps its own systems
and only timing and end-of-run summaries cross ranks.
"""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> list[int]:
    """Indices of the items owned by `rank` (round robin, balanced to +-1)."""
    return list(range(rank, n_items, world))


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank float over the process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
