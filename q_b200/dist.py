"""Multi-GPU plumbing: one process per GPU, whole systems per rank.

The MD systems of a campaign (lambda windows, replicas, spheres) are
independent, so ranks share no per-step data: each rank steps its own systems
and only timing and end-of-run results cross ranks.  Systems are spread over
ranks by their cost (atoms x steps), so that uneven sphere sizes do not leave
one rank with the slowest share.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def shard(n_items: int, rank: int, world: int, costs: Sequence[float] | None = None) -> list[int]:
    """Indices of the items owned by `rank`.  Without costs: round robin,
    balanced to +-1 item.  With costs (e.g. atoms x steps per system): the
    longest-processing-time rule -- items in decreasing cost, each to the rank
    with the least cost so far (ties to the lower rank) -- which keeps the
    largest rank total within 4/3 of the optimum.  Every rank computes the same
    assignment from the same costs, with no communication; each rank's list
    is in ascending item order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    if costs is None:
        return list(range(rank, n_items, world))
    if len(costs) != n_items:
        raise ValueError("one cost per item")
    heap = [(0.0, r) for r in range(world)]
    owner = [0] * n_items
    for i in sorted(range(n_items), key=lambda i: (-float(costs[i]), i)):
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [i for i in range(n_items) if owner[i] == rank]


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


def gather_series(series: dict, device=None) -> dict:
    """The end-of-run exchange of a campaign: every rank holds the energy
    series of its own systems ({system index: 2-D float64 array}); every rank
    receives all of them.  One all-gather of the arrays' sizes and one of the
    padded data (NCCL over NVLink on GPUs, gloo on the host); without a
    process group the input is returned."""
    import numpy as np
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return dict(series)
    world = dist.get_world_size()
    keys = sorted(series)
    shapes = [series[k].shape for k in keys]
    meta = torch.tensor([len(keys)] + [v for k, sh in zip(keys, shapes) for v in (k, sh[0], sh[1])],
                        dtype=torch.int64, device=device)
    n = torch.tensor([meta.numel()], dtype=torch.int64, device=device)
    ns = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(ns, n)
    width = int(max(x.item() for x in ns))
    metas = [torch.zeros(width, dtype=torch.int64, device=device) for _ in range(world)]
    pad = torch.zeros(width, dtype=torch.int64, device=device)
    pad[:meta.numel()] = meta
    dist.all_gather(metas, pad)
    flat = np.concatenate([series[k].ravel() for k in keys]) if keys else np.zeros(0)
    sizes = [int(sum(m[2 + 3 * j].item() * m[3 + 3 * j].item() for j in range(int(m[0].item())))) for m in metas]
    buf = torch.zeros(max(sizes + [1]), dtype=torch.float64, device=device)
    buf[:flat.size] = torch.from_numpy(flat).to(buf.device)
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf)
    out = {}
    for m, b in zip(metas, bufs):
        data = b.cpu().numpy()
        off = 0
        for j in range(int(m[0].item())):
            k, r, c = (int(m[1 + 3 * j + q].item()) for q in range(3))
            out[k] = data[off:off + r * c].reshape(r, c).copy()
            off += r * c
    return out
