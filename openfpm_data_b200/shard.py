"""Multi-GPU placement of independent work: one process per GPU, no
collective on the data path.

A single sparse grid runs as replicas (one per rank).  Batched grids and
served requests are independent units, so ranks split them without any
exchange: grids dealt by active points, requests round-robin by request id.
The only collectives are host-side timing reductions (max over ranks) and
gathers of per-rank summaries, over whatever torch.distributed process group
is set up (NCCL on GPUs, gloo on CPUs).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [lo, hi) share of n units for `rank` (sizes differ by at most one)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    return n * rank // world, n * (rank + 1) // world


def shard_weighted(weights: Sequence[float], rank: int, world: int) -> List[int]:
    """Indices of the units given to `rank` when units with the given weights
    (e.g. active points of a grid) are dealt largest-first to the currently
    lightest rank: every rank computes the same assignment without talking."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0.0] * world
    mine: List[int] = []
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += weights[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


def shard_requests(reqs, rank: int, world: int):
    """Requests of `rank`: round-robin by request id."""
    return [r for r in reqs if r.rid % world == rank]


def max_over_ranks(x: float) -> float:
    """Max of a host value over the default process group (x itself when none)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    dev = "cpu"
    if dist.get_backend() == "nccl":
        dev = f"cuda:{torch.cuda.current_device()}"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
