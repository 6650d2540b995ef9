"""Host-side plumbing for one process per GPU.

Frame pairs are independent, so the data path needs no collective: pairs are assigned to
ranks up front (balanced by cost for uneven batches) and every rank runs its own.  The
collectives here are the bookkeeping around that — the max-over-ranks step time, a gather
of per-pair metrics at the end — and the one real exchange of the learned warm start's
data-parallel training: averaging the flat gradient vector before the optimizer step.
All functions take the default torch.distributed group and work with any backend (NCCL on
GPUs, gloo on CPU ranks).
"""
from __future__ import annotations

import heapq

__all__ = ["pair_cost", "shard_by_cost", "shard_range", "max_over_ranks", "gather_objects", "average_gradients"]

# relative cost per pixel of each method's pyramid pipeline (estimates; only the ordering
# and rough ratios matter for balancing)
METHOD_WEIGHT = {"hs": 1.0, "lk": 2.5, "fb": 1.2, "ls": 2.0}


def pair_cost(size: int, method: str) -> float:
    return float(size) * float(size) * METHOD_WEIGHT.get(method, 1.0)


def shard_range(n: int, rank: int, world: int) -> range:
    """Contiguous share of n equal-cost items for `rank` (sizes differ by at most one)."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def shard_by_cost(costs, world: int):
    """Longest-processing-time assignment: items in decreasing cost, each to the currently
    lightest rank.  Returns one sorted index list per rank; every index appears once."""
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(x) for x in out]


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks (the job's step time is its slowest rank's)."""
    import torch
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_objects(obj):
    """Every rank's object, in rank order, on every rank."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def average_gradients(grads):
    """In-place mean of a flat gradient tensor over the ranks (one all-reduce)."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return grads
    dist.all_reduce(grads, op=dist.ReduceOp.SUM)
    grads.div_(dist.get_world_size())
    return grads
