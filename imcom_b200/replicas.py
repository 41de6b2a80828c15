"""Host-side logic of multi-GPU runs: one process per GPU, no data-path
collective.

The solve path of one system does not shard before its eigendecomposition;
independent systems (replicas of the n=4096 workload, or the patches of a
batched run) go to different GPUs whole.  What the ranks share is host
bookkeeping: which patches each rank solves, and the job's time, which is the
slowest rank's (a MAX reduction of device-timed seconds).

* ``shard_by_cost`` assigns items to ranks largest-cost first, each to the
  least-loaded rank (ties to the lower rank), so every rank computes the same
  partition from the same list without communicating.  The cost of a patch is
  n^3 (its eigendecomposition dominates).
* ``max_over_ranks`` reduces a float with MAX over the process group (any
  backend: NCCL on GPUs, gloo on CPU).
* ``job_rate`` is the whole-job throughput: all ranks' units over the slowest
  rank's time.
"""
from __future__ import annotations

import heapq


def shard_by_cost(costs, rank: int, world: int) -> list[int]:
    """Indices of the items that `rank` of `world` solves (ascending)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    mine = []
    for i in order:
        load, r = heapq.heappop(heap)
        if r == rank:
            mine.append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return sorted(mine)


def patch_cost(problem) -> float:
    """Relative solve cost of a patch: n^3 (the eigendecomposition)."""
    return float(problem.n) ** 3


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """MAX of `x` over the process group (`x` itself without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(total_units: float, slowest_seconds: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return total_units / slowest_seconds if slowest_seconds > 0 else 0.0


__all__ = ["shard_by_cost", "patch_cost", "max_over_ranks", "job_rate"]
