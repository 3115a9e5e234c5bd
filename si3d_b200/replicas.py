"""Work placement across ranks: one process per GPU and no collective on the data path.

A single-basin workload runs as independent replicas: every rank advances its own copy of the
basin, and the only collective is the maximum over ranks of the device timings.  An ensemble of
independent basins is partitioned across ranks by estimated cost (wet 3-D cells x expected
solver work), longest job first onto the least-loaded rank, so each basin runs on exactly one
rank and ranks never exchange state.
"""
from __future__ import annotations

import heapq
from typing import Iterable, List, Sequence


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Greedy longest-processing-time split of basins (by cost) over `world` ranks.  Returns, per
    rank, the basin indices it owns in ascending order.  Deterministic: ties go to the lower rank
    and, among equal costs, to the lower basin index."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    owned: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        load, r = heapq.heappop(heap)
        owned[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(o) for o in owned]


def imbalance(costs: Sequence[float], parts: Iterable[Sequence[int]]) -> float:
    """max rank load / mean rank load of a partition."""
    loads = [sum(float(costs[i]) for i in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """The maximum of `x` over all ranks of the default process group (identity without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
