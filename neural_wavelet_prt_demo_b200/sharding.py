"""Host-side work partitioning for several GPUs (one process per GPU).

The relight path needs no collective on its data path: pixels are independent given the
resident weights and env tables, and requests are independent.  Ranks therefore split
*work*, never data.  This module holds the pure partitioning logic plus the only
collective the bench uses (a max over ranks of the elapsed time).

* ``row_band``       -- contiguous rows of one frame for one rank (a large frame split
  across GPUs; each rank relights its band from its own copy of the G-buffer rows).
* ``assign_requests``-- requests to ranks, balanced by estimated cost W*H*K (longest
  processing time first, ties by request index, so every rank computes the same plan).
* ``max_over_ranks`` -- torch.distributed all-reduce MAX (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence, Tuple


def row_band(height: int, rank: int, world: int) -> Tuple[int, int]:
    """Rows [begin, end) of a frame of `height` rows owned by `rank` (balanced to one row)."""
    if world < 1 or not (0 <= rank < world) or height < 0:
        raise ValueError("bad rank/world/height")
    base, extra = divmod(height, world)
    begin = rank * base + min(rank, extra)
    end = begin + base + (1 if rank < extra else 0)
    return begin, end


def request_cost(width: int, height: int, K: int) -> int:
    """Pixel*wavelet evaluations of one relight request (the work the MLP does)."""
    return int(width) * int(height) * int(K)


def assign_requests(costs: Sequence[int], world: int) -> List[List[int]]:
    """Partition request indices over `world` ranks, balancing the summed cost.

    Longest-processing-time-first greedy: requests sorted by cost descending (index
    ascending on ties) each go to the currently least-loaded rank (lowest rank on ties).
    Deterministic, so every rank derives the same plan without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(costs[i]), r))
    for lst in out:
        lst.sort()
    return out


def max_over_ranks(value: float, device=None) -> float:
    """Max of `value` over all ranks of the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
