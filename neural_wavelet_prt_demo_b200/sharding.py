"""Host-side work partitioning for several GPUs (one process per GPU).

The relight path needs no collective on its data path: pixels are independent given the
resident weights and env tables, and requests are independent.  Ranks therefore split
*work*, never data.  This module holds the pure partitioning logic plus the only
collective the bench uses (a max over ranks of the elapsed time).

* ``row_band``       -- contiguous rows of one frame for one rank (a large frame split
  across GPUs; each rank relights its band from its own copy of the G-buffer rows).
* ``assign_requests``-- requests to ranks, balanced by estimated cost W*H*K (longest
  processing time first, ties by request index, so every rank computes the same plan).
* ``assign_online``  -- the same balance for a stream, decided in arrival order from the
  estimated backlog of every rank; large requests are split into row bands across ranks.
* ``max_over_ranks`` -- torch.distributed all-reduce MAX (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq
from typing import List, Optional, Sequence, Tuple


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


def assign_online(arrivals: Sequence[float], costs: Sequence[int], world: int, evals_per_s: float,
                  split_min_evals: Optional[int] = None, heights: Optional[Sequence[int]] = None
                  ) -> List[Tuple[int, bool]]:
    """Placement of a request stream on ranks, decided request by request in arrival order.

    Every rank keeps the same estimate of each rank's backlog (draining at `evals_per_s`),
    so every rank computes the same plan without communicating.  A request goes to the rank
    that would start it first (lowest rank on ties).  A request of at least
    `split_min_evals` evaluations whose frame has at least `world` rows is split into one
    row band per rank (``row_band``); each band adds its share to its rank's backlog, and the
    request is owned (its bands gathered and its latency reported) by the rank that would
    have started it first.  Returns (owner, split) per request."""
    if world < 1 or evals_per_s <= 0:
        raise ValueError("world must be >= 1 and evals_per_s > 0")
    free = [0.0] * world
    out: List[Tuple[int, bool]] = []
    for i, (a, c) in enumerate(zip(arrivals, costs)):
        a = float(a)
        starts = [max(f, a) for f in free]
        owner = min(range(world), key=lambda r: (starts[r], r))
        h = heights[i] if heights is not None else world
        split = world > 1 and split_min_evals is not None and int(c) >= split_min_evals and h >= world
        if split:
            for r in range(world):
                b, e = row_band(h, r, world)
                free[r] = starts[r] + int(c) * (e - b) / h / evals_per_s
        else:
            free[owner] = starts[owner] + int(c) / evals_per_s
        out.append((owner, split))
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
