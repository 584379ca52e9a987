"""Bodies across GPUs: one process per GPU, each stepping its own share.

Scenes never exchange forces, so a batch or a request population shards
across ranks with no collective on the data path (the reference runs one
ExplicitLoop per process and has no multi-GPU path at all; explicitloop.py:
72-85).  This module holds the host-side pieces:

* ``partition(weights, world)`` -- a deterministic split of scenes over ranks
  balanced by weight (element count): longest-processing-time first, ties to
  the lower index and the lower rank, each share returned in ascending scene
  order so a rank's packed world keeps the population's order;
* ``aggregate(work, ms)`` -- the whole-job figures of a timed region: total
  work summed over ranks, time as the maximum over ranks (the slowest rank
  finishes the job), through ``torch.distributed`` when a process group is
  up, else the local values.
"""

from __future__ import annotations

import heapq


def partition(weights, world: int) -> list[list[int]]:
    """Split scene indices over ``world`` ranks, balancing the summed weight."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(s) for s in shares]


def share(weights, rank: int, world: int) -> list[int]:
    """The scene indices rank ``rank`` steps."""
    return partition(weights, world)[rank]


def aggregate(work: float, ms: float):
    """(total work over ranks, max time over ranks) of one timed region."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(work), float(ms)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    w = torch.tensor([float(work)], dtype=torch.float64, device=dev)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(w.item()), float(t.item())
