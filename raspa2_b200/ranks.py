"""One process per GPU: rank discovery, the placement of independent
systems and jobs on the GPUs, and the reductions a multi-GPU run needs.

Systems are independent, so the data path has no collective: every rank
builds and advances the systems placed on it. Placement is greedy
bin-packing by device-memory footprint (`place`), computed the same way on
every rank from the same list, so it needs no communication. The only
collectives combine results: the maximum of the ranks' device times and the
sum of their moves (max-over-ranks timing), and the per-job results gathered
on rank 0. The process group may be NCCL (GPUs) or gloo (CPU tests); the
calls are the same on every rank and in the same order.
"""
from __future__ import annotations

import os
from typing import List, Optional, Sequence, Tuple

# seeds of a rank's batch are spaced by a prime, so no two ranks share one
RANK_SEED_STRIDE = 7919


def rank_env() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def batch_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s batch: weak scaling, every rank its own systems."""
    return base + RANK_SEED_STRIDE * rank


def place(footprints: Sequence[int], work: Sequence[float], n_ranks: int, budget: Optional[float] = None,
          max_items: Optional[int] = None) -> List[List[int]]:
    """Greedy bin-packing of independent items (systems or jobs) over
    `n_ranks` GPUs: items in decreasing order of device-memory footprint
    (ties by index), each to the rank with the least work placed so far among
    the ranks whose memory (`budget` bytes, if given) and item count
    (`max_items`, if given) still take it; ties go to the lower rank.
    Returns each rank's item indices in increasing order. Every rank computes
    the same placement from the same inputs. Raises ValueError when an item
    fits no rank."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(footprints)), key=lambda i: (-int(footprints[i]), i))
    mem = [0] * n_ranks
    load = [0.0] * n_ranks
    parts: List[List[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        best = None
        for r in range(n_ranks):
            if budget is not None and mem[r] + int(footprints[i]) > budget:
                continue
            if max_items is not None and len(parts[r]) >= max_items:
                continue
            if best is None or load[r] < load[best]:
                best = r
        if best is None:
            raise ValueError(f"item {i} ({int(footprints[i])} bytes) fits no rank")
        parts[best].append(i)
        mem[best] += int(footprints[i])
        load[best] += float(work[i])
    return [sorted(p) for p in parts]


def gather_results(obj, device=None):
    """The list of every rank's `obj` on rank 0 (None on the other ranks);
    [obj] on a single process."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out


def reduce_time_and_count(seconds: float, count: float, device=None) -> Tuple[float, float]:
    """(max over ranks of `seconds`, sum over ranks of `count`); the
    arguments themselves on a single process."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds), float(count)
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    c = torch.tensor([count], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())
