"""One process per GPU: rank discovery, the per-rank share of a batch of
independent systems, and the two reductions a multi-GPU measurement needs.

Systems are independent, so the data path has no collective: every rank
builds and advances its own systems. The only collectives combine the
measurement: the maximum of the ranks' device times and the sum of their
moves (max-over-ranks timing). The process group may be NCCL (GPUs) or gloo
(CPU tests); the calls are the same on every rank and in the same order.
"""
from __future__ import annotations

import os
from typing import Tuple

# seeds of a rank's batch are spaced by a prime, so no two ranks share one
RANK_SEED_STRIDE = 7919


def rank_env() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def batch_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s batch: weak scaling, every rank its own systems."""
    return base + RANK_SEED_STRIDE * rank


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
