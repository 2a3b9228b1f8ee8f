"""Independent replicas, one process per GPU (weak scaling).

Both hot paths split into independent units -- (a,b,c) triples for the sieve,
candidates for the tests -- with no exchange step, so N GPUs run N replicas:
rank r takes its own shard of the units, nothing crosses between ranks on the
data path, and the only collectives are the barrier around the timed region
and the max over ranks of its duration (the job takes as long as its slowest
rank).  Works with any torch.distributed backend (nccl on GPUs, gloo on CPU).
"""
from __future__ import annotations

import os
from typing import List, Sequence


def rank_world():
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(units: Sequence, rank: int, world: int) -> List:
    """Rank r's units: every world-th unit from r (disjoint, covering)."""
    return list(units[rank::world])


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank r's synthetic draws (rank 0 keeps the single-GPU seed)."""
    return seed + 7919 * rank


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, seconds_max: float, world: int) -> float:
    """Whole-job throughput: the units of all ranks over the slowest rank's time."""
    return units_per_rank * world / seconds_max
