"""Multi-GPU by replicas: stereo pairs are independent, so N GPUs run N copies of the
pipeline on disjoint pairs with no data exchange (one process per GPU,
torch.distributed for the plumbing).  The only collective is the max-over-ranks of
a device-timed duration (a scalar), used to report whole-job throughput.

  shard(items, rank, world)    the pairs this rank matches (round robin: ranks stay
                               within one pair of each other in count and, for mixed
                               sizes drawn at random, in work)
  rank_seed(rank, base)        disjoint synthetic-data seeds per rank
  max_over_ranks(x)            the slowest rank's value, on the process group's device
"""
from __future__ import annotations

from typing import Sequence


def shard(items: Sequence, rank: int, world: int) -> list:
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return list(items[rank::world])


def rank_seed(rank: int, base: int = 0, stride: int = 1000) -> int:
    return base + stride * rank


def max_over_ranks(x: float) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
