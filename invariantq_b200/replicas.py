"""Helpers for runs with one process per GPU (``torchrun``; RANK, WORLD_SIZE,
LOCAL_RANK in the environment).

The gate-application path does not split a state across GPUs (a 30-qubit
complex128 state is 16 GiB of one B200's 180 GB), so ranks run independent
replicas of a workload, or disjoint shares of independent jobs (circuits of
a gradient batch).  Nothing is exchanged on the data path; the only
collective combines timings: a rank's device time is reduced by MAX, so the
reported throughput is the work of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import os
from typing import Sequence, Tuple, TypeVar

T = TypeVar("T")


def env_ranks() -> Tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def shard(items: Sequence[T], rank: int, world: int) -> list:
    """This rank's share: every world-th item starting at `rank` (interleaved,
    so shares of a batch ordered by size get similar work)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(items[rank::world])


def max_over_ranks(x: float, device=None) -> float:
    """MAX of x over the ranks of the default process group (x itself when no
    group is initialised or the world has one rank).  `device`: where the
    reduction tensor lives (a CUDA device for NCCL, None for gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
