"""Pictures across GPUs: one process per GPU, each solving its own share of the pictures (they are
independent: no data crosses between GPUs while they are solved), the timing taken as the
slowest rank's. torch.distributed carries the few scalars and, where wanted, the results'
collection; NCCL between GPUs, gloo between CPU processes (as the tests run it).
"""

from __future__ import annotations

from collections.abc import Sequence

import torch
import torch.distributed as dist


def rank_and_world() -> tuple[int, int]:
    """This process's rank and the number of ranks (1 and 0 without a process group)."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(weights: Sequence[int], world: int) -> list[list[int]]:
    """The indices of the pictures each of `world` ranks solves: the largest first, each to the
    rank with the least work so far (pixels), so that the slowest rank has as little as can be."""
    if world < 1:
        raise ValueError("at least one rank")
    loads = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for index in sorted(range(len(weights)), key=lambda n: (-weights[n], n)):
        rank = min(range(world), key=lambda r: (loads[r], r))
        out[rank].append(index)
        loads[rank] += int(weights[index])
    for indices in out:
        indices.sort()
    return out


def max_over_ranks(value: float) -> float:
    """The largest of every rank's value (every rank calls it, in the same order)."""
    rank, world = rank_and_world()
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float) -> float:
    """The sum of every rank's value (every rank calls it, in the same order)."""
    rank, world = rank_and_world()
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
