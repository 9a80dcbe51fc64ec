"""Row-block sharding of the sketch update over ranks (one process per GPU).

The rows of A (or of the kernel matrix) are split into contiguous blocks,
one per rank; each rank streams its own block through its own context.
Y rows are disjoint across ranks and stay where they are. X and Z are sums
of per-window terms, so the whole-matrix sketches are an all-reduce (sum)
of the ranks' partial X and Z -- with one correction for nu != 1: the
reference applies X = nu X + eta x_w window after window over the whole
matrix (src/Skema_SketchySVD.cpp:167-233), so the terms a rank adds are
later multiplied by nu once per window of the ranks after it. Scaling each
rank's partial by nu^(windows after its block) before the sum reproduces
that sequence exactly.
"""
from __future__ import annotations

import math


def shard_rows(m: int, world: int, rank: int, window: int = 1) -> tuple[int, int]:
    """(row0, nrows) of `rank`'s block. Blocks are contiguous and, except
    the last, a whole number of windows long, so every rank's windows start
    where the one-process window sequence has them."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    nwin = (m + window - 1) // window
    per = (nwin + world - 1) // world * window
    row0 = min(m, rank * per)
    return row0, max(0, min(per, m - row0))


def windows_after(m: int, world: int, rank: int, window: int = 1) -> int:
    """Windows of the one-process sequence that follow `rank`'s block."""
    row0, nrows = shard_rows(m, world, rank, window)
    end = row0 + nrows
    return (m - end + window - 1) // window


def reduce_partial_sketches(X, Z, m: int, window: int, nu: float, group=None) -> None:
    """In-place sum over the ranks of the partial X and Z (torch tensors on
    this rank's device), weighted so the result equals the one-process
    sequence. Every rank must call it (a collective)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if nu != 1.0:
        w = math.pow(nu, windows_after(m, world, rank, window))
        X.mul_(w)
        Z.mul_(w)
    dist.all_reduce(X, group=group)
    dist.all_reduce(Z, group=group)


class _DeviceBuffer:
    """A CUDA array interface over count FP64 values at a device pointer,
    so that torch can view the library's buffer without a copy."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_allreduce(group=None):
    """allreduce(ptr, count) for SketchySVD.low_rank_approx_rows: sums
    count FP64 values at a device pointer over the process group with
    torch.distributed (NCCL) and waits for the sum before returning."""
    import torch
    import torch.distributed as dist

    def allreduce(ptr: int, count: int) -> None:
        t = torch.as_tensor(_DeviceBuffer(ptr, count), device="cuda")
        dist.all_reduce(t, group=group)
        torch.cuda.current_stream().synchronize()

    return allreduce


def low_rank_approx_sharded(ctx, m: int, window: int, group=None):
    """The fixed-rank approximation of a row-block sharded sketch: this
    rank's rows of U, and S, V of the whole matrix. X and Z must already be
    summed over the ranks (reduce_partial_sketches). Every rank calls it."""
    import torch.distributed as dist

    row0, nrows = shard_rows(m, dist.get_world_size(group), dist.get_rank(group), window)
    return ctx.low_rank_approx_rows(row0, nrows, device_allreduce(group))
