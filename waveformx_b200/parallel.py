"""Data parallelism over binaries: one process per GPU.

Binaries are independent, so a batch is split into contiguous ranges of
binaries, one per rank, with the frequency grid (and a likelihood's data and
weights) replicated: the hot path needs no collective. A ragged batch is
split by the prefix sum of its grid lengths, so that every rank evaluates
about the same number of (binary, frequency) pairs. Where a caller wants
every rank to hold every binary's result (a sampler's log-likelihoods and
gradients: tens of bytes per binary), :func:`gather_rows` all-gathers them
(NCCL between GPUs, gloo on CPU).
"""

from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

__all__ = ["shard", "shard_ragged", "gather_rows", "rank_and_world", "local_slice"]


def rank_and_world(group=None) -> tuple[int, int]:
    """``(rank, world size)`` of the default (or given) process group, or
    ``(0, 1)`` without one."""
    try:
        import torch.distributed as dist
    except ImportError:  # pragma: no cover
        return 0, 1
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def shard(batch: int, rank: int, world: int) -> slice:
    """Rank ``rank``'s contiguous range of ``batch`` binaries: the first
    ``batch % world`` ranks take one binary more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of a world of {world}")
    if batch < 0:
        raise ValueError("batch must be non-negative")
    base, extra = divmod(batch, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def shard_ragged(offsets: Sequence[int], rank: int, world: int) -> slice:
    """Rank ``rank``'s contiguous range of binaries of a ragged batch
    (``offsets``: the ``B + 1`` starts of the binaries' grids in the flat
    frequency array), balanced by the number of frequencies: the range whose
    frequencies start at or after ``rank / world`` of the total and before
    ``(rank + 1) / world`` of it."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of a world of {world}")
    offsets = np.asarray(offsets, dtype=np.int64)
    if offsets.ndim != 1 or len(offsets) < 1 or np.any(np.diff(offsets) < 0):
        raise ValueError("offsets must be a non-decreasing 1-d array of B + 1 starts")
    total = int(offsets[-1] - offsets[0])
    starts = offsets[:-1] - offsets[0]
    lo = int(np.searchsorted(starts, rank * total / world, side="left")) if rank else 0
    hi = int(np.searchsorted(starts, (rank + 1) * total / world, side="left")) if rank + 1 < world else len(starts)
    return slice(lo, max(lo, hi))


def gather_rows(local, batch: int, group=None):
    """All ranks' rows (their :func:`shard` ranges of ``batch`` binaries) in
    order, on every rank: ``local`` is this rank's ``(rows, ...)`` tensor.
    Uneven shards are padded to the largest for the collective."""
    import torch
    import torch.distributed as dist

    rank, world = rank_and_world(group)
    if world == 1:
        return local
    sizes = [shard(batch, r, world).stop - shard(batch, r, world).start for r in range(world)]
    if local.shape[0] != sizes[rank]:
        raise ValueError(f"rank {rank} holds {local.shape[0]} rows, its shard has {sizes[rank]}")
    width = max(sizes)
    padded = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    padded[: local.shape[0]] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p[:n] for p, n in zip(parts, sizes)], dim=0)


def local_slice(batch: int, group=None, offsets: Optional[Sequence[int]] = None) -> slice:
    """This rank's range of a batch (ragged when ``offsets`` is given)."""
    rank, world = rank_and_world(group)
    return shard_ragged(offsets, rank, world) if offsets is not None else shard(batch, rank, world)
