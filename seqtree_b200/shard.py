"""Row sharding of an all-vs-all matrix across processes (one process per GPU).

Every (query, ref) pair is independent, so N GPUs split the query rows into contiguous blocks
and each computes its block against all refs; there is no collective on the data path.  The
result is assembled on the host by concatenating the row blocks in rank order.
``torch.distributed`` (NCCL on GPUs, gloo on CPU) carries only the host-side assembly.
"""
from __future__ import annotations

from collections.abc import Callable, Sequence

import numpy as np


def row_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced block [start, stop) of n rows owned by `rank` of `world`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def sharded_matrix(fn: Callable[[Sequence[str], Sequence[str]], object], queries: Sequence[str],
                   refs: Sequence[str], group=None, gather: bool = True):
    """Compute ``fn(queries_block, refs)`` for this rank's row block.

    ``fn`` is any of the matrix calls (e.g. ``lambda q, r: gapblock.score_matrix(q, r, m)``).
    With ``gather`` the blocks are all-gathered and every rank returns the full (N, K) int32
    matrix; otherwise the rank's own block is returned with its row offset.
    """
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    start, stop = row_range(len(queries), world, rank)
    block = np.ascontiguousarray(np.asarray(fn(list(queries[start:stop]), list(refs))),
                                 dtype=np.int32)
    if not gather:
        return start, block
    parts: list = [None] * world
    dist.all_gather_object(parts, (start, block), group=group)
    parts.sort(key=lambda p: p[0])
    if not parts:
        return np.zeros((0, len(refs)), np.int32)
    return np.concatenate([p[1].reshape(-1, len(refs)) for p in parts], axis=0)
