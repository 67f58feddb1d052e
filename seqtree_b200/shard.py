"""Row sharding of the all-vs-all calls across processes (one process per GPU).

Every (query, ref) pair is independent, so N GPUs split the query rows into contiguous blocks and
each computes its block against all refs (the refs, and for the learned search their embeddings,
are replicated on every rank); there is no collective on the data path.  Results are assembled on
the host by concatenating the row blocks in rank order:

* dense matrices (``sharded_matrix``): the int32 row blocks stacked;
* thresholded sparse rows (``sharded_sparse``) and learned searches (``sharded_learned_search``):
  the CSR blocks joined, each block's ``indptr`` shifted by the hits of the blocks before it
  (the rows of ``score_sparse`` / ``GapBlockIndex.search`` consumers, python/seqtree/
  gapblock.py:611-634, read the same CSR either way).

``gather`` chooses where the result lands: ``"root"`` (the default) sends every block to rank
``dst`` only, which returns the whole result while the other ranks return ``None`` -- host memory
is one copy of the result on one rank; ``"all"`` gives every rank the whole result (one copy per
rank); ``"none"`` returns this rank's block with its first row, and nothing crosses ranks.
``torch.distributed`` (NCCL on GPUs, gloo on CPU) carries only this host-side assembly.
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


def _collect(part, group, gather: str, dst: int):
    """The (start, payload) parts of every rank, in row order, where ``gather`` puts them (None on
    ranks that receive nothing)."""
    import torch.distributed as dist

    if gather not in ("root", "all"):
        raise ValueError("gather must be 'root', 'all' or 'none'")
    world = dist.get_world_size(group)
    if gather == "all":
        parts: list = [None] * world
        dist.all_gather_object(parts, part, group=group)
    else:
        root = dist.get_global_rank(group, dst) if group is not None else dst
        parts = [None] * world if dist.get_rank(group) == dst else None
        dist.gather_object(part, parts, dst=root, group=group)
        if parts is None:
            return None
    return sorted(parts, key=lambda p: p[0])


def sharded_matrix(fn: Callable[[Sequence[str], Sequence[str]], object], queries: Sequence[str],
                   refs: Sequence[str], group=None, gather: str = "root", dst: int = 0):
    """``fn(queries_block, refs)`` for this rank's row block, assembled per ``gather``.

    ``fn`` is any of the dense matrix calls (e.g. ``lambda q, r: gapblock.score_matrix(q, r, m)``).
    Returns the (N, K) int32 matrix (``"root"``: on rank ``dst`` only, None elsewhere;
    ``"all"``: on every rank), or with ``"none"`` this rank's ``(start, block)``.
    """
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    start, stop = row_range(len(queries), world, rank)
    block = np.ascontiguousarray(np.asarray(fn(list(queries[start:stop]), list(refs))),
                                 dtype=np.int32).reshape(stop - start, len(refs))
    if gather == "none":
        return start, block
    parts = _collect((start, block), group, gather, dst)
    if parts is None:
        return None
    return np.concatenate([p[1] for p in parts], axis=0)


def join_csr(parts, cols: int, max_penalty: int):
    """One ``SparseScores`` from row blocks ``[(start, indptr, ref_ids, scores), ...]`` given in
    row order (each block's indptr starting at 0)."""
    from .gapblock import SparseScores
    rows = sum(int(p[1].size) - 1 for p in parts)
    indptr = np.zeros(rows + 1, np.int64)
    at, base = 0, 0
    for start, ip, _, _ in parts:
        if start != at:
            raise ValueError("row blocks are not contiguous")
        n = int(ip.size) - 1
        indptr[at + 1:at + n + 1] = np.asarray(ip[1:], np.int64) + base
        at += n
        base += int(ip[-1])
    ref_ids = np.concatenate([np.asarray(p[2], np.int32) for p in parts]) if parts else \
        np.zeros(0, np.int32)
    scores = np.concatenate([np.asarray(p[3], np.int32) for p in parts]) if parts else \
        np.zeros(0, np.int32)
    return SparseScores(indptr, ref_ids, scores, (rows, cols), max_penalty)


def sharded_sparse(fn: Callable[[Sequence[str], Sequence[str]], object], queries: Sequence[str],
                   refs: Sequence[str], group=None, gather: str = "root", dst: int = 0):
    """Thresholded rows (``SparseScores``) of this rank's row block, assembled per ``gather``.

    ``fn`` returns a ``SparseScores`` for a query block against all refs, e.g.
    ``lambda q, r: gapblock.score_sparse(q, r, 24, m)``.  The joined CSR equals the single-rank
    call's: the same rows, refs ascending inside each, the same scores.
    """
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    start, stop = row_range(len(queries), world, rank)
    sp = fn(list(queries[start:stop]), list(refs))
    part = (start, np.asarray(sp.indptr, np.int64), np.asarray(sp.ref_ids, np.int32),
            np.asarray(sp.scores, np.int32))
    if gather == "none":
        return start, sp
    parts = _collect(part, group, gather, dst)
    if parts is None:
        return None
    return join_csr(parts, len(refs), sp.max_penalty)


def sharded_learned_search(index, queries: Sequence[str], group=None, gather: str = "root",
                           dst: int = 0):
    """``index.search_strings`` over this rank's row block of ``queries``, assembled per
    ``gather``.  ``index`` is a ``learned.LearnedIndex`` built on every rank over the same refs
    (the refs and their embeddings are replicated; only query rows are split)."""
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    start, stop = row_range(len(queries), world, rank)
    sp = index.search_strings(list(queries[start:stop]))
    part = (start, np.asarray(sp.indptr, np.int64), np.asarray(sp.ref_ids, np.int32),
            np.asarray(sp.scores, np.int32))
    if gather == "none":
        return start, sp
    parts = _collect(part, group, gather, dst)
    if parts is None:
        return None
    return join_csr(parts, int(sp.shape[1]), sp.max_penalty)
