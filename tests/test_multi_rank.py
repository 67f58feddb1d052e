"""Row sharding across ranks (the multi-GPU form of the path), exercised with world_size 2 on
the gloo backend on CPU.  What is tested is the sharding and the host-side assembly (row
blocks, CSR joins, where the result lands); the per-block scorer is a CPU stand-in built on the
oracle here (dense rows, thresholded rows, and a learned index's ``search_strings``), where on
GPUs it is the CUDA library.  No GPU is needed."""
from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, kind: str, out_q) -> None:
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist

    import oracle
    from conftest import cdr3, rand_seqs
    from seqtree_b200.matrix import SubstitutionMatrix
    from seqtree_b200.shard import sharded_matrix

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(5)
        if kind == "gapblock":
            q, r = cdr3(rng, 37), cdr3(rng, 53)
            pen = SubstitutionMatrix.blosum62().penalty_grid
            fn = lambda a, b: oracle.gapblock_matrix(a, b, pen, gap_open=8, threads=1)  # noqa: E731
        else:
            q, r = rand_seqs(rng, 29, 0, 20, "ACGT"), rand_seqs(rng, 31, 0, 20, "ACGT")
            fn = lambda a, b: oracle.levenshtein_matrix(a, b, threads=1)  # noqa: E731
        full = sharded_matrix(fn, q, r, gather="all")
        root = sharded_matrix(fn, q, r)  # to rank 0 only
        assert (root is None) == (rank != 0)
        if root is not None:
            assert np.array_equal(root, full)
        start, block = sharded_matrix(fn, q, r, gather="none")
        out_q.put((rank, full.tolist(), start, block.shape[0], fn(q, r).tolist()))
    finally:
        dist.destroy_process_group()


def _sparse_worker(rank: int, world: int, port: int, kind: str, out_q) -> None:
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist

    import oracle
    from conftest import cdr3
    from seqtree_b200.gapblock import SparseScores
    from seqtree_b200.matrix import SubstitutionMatrix
    from seqtree_b200.shard import sharded_learned_search, sharded_sparse

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(9)
        q, r = cdr3(rng, 41, 8, 16), cdr3(rng, 97, 8, 16)
        pen = SubstitutionMatrix.blosum62().penalty_grid

        def thresholded(a, b):  # the CPU stand-in of score_sparse
            d = oracle.gapblock_matrix(a, b, pen, gap_open=8, threads=1)
            keep = d <= 24
            indptr = np.concatenate([[0], np.cumsum(keep.sum(axis=1))]).astype(np.int64)
            rows, cols = np.nonzero(keep)
            return SparseScores(indptr, cols.astype(np.int32), d[rows, cols].astype(np.int32),
                                d.shape, 24)

        class StandInIndex:  # the CPU stand-in of a LearnedIndex built over r on every rank
            def search_strings(self, queries):
                return thresholded(queries, r)

        if kind == "sparse":
            got = sharded_sparse(thresholded, q, r, gather="all")
            root = sharded_sparse(thresholded, q, r)
        else:
            got = sharded_learned_search(StandInIndex(), q, gather="all")
            root = sharded_learned_search(StandInIndex(), q)
        assert (root is None) == (rank != 0)
        one = thresholded(q, r)
        out_q.put((rank, got.shape == one.shape and got.indptr.tolist() == one.indptr.tolist()
                   and got.ref_ids.tolist() == one.ref_ids.tolist()
                   and got.scores.tolist() == one.scores.tolist() and one.nnz > 0,
                   root is None or (root.indptr.tolist() == one.indptr.tolist()
                                    and root.scores.tolist() == one.scores.tolist())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["sparse", "learned"])
def test_two_ranks_join_the_single_rank_csr(kind):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sparse_worker, args=(r, 2, port, kind, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok_all and ok_root for _, ok_all, ok_root in results)


def test_join_csr_offsets_each_block():
    from seqtree_b200.shard import join_csr
    parts = [(0, np.array([0, 2, 2]), np.array([1, 5]), np.array([3, 4])),
             (2, np.array([0, 1]), np.array([0]), np.array([7]))]
    sp = join_csr(parts, 6, 24)
    assert sp.shape == (3, 6) and sp.indptr.tolist() == [0, 2, 2, 3]
    assert sp.ref_ids.tolist() == [1, 5, 0] and sp.scores.tolist() == [3, 4, 7]
    with pytest.raises(ValueError, match="contiguous"):
        join_csr(parts[1:], 6, 24)


@pytest.mark.parametrize("kind", ["gapblock", "levenshtein"])
def test_two_ranks_assemble_the_single_rank_matrix(kind):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, kind, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    (_, full0, s0, n0, ref), (_, full1, s1, n1, _) = results
    assert full0 == full1 == ref
    assert (s0, s1) == (0, n0) and n0 + n1 == len(ref)


def test_row_range_balances_and_covers():
    from seqtree_b200.shard import row_range
    for n in (0, 1, 7, 100):
        for world in (1, 2, 3, 8):
            blocks = [row_range(n, world, r) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        row_range(3, 2, 2)
