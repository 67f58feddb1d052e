"""Row sharding across ranks (the multi-GPU form of the path), exercised with world_size 2 on
the gloo backend on CPU.  The per-block scorer is the CPU oracle here; on GPUs it is the CUDA
library.  No GPU is needed."""
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
        full = sharded_matrix(fn, q, r)
        start, block = sharded_matrix(fn, q, r, gather=False)
        out_q.put((rank, full.tolist(), start, block.shape[0], fn(q, r).tolist()))
    finally:
        dist.destroy_process_group()


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
