"""The tensor-core proposal kernel (st_propose_topk) against an exact top-k.

Embedding entries are multiples of 1/16 in [-1/2, 1/2], so every product is a multiple of 2^-8 and
every 64-term dot product is exact in fp32 whatever the summation order: the kernel's scores and
ranking can be compared bit for bit, ties included (many rows repeat, so ties are common).  The
expected order is score descending, then ref id ascending."""
from __future__ import annotations

import numpy as np
import pytest


def _emb(rng, n, distinct=None):
    vals = rng.integers(-8, 9, size=(n if distinct is None else distinct, 64)) / 16.0
    if distinct is not None:  # repeated rows: exact ties between different refs
        vals = vals[rng.integers(0, distinct, size=n)]
    return vals.astype(np.float32)


def _expected(q, r, k):
    s = q.astype(np.float64) @ r.astype(np.float64).T  # exact
    ids = np.full((q.shape[0], k), -1, np.int64)
    sc = np.full((q.shape[0], k), -np.inf)
    order = np.lexsort((np.broadcast_to(np.arange(r.shape[0]), s.shape), -s), axis=1)
    take = min(k, r.shape[0])
    ids[:, :take] = order[:, :take]
    sc[:, :take] = np.take_along_axis(s, order[:, :take], axis=1)
    return ids, sc


def _run(q, r, k):
    import torch

    from seqtree_b200.learned import propose_topk, swizzle_rows
    qt = swizzle_rows(torch.from_numpy(q).cuda())
    rt = swizzle_rows(torch.from_numpy(r).cuda()) if r.shape[0] else torch.empty(
        (0, 64), dtype=torch.bfloat16, device="cuda")
    ids, sc = propose_topk(qt, rt, k)
    return ids.cpu().numpy(), sc.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("nq,nr,k,distinct", [
    (300, 1000, 256, None),     # partial query and ref tiles
    (257, 4097, 7, None),       # small k: many list cuts
    (40, 100, 256, None),       # fewer refs than k: padded rows
    (513, 20000, 256, 50),      # heavy exact ties
    (96, 3000, 100, 3),         # almost everything tied
])
def test_topk_matches_exact_ranking(cuda_ready, nq, nr, k, distinct):
    rng = np.random.default_rng(nq * 7 + nr)
    q, r = _emb(rng, nq), _emb(rng, nr, distinct)
    ids, sc = _run(q, r, k)
    want_ids, want_sc = _expected(q, r, k)
    np.testing.assert_array_equal(sc, want_sc.astype(np.float32))
    np.testing.assert_array_equal(ids, want_ids)


@pytest.mark.gpu
def test_topk_many_tiles_and_cuts(cuda_ready):
    """2,000 queries x 300,000 refs (2,344 ref tiles, 8 query tiles): against torch.topk on
    the same exact scores, checking the score multiset and the tie rule."""
    import torch

    from seqtree_b200.learned import propose_topk, swizzle_rows
    rng = np.random.default_rng(5)
    q, r = _emb(rng, 2000), _emb(rng, 300_000)
    qt, rt = torch.from_numpy(q).cuda(), torch.from_numpy(r).cuda()
    ids, sc = propose_topk(swizzle_rows(qt), swizzle_rows(rt), 256)
    s = qt @ rt.T  # exact (multiples of 2^-8, |s| <= 16)
    want = torch.topk(s, 256, dim=1).values
    torch.testing.assert_close(sc, want, rtol=0, atol=0)
    # the ids are the refs that carry those scores, each once, ties by ascending id
    got = torch.gather(s, 1, ids.long())
    torch.testing.assert_close(got, sc, rtol=0, atol=0)
    idn = ids.cpu().numpy()
    assert all(len(set(row)) == 256 for row in idn[:50])
    scn = sc.cpu().numpy()
    same = scn[:, 1:] == scn[:, :-1]
    assert np.all(idn[:, 1:][same] > idn[:, :-1][same])
    # a tied ref left out of a row has a larger id than every ref of that score kept in the row
    kth = scn[:, -1]
    sn = s.cpu().numpy()
    for i in range(0, 2000, 97):
        tied = np.flatnonzero(sn[i] == kth[i])
        kept = idn[i][scn[i] == kth[i]]
        assert set(kept) == set(tied[:kept.size])


@pytest.mark.gpu
def test_topk_arguments(cuda_ready):
    import torch

    from seqtree_b200.learned import propose_topk, swizzle_rows
    q = swizzle_rows(torch.zeros((4, 64), device="cuda"))
    with pytest.raises(ValueError, match="k must be in 1..256"):
        propose_topk(q, q, 257)
    buf = torch.zeros(8 * 64 + 1, dtype=torch.bfloat16, device="cuda")
    with pytest.raises(ValueError, match="16-byte aligned"):
        propose_topk(buf[1:].view(8, 64), q, 4)
    ids, sc = propose_topk(q, q[:0], 3)  # no refs: every slot empty
    assert (ids.cpu().numpy() == -1).all() and np.isneginf(sc.cpu().numpy()).all()
