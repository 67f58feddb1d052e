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


@pytest.mark.gpu
def test_topk_over_per_tile_ref_ranges(cuda_ready):
    """st_propose_topk_ranges: each 256-query tile ranks only the 128-ref tiles of its range
    (an empty range yields no candidates; out-of-range values are clamped), exactly as the exact
    top-k over those refs."""
    import torch

    from seqtree_b200.learned import propose_topk_into, swizzle_rows
    rng = np.random.default_rng(17)
    nq, nr, k = 700, 2000, 64
    q, r = _emb(rng, nq), _emb(rng, nr, 40)
    ranges = np.array([[2, 9], [0, 0], [10, 99]], np.int32)  # tile 3 asks past the end: clamped
    qt, rt = swizzle_rows(torch.from_numpy(q).cuda()), swizzle_rows(torch.from_numpy(r).cuda())
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    sc = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    rg = torch.from_numpy(ranges.ravel()).cuda()
    propose_topk_into(qt.data_ptr(), nq, rt.data_ptr(), nr, k, ids.data_ptr(), sc.data_ptr(),
                      torch.cuda.current_stream().cuda_stream, rg.data_ptr())
    torch.cuda.synchronize()
    ids, sc = ids.cpu().numpy(), sc.cpu().numpy()
    ntr = -(-nr // 128)
    for t in range(3):
        rows = slice(256 * t, min(256 * (t + 1), nq))
        lo, hi = max(0, min(ranges[t, 0], ntr)), max(0, min(ranges[t, 1], ntr))
        lo_ref, hi_ref = lo * 128, min(max(hi, lo) * 128, nr)
        want_ids, want_sc = _expected(q[rows], r[lo_ref:hi_ref], k)
        want_ids = np.where(want_ids >= 0, want_ids + lo_ref, -1)
        np.testing.assert_array_equal(sc[rows], want_sc.astype(np.float32))
        np.testing.assert_array_equal(ids[rows], want_ids)


@pytest.mark.gpu
def test_banded_learned_search_is_exact(cuda_ready):
    """A length band restricts the proposals; every reported hit is still an exhaustive hit with
    its exact score, and with every length in the band's reach the recall is unchanged."""
    import seqtree_b200 as stb
    from seqtree_b200 import learned as L
    M = stb.SubstitutionMatrix.blosum62()
    enc = L.Encoder(seed=3)
    rc, rl = L.cdr3_codes(60, 6000)
    qc, ql = L.cdr3_codes(61, 400)
    for band in (0, 2, 40):
        idx = L.LearnedIndex(enc, rc, rl, matrix=M, gap_open=8, max_penalty=24, k=32, band=band)
        rec = idx.recall(qc, ql)
        assert rec["subset_of_exact"]
    wide = L.LearnedIndex(enc, rc, rl, matrix=M, gap_open=8, max_penalty=24, k=32, band=40)
    full = L.LearnedIndex(enc, rc, rl, matrix=M, gap_open=8, max_penalty=24, k=32)
    assert wide.recall(qc, ql)["found"] == full.recall(qc, ql)["found"]
