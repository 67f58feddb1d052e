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


# ------------------------------------------------------------------ threshold form ----------
def _range_expected(q, r, ql, rl, thr):
    s = q.astype(np.float64) @ r.astype(np.float64).T  # exact
    t = thr.astype(np.float64)[np.minimum(ql, 32)[:, None], np.minimum(rl, 32)[None, :]]
    qi, ri = np.nonzero(s >= t)
    return np.stack([qi, ri], 1)


def _range_run(q, r, ql, rl, thr, capacity=None, ranges=None):
    import torch

    from seqtree_b200.learned import propose_range, swizzle_rows
    qt = swizzle_rows(torch.from_numpy(q).cuda())
    rt = swizzle_rows(torch.from_numpy(r).cuda())
    qlt = torch.from_numpy(ql.astype(np.uint8)).cuda()
    rlt = torch.from_numpy(rl.astype(np.uint8)).cuda()
    rg = None if ranges is None else torch.from_numpy(np.asarray(ranges, np.int32).ravel()).cuda()
    pq, pr = propose_range(qt, qlt, rt, rlt, thr, capacity, rg)
    got = np.stack([pq.cpu().numpy(), pr.cpu().numpy()], 1).astype(np.int64)
    return got[np.lexsort((got[:, 1], got[:, 0]))]


def _thr_table(rng, off=0.3):
    """Thresholds on the 2^-8 grid (ties with exact scores happen), a few cells switched off."""
    thr = (np.round(rng.uniform(-0.5, 1.5, size=(33, 33)) * 256) / 256 + off).astype(np.float32)
    thr[rng.random((33, 33)) < 0.1] = np.inf
    return thr


@pytest.mark.gpu
@pytest.mark.parametrize("nq,nr,sort_refs,distinct", [
    (300, 1000, True, None),       # partial query and ref tiles
    (600, 50_000, True, 40),       # many tiles, exact ties between refs
    (257, 4099, False, None),      # unsorted ref lengths: every group straddles lengths
    (1, 1, True, None),            # one pair
])
def test_range_matches_exact_threshold(cuda_ready, nq, nr, sort_refs, distinct):
    """st_propose_range returns exactly the pairs whose exact dot product reaches the threshold
    of their (query length, ref length) cell, each once."""
    rng = np.random.default_rng(nq * 13 + nr)
    q, r = _emb(rng, nq), _emb(rng, nr, distinct)
    ql = rng.integers(8, 26, size=nq)
    rl = rng.integers(8, 26, size=nr)
    if sort_refs:
        rl = np.sort(rl)
    thr = _thr_table(rng)
    got = _range_run(q, r, ql, rl, thr)
    want = _range_expected(q, r, ql, rl, thr)
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_range_capacity_ranges_and_lengths_past_32(cuda_ready):
    """A capacity below the count still returns the full count and then the exact set (the
    wrapper repeats the call); per-tile ranges limit the scanned refs; lengths above 32 use the
    table's last row and column; a table of +inf proposes nothing."""
    import torch

    from seqtree_b200.learned import propose_range_into, swizzle_rows
    rng = np.random.default_rng(23)
    nq, nr = 520, 3000
    q, r = _emb(rng, nq), _emb(rng, nr)
    ql = rng.integers(20, 40, size=nq)
    rl = np.sort(rng.integers(20, 40, size=nr))
    thr = np.full((33, 33), 0.25, np.float32)
    thr[32, 32] = 0.0
    want = _range_expected(q, r, ql, rl, thr)
    assert want.shape[0] > 200
    got = _range_run(q, r, ql, rl, thr, capacity=7)
    np.testing.assert_array_equal(got, want)
    # a raw call with room for 7 pairs: the full count, seven distinct expected pairs written
    qt, rt = swizzle_rows(torch.from_numpy(q).cuda()), swizzle_rows(torch.from_numpy(r).cuda())
    qlt = torch.from_numpy(ql.astype(np.uint8)).cuda()
    rlt = torch.from_numpy(rl.astype(np.uint8)).cuda()
    pq = torch.full((7,), -1, dtype=torch.int32, device="cuda")
    pr = torch.full((7,), -1, dtype=torch.int32, device="cuda")
    n = propose_range_into(qt.data_ptr(), nq, qlt.data_ptr(), rt.data_ptr(), nr, rlt.data_ptr(),
                           thr, pq.data_ptr(), pr.data_ptr(), 7,
                           torch.cuda.current_stream().cuda_stream)
    assert n == want.shape[0]
    part = set(zip(pq.cpu().tolist(), pr.cpu().tolist()))
    assert len(part) == 7 and part <= set(map(tuple, want.tolist()))
    # per-tile ranges: tile 0 scans ref tiles [3, 9), tile 1 none, tile 2 past the end (clamped)
    ranges = np.array([[3, 9], [0, 0], [20, 99]], np.int32)
    got = _range_run(q, r, ql, rl, thr, ranges=ranges)
    keep = np.zeros(len(want), bool)
    for t, (lo, hi) in enumerate(ranges):
        lo_ref, hi_ref = min(lo, 24) * 128, min(max(hi, lo), 24) * 128
        keep |= (want[:, 0] // 256 == t) & (want[:, 1] >= lo_ref) & (want[:, 1] < hi_ref)
    np.testing.assert_array_equal(got, want[keep])
    off = np.full((33, 33), np.inf, np.float32)
    assert _range_run(q, r, ql, rl, off).shape[0] == 0


@pytest.mark.gpu
def test_embed_dots_are_the_exact_dot_products(cuda_ready):
    import torch

    from seqtree_b200.learned import embed_dots_into, swizzle_rows
    rng = np.random.default_rng(29)
    q, r = _emb(rng, 77), _emb(rng, 301)
    qi = rng.integers(0, 77, size=5000).astype(np.int32)
    ri = rng.integers(0, 301, size=5000).astype(np.int32)
    qi[:3] = [77, -1, 0]  # out of range: NaN
    ri[:3] = [0, 0, 301]
    qt, rt = swizzle_rows(torch.from_numpy(q).cuda()), swizzle_rows(torch.from_numpy(r).cuda())
    qit, rit = torch.from_numpy(qi).cuda(), torch.from_numpy(ri).cuda()
    out = torch.empty(5000, dtype=torch.float32, device="cuda")
    embed_dots_into(qt.data_ptr(), 77, rt.data_ptr(), 301, qit.data_ptr(), rit.data_ptr(), 5000,
                    out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    got = out.cpu().numpy()
    assert np.isnan(got[:3]).all()
    want = (q[qi[3:]].astype(np.float64) * r[ri[3:]].astype(np.float64)).sum(1)
    np.testing.assert_array_equal(got[3:], want.astype(np.float32))


@pytest.mark.gpu
def test_range_learned_search_is_exact_and_calibrated(cuda_ready):
    """The threshold form of LearnedIndex: every reported hit is an exhaustive hit with its exact
    score, calibration reaches the bound on its batch, and a model file keeps the thresholds."""
    import seqtree_b200 as stb
    from seqtree_b200 import learned as L
    M = stb.SubstitutionMatrix.blosum62()
    enc = L.Encoder(seed=3)
    rc, rl = L.cdr3_codes(70, 8000)
    cc, cl = L.cdr3_codes(71, 600)
    idx = L.LearnedIndex(enc, rc, rl, matrix=M, gap_open=8, max_penalty=24, proposal="range")
    cal = idx.calibrate(cc, cl, bound=0.99)
    assert cal["subset_of_exact"] and cal["recall"] >= 0.99
    qc, ql = L.cdr3_codes(72, 500)
    rec = idx.recall(qc, ql)
    assert rec["subset_of_exact"]
    assert rec["recall"] >= 0.9


@pytest.mark.gpu
def test_search_strings_matches_the_code_path(cuda_ready):
    """search_strings (strings packed by the library, rows copied into pinned blocks) returns
    exactly the CSR of search() on padded codes, and rejects bad input with pad_codes' errors."""
    import seqtree_b200 as stb
    from seqtree_b200 import learned as L
    M = stb.SubstitutionMatrix.blosum62()
    enc = L.Encoder(seed=5)
    rc, rl = L.cdr3_codes(80, 5000)
    cc, cl = L.cdr3_codes(81, 400)
    idx = L.LearnedIndex(enc, rc, rl, matrix=M, gap_open=8, max_penalty=24, proposal="range")
    idx.calibrate(cc, cl, bound=0.99)
    qc, ql = L.cdr3_codes(82, 700)
    strings = L.codes_to_strings(qc, ql)
    got = idx.search_strings(strings)
    ip, ri, sc = (t.cpu().numpy() for t in idx.search(idx.queries(qc, ql)))
    assert np.array_equal(got.indptr, ip) and np.array_equal(got.ref_ids, ri)
    assert np.array_equal(got.scores, sc) and got.shape == (700, 5000)
    with pytest.raises(ValueError, match="symbol 'J'"):
        idx.search_strings(["CASSLF", "CAJSF", "CAS#F"])
    with pytest.raises(ValueError, match="1..32 residues"):
        idx.search_strings(["CASSLF", ""])
