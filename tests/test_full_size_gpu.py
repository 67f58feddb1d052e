"""Full-size parity of the named configurations, on the same seeded inputs the benchmark times
(``seqtree_b200.workloads``, seed 1 for queries and 0 for refs), against the reference's own C++
built from its sources (``oracle/_ref``; the C port where that build is absent).

* Hamming 20,000 x 20,000 ACGT, L = 12: every cell.
* Levenshtein 20,000 x 20,000 ACGT, lengths 30-60: 256 rows spread over the matrix, plus the
  |m - n| <= d <= max(m, n) bound on every cell.
* NW and SW 4,096 x 4,096 proteins (background frequencies, log-normal lengths), score and
  distance: 64 rows spread over the matrix, plus d >= 0 everywhere and a zero diagonal on a
  self-distance matrix.
* Sparse 100,000 x 1,000,000 with the structural matrix (2.75e9 hits, run in row blocks): CSR
  order and threshold on every row (on the device), 24 sampled rows against the reference's dense
  rows thresholded.

Rows are independent in every one of these computations, so sampled rows are a faithful check of
the rows they cover; the sampled rows include the first and the last.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
from seqtree_b200 import workloads as W

pytestmark = pytest.mark.gpu
CORES = os.cpu_count() or 1


def spread(n_total, n):
    return np.unique(np.linspace(0, n_total - 1, n).round().astype(np.int64))


def _distance_checker(a, b, lev):
    if oracle.ref_available():
        return oracle.ref_distance_matrix(a, b, lev, threads=0)
    fn = oracle.levenshtein_matrix if lev else oracle.hamming_matrix
    return fn(a, b, threads=CORES)


def _align_checker(q, r, mode, dist):
    if oracle.ref_available():
        return oracle.ref_align_matrix(q, r, "blosum62", mode=mode, dist=dist, threads=0)
    from seqtree_b200 import SubstitutionMatrix
    return oracle.align_matrix(q, r, SubstitutionMatrix.blosum62().similarity_grid, mode=mode,
                               dist=dist, threads=CORES)


def test_hamming_20000_every_cell(cuda_ready):
    from seqtree_b200 import distance
    q = W.uniform_strings(1, 20000, 12, 12, "ACGT")
    r = W.uniform_strings(0, 20000, 12, 12, "ACGT")
    got = np.asarray(distance.hamming_matrix(q, r))
    assert got.shape == (20000, 20000) and got.dtype == np.int32
    r_packed = oracle.Prepacked(r)
    for lo in range(0, 20000, 5000):  # the checker in row blocks of 400 MB
        want = _distance_checker(q[lo:lo + 5000], r_packed, False)
        assert np.array_equal(got[lo:lo + 5000], want), f"rows {lo}..{lo + 4999}"


def test_levenshtein_20000_sampled_rows(cuda_ready):
    from seqtree_b200 import distance
    q = W.uniform_strings(1, 20000, 30, 60, "ACGT")
    r = W.uniform_strings(0, 20000, 30, 60, "ACGT")
    got = np.asarray(distance.levenshtein_matrix(q, r))
    la = np.array([len(s) for s in q], np.int32)[:, None]
    lb = np.array([len(s) for s in r], np.int32)[None, :]
    for lo in range(0, 20000, 2000):  # the bound on every cell, in row blocks
        g = got[lo:lo + 2000]
        assert (g >= np.abs(la[lo:lo + 2000] - lb)).all()
        assert (g <= np.maximum(la[lo:lo + 2000], lb)).all()
    rows = spread(20000, 256)
    assert len(rows) == 256
    want = _distance_checker([q[i] for i in rows], oracle.Prepacked(r), True)
    assert np.array_equal(got[rows], want)


@pytest.mark.parametrize("mode", ["global", "local"])
@pytest.mark.parametrize("dist", [True, False])
def test_protein_4096_sampled_rows(cuda_ready, mode, dist):
    import seqtree_b200 as stb
    q, r = W.proteins(1, 4096), W.proteins(0, 4096)
    m = stb.SubstitutionMatrix.blosum62()
    fn = stb.pairwise.dist_matrix if dist else stb.pairwise.score_matrix
    got = np.asarray(fn(q, r, m, mode=mode))
    assert got.shape == (4096, 4096)
    rows = spread(4096, 64)
    assert len(rows) == 64
    want = _align_checker([q[i] for i in rows], oracle.Prepacked(r), mode, dist)
    assert np.array_equal(got[rows], want)
    if dist:
        assert got.min() >= 0
        sub = [q[i] for i in rows[:16]]
        self_d = np.asarray(fn(sub, sub, m, mode=mode))
        assert (np.diagonal(self_d) == 0).all() and (self_d == self_d.T).all()


def test_sparse_structural_100000x1000000(cuda_ready):
    """The configuration whose hits (2.75e9, 22 GB of CSR) exceed one sort's cap, so the call
    runs in row blocks.  Checked on the device: the CSR is well formed (indptr monotone from 0 to
    nnz, ref ids strictly ascending inside a row, every score within the threshold); 24 rows
    against the reference's dense rows thresholded."""
    import torch

    import seqtree_b200 as stb
    from seqtree_b200 import device
    q, r = W.cdr3_skewed(1, 100000), W.cdr3_skewed(0, 1000000)
    m = stb.SubstitutionMatrix.structural()
    qs, rs = device.SeqSet(q, "aa"), device.SeqSet(r, "aa")
    hits = device.Hits()
    nnz = device.gapblock_sparse_into(qs, rs, hits, torch.cuda.current_stream().cuda_stream,
                                      max_penalty=24, matrix=m, gap_open=8, gap_extend=1)
    torch.cuda.synchronize()
    info = hits.info()
    assert info["rows"] == 100000 and info["cols"] == 1000000 and nnz == info["nnz"] > 2**31
    ip = torch.as_tensor(device._DeviceArray(info["indptr"], 100001, "<i8"), device="cuda")
    assert int(ip[0]) == 0 and int(ip[-1]) == nnz and bool((ip[1:] >= ip[:-1]).all())
    ri = torch.as_tensor(device._DeviceArray(info["ref_ids"], nnz, "<i4"), device="cuda")
    sc = torch.as_tensor(device._DeviceArray(info["scores"], nnz, "<i4"), device="cuda")
    chunk = 1 << 28
    for lo in range(0, nnz, chunk):  # bounded temporaries
        s = sc[lo:lo + chunk]
        assert int(s.min()) >= 0 and int(s.max()) <= 24
    starts = torch.zeros(nnz, dtype=torch.bool, device="cuda")
    starts[ip[:-1][ip[1:] > ip[:-1]]] = True
    for lo in range(1, nnz, chunk):
        hi = min(lo + chunk, nnz)
        up = ri[lo:hi] > ri[lo - 1:hi - 1]
        assert bool((up | starts[lo:hi]).all()), f"order broken near {lo}"
    del starts
    rows = spread(100000, 24)
    rows_got = device.hits_rows(hits, rows)
    if oracle.ref_available():
        dense = oracle.ref_gapblock_matrix([q[i] for i in rows], oracle.Prepacked(r),
                                           matrix="structural", gap_open=8, gap_extend=1)
    else:
        dense = oracle.gapblock_matrix([q[i] for i in rows], r, m.penalty_grid, gap_open=8,
                                       gap_extend=1, threads=CORES)
    for k, (ids, s) in enumerate(rows_got):
        want = np.flatnonzero(dense[k] <= 24)
        np.testing.assert_array_equal(ids, want)
        np.testing.assert_array_equal(s, dense[k, want])
