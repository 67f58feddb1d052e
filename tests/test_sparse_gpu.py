"""Thresholded sparse gap-block matrix: every row must hold exactly the dense matrix's cells with
score <= max_penalty, in ref order, with their scores -- checked against the oracle's dense
matrix on small sets and against the GPU's own dense matrix at larger sizes."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cdr3, prior_by_name, rand_seqs
from seqtree_b200.gapblock import prior_cube, score_sparse
from seqtree_b200.matrix import SubstitutionMatrix


def csr_of(dense: np.ndarray, thresh: int):
    keep = dense <= thresh
    indptr = np.zeros(dense.shape[0] + 1, np.int64)
    np.cumsum(keep.sum(axis=1), out=indptr[1:])
    rows, cols = np.nonzero(keep)
    return indptr, cols.astype(np.int32), dense[rows, cols].astype(np.int32)


def assert_same(sp, dense, thresh):
    indptr, ref_ids, scores = csr_of(dense, thresh)
    assert sp.shape == dense.shape
    np.testing.assert_array_equal(sp.indptr, indptr)
    np.testing.assert_array_equal(sp.ref_ids, ref_ids)
    np.testing.assert_array_equal(sp.scores, scores)


def oracle_dense(q, r, matrix, go, ge, prior_name):
    pen = (matrix or SubstitutionMatrix.unit(24)).penalty_grid
    prior = prior_by_name(prior_name)
    width = max(map(len, q + r))
    cube = None if prior is None else np.asarray(prior_cube(prior, width), np.int32).ravel()
    return oracle.gapblock_matrix(q, r, pen, gap_open=go, gap_extend=ge, prior=cube,
                                  prior_width=width)


@pytest.mark.gpu
@pytest.mark.parametrize("matrix_name,prior_name,thresh", [
    ("blosum62", "none", 24), ("blosum62", "central21", 40), ("structural", "none", 24),
    ("blosum62", "frame21_5", 60), (None, "none", 3), ("blosum62", "none", 0),
])
def test_sparse_matches_thresholded_oracle(cuda_ready, matrix_name, prior_name, thresh):
    rng = np.random.default_rng(11)
    q = cdr3(rng, 150, 8, 25)
    r = cdr3(rng, 700, 8, 25)
    r[:40] = q[:40]                       # exact hits
    r[40:60] = [s[:-2] + "F" for s in q[40:60]]  # one-column deletions
    matrix = None if matrix_name is None else getattr(SubstitutionMatrix, matrix_name)()
    go = 8 if matrix is not None else 1
    dense = oracle_dense(q, r, matrix, go, 1, prior_name)
    sp = score_sparse(q, r, thresh, matrix, gap_open=go, gap_extend=1,
                      gap_prior=prior_by_name(prior_name))
    assert sp.nnz > 0
    assert_same(sp, dense, thresh)


@pytest.mark.gpu
def test_sparse_general_path_long_sequences(cuda_ready):
    rng = np.random.default_rng(3)
    q = rand_seqs(rng, 40, 60, 90)
    r = rand_seqs(rng, 90, 60, 90) + q[:10]
    m = SubstitutionMatrix.blosum62()
    dense = oracle_dense(q, r, m, 8, 1, "none")
    thresh = int(np.percentile(dense, 5))
    sp = score_sparse(q, r, thresh, m, gap_open=8)
    assert_same(sp, dense, thresh)


@pytest.mark.gpu
def test_sparse_every_cell_passes_grows_the_buffer(cuda_ready):
    # 1100 x 1000 hits exceed the first hit buffer (2^20): the call must rerun at the exact size.
    rng = np.random.default_rng(5)
    q, r = cdr3(rng, 1100, 10, 14), cdr3(rng, 1000, 10, 14)
    m = SubstitutionMatrix.blosum62()
    dense = oracle_dense(q, r, m, 8, 1, "none")
    sp = score_sparse(q, r, 10 ** 6, m, gap_open=8)
    assert sp.nnz == 1100 * 1000
    assert_same(sp, dense, 10 ** 6)
    np.testing.assert_array_equal(sp.to_dense(), dense)


@pytest.mark.gpu
def test_sparse_edge_cases(cuda_ready):
    m = SubstitutionMatrix.blosum62()
    e = score_sparse([], ["CASSF"], 5, m)
    assert e.shape == (0, 1) and e.nnz == 0 and e.indptr.tolist() == [0]
    e = score_sparse(["CASSF", "CF"], [], 5, m)
    assert e.shape == (2, 0) and e.indptr.tolist() == [0, 0, 0]
    none = score_sparse(["CASSLGQF"], ["WWWWWWWW"], 0, m)
    assert none.nnz == 0 and none.indptr.tolist() == [0, 0]
    with pytest.raises(ValueError, match="max_penalty must be >= 0"):
        score_sparse(["CASSF"], ["CASSF"], -1, m)
    with pytest.raises(ValueError, match="symbol 'J'"):
        score_sparse(["CASJF"], ["CASSF"], 5, m)
    with pytest.raises(ValueError, match="gap_open and gap_extend must be >= 0"):
        score_sparse(["CASSF"], ["CASSF"], 5, m, gap_open=-1)
    one = score_sparse(["CASSF", "CASSF"], ["CASSF", "CASF", "CASSF"], 0, m, gap_open=0,
                       gap_extend=0)
    dense = oracle_dense(["CASSF", "CASSF"], ["CASSF", "CASF", "CASSF"], m, 0, 0, "none")
    assert_same(one, dense, 0)
    assert one.row(1)[0].tolist() == np.nonzero(dense[1] <= 0)[0].tolist()
    with pytest.raises(IndexError):
        one.row(2)


@pytest.mark.gpu
def test_device_hits_match_the_host_call_and_the_dense_gpu_matrix(cuda_ready):
    import torch

    from seqtree_b200 import device
    rng = np.random.default_rng(17)
    q, r = cdr3(rng, 2000, 8, 25), cdr3(rng, 50000, 8, 25)
    r[::1000] = q[:50]
    m = SubstitutionMatrix.blosum62()
    qs, rs = device.SeqSet(q, "aa"), device.SeqSet(r, "aa")
    dense = torch.empty((len(q), len(r)), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    device.gapblock_into(qs, rs, dense.data_ptr(), stream, matrix=m, gap_open=8)
    hits = device.Hits()
    for thresh in (24, 30):  # the handle is refilled in place
        nnz = device.gapblock_sparse_into(qs, rs, hits, stream, max_penalty=thresh, matrix=m,
                                          gap_open=8)
        torch.cuda.synchronize()
        info = hits.info()
        assert (info["rows"], info["cols"], info["nnz"]) == (len(q), len(r), nnz)
        d = dense.cpu().numpy()
        indptr, ref_ids, scores = csr_of(d, thresh)
        assert nnz == ref_ids.size > 0
        assert info["indptr"] and info["ref_ids"] and info["scores"]
        got_ip, got_ri, got_sc = hits.to_host()
        np.testing.assert_array_equal(got_ip, indptr)
        np.testing.assert_array_equal(got_ri, ref_ids)
        np.testing.assert_array_equal(got_sc, scores)
        host = score_sparse(q, r, thresh, m, gap_open=8)
        np.testing.assert_array_equal(host.indptr, indptr)
        np.testing.assert_array_equal(host.ref_ids, ref_ids)
        np.testing.assert_array_equal(host.scores, scores)


@pytest.mark.gpu
@pytest.mark.parametrize("thresh", [40, 10 ** 6])
def test_sparse_in_row_blocks(cuda_ready, monkeypatch, thresh):
    # A sort cap of 1024 hits forces the row-block path; at 10**6 every row (1,300 hits) exceeds
    # the cap by itself and is taken alone.
    monkeypatch.setenv("SEQTREE_B200_SPARSE_BLOCK_HITS", "1024")
    rng = np.random.default_rng(23)
    q, r = cdr3(rng, 90, 8, 25), cdr3(rng, 1300, 8, 25)
    r[:30] = q[:30]
    m = SubstitutionMatrix.blosum62()
    dense = oracle_dense(q, r, m, 8, 1, "central21")
    from seqtree_b200 import device
    hits = device.Hits()
    qs, rs = device.SeqSet(q, "aa"), device.SeqSet(r, "aa")
    cube = np.asarray(prior_cube(prior_by_name("central21"), 25), np.int32).ravel()
    for _ in range(2):  # the second call starts from the first one's block size
        nnz = device.gapblock_sparse_into(qs, rs, hits, 0, max_penalty=thresh, matrix=m,
                                          gap_open=8, prior=cube, prior_width=25)
        indptr, ref_ids, scores = hits.to_host()
        want = csr_of(dense, thresh)
        assert nnz == want[1].size > 1024
        np.testing.assert_array_equal(indptr, want[0])
        np.testing.assert_array_equal(ref_ids, want[1])
        np.testing.assert_array_equal(scores, want[2])
    sp = score_sparse(q, r, thresh, m, gap_open=8, gap_prior=prior_by_name("central21"))
    assert_same(sp, dense, thresh)


def _junctions_packed(rng, n):
    """n CDR3-like junctions ('CASS' + uniform middle + 'F', lengths 8-25 with mode 14, wider on
    the long side) as packed bytes + offsets, built with numpy (no per-string Python work)."""
    from seqtree_b200 import _lib
    z = rng.standard_normal(n)
    lens = np.clip(np.rint(14 + np.where(z < 0, 2.5, 3.5) * z), 8, 25).astype(np.int64)
    off = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    aa = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", np.uint8)
    data = aa[rng.integers(0, 20, int(off[-1]))]
    pos = np.arange(int(off[-1])) - np.repeat(off[:-1], lens)
    data[pos < 4] = np.frombuffer(b"CASS", np.uint8)[pos[pos < 4]]
    data[pos == np.repeat(lens, lens) - 1] = ord("F")
    return _lib.Packed.from_arrays(data, off)


def _strings(p):
    raw = p.data.tobytes()
    return [raw[a:b].decode() for a, b in zip(p.offsets[:-1], p.offsets[1:])]


@pytest.mark.gpu
def test_full_size_sparse_configuration(cuda_ready):
    """The 100,000 x 1,000,000 sparse configuration (BLOSUM62, gap 8/1, max_penalty 24) at full
    size.  Every row is in ref order within the threshold; 24 sampled rows (rows are independent)
    equal the oracle's thresholded rows; a 64-row block equals the GPU's dense matrix thresholded."""
    import seqtree_b200 as stb
    rng = np.random.default_rng(0)
    refs = _junctions_packed(rng, 1_000_000)
    queries = _junctions_packed(np.random.default_rng(1), 100_000)
    m = SubstitutionMatrix.blosum62()
    sp = score_sparse(queries, refs, 24, m, gap_open=8)
    assert sp.shape == (100_000, 1_000_000) and sp.indptr[0] == 0
    assert np.all(np.diff(sp.indptr) >= 0) and sp.indptr[-1] == sp.nnz > 0
    assert sp.scores.min() >= 0 and sp.scores.max() <= 24
    starts = np.zeros(sp.nnz, bool)
    starts[sp.indptr[:-1][np.diff(sp.indptr) > 0]] = True
    step = np.diff(sp.ref_ids.astype(np.int64), prepend=-1)
    assert np.all((step > 0) | starts)
    qs, rs = _strings(queries), _strings(refs)
    rows = np.sort(rng.choice(100_000, 24, replace=False))
    dense = oracle.gapblock_matrix([qs[i] for i in rows], rs, m.penalty_grid, gap_open=8,
                                   gap_extend=1)
    for k, i in enumerate(rows):
        ids, sc = sp.row(int(i))
        want = np.flatnonzero(dense[k] <= 24)
        np.testing.assert_array_equal(ids, want)
        np.testing.assert_array_equal(sc, dense[k, want])
    block = np.asarray(stb.gapblock.score_matrix(qs[5000:5064], refs, m, gap_open=8))
    for k in range(64):
        ids, sc = sp.row(5000 + k)
        want = np.flatnonzero(block[k] <= 24)
        np.testing.assert_array_equal(ids, want)
        np.testing.assert_array_equal(sc, block[k, want])
