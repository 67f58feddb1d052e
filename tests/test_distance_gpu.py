"""Hamming / Levenshtein matrices on the GPU, mirroring tests/test_distance.py of the reference."""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
from conftest import AA20, as_np, rand_seqs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dist(cuda_ready):
    from seqtree_b200 import distance
    return distance


def test_golden_vectors(dist, golden_distance):
    for case in golden_distance:
        fn = dist.levenshtein_matrix if case["kind"] == "levenshtein" else dist.hamming_matrix
        got = as_np(fn(case["a"], case["b"]))
        assert got.dtype == np.int32 and got.tolist() == case["expected"], case["name"]


@pytest.mark.parametrize("a,b,d", [("kitten", "sitting", 3), ("flaw", "lawn", 2),
                                   ("CASSLGQAYEQYF", "CASSPGQAYEQF", 2), ("", "", 0),
                                   ("abc", "", 3), ("", "abc", 3), ("abc", "abc", 0),
                                   ("ABC", "abc", 3)])
def test_levenshtein_known(dist, a, b, d):
    assert dist.levenshtein(a, b) == d


@pytest.mark.parametrize("a,b,d", [("AAAA", "AAAA", 0), ("AAAA", "ATAT", 2),
                                   ("CASSLGQYF", "CASSPGQYF", 1), ("", "", 0), ("ABC", "abc", 3)])
def test_hamming_known(dist, a, b, d):
    assert dist.hamming(a, b) == d


def test_hamming_length_mismatch_raises(dist):
    with pytest.raises(ValueError, match="equal-length"):
        dist.hamming("AAAA", "AAA")
    with pytest.raises(ValueError, match=r"equal-length sequences \(got 3 and 4\)"):
        dist.hamming_matrix(["AAAA", "AAA"], ["AAAA"])
    with pytest.raises(ValueError, match=r"\(got 4 and 2\)"):
        dist.hamming_matrix(["AAAA", "AAA"], ["AAAA", "AA"])


@pytest.mark.parametrize("alphabet,L", [("AC", 33), ("ACGT", 12), ("ACGT", 64), (AA20, 12),
                                        (AA20 + AA20.lower() + "-*", 40), ("ACGT", 200)])
def test_hamming_against_oracle(dist, alphabet, L):
    rng = np.random.default_rng(L)
    a = rand_seqs(rng, 70, L, L, alphabet)
    b = rand_seqs(rng, 1027, L, L, alphabet)
    assert np.array_equal(as_np(dist.hamming_matrix(a, b)),
                          oracle.hamming_matrix(a, b, threads=os.cpu_count() or 1))


@pytest.mark.parametrize("alphabet,lo,hi", [("ACGT", 30, 60), ("ACGT", 0, 15), (AA20, 1, 64),
                                            ("ACGT", 50, 130), (AA20 + AA20.lower(), 0, 90)])
def test_levenshtein_against_oracle(dist, alphabet, lo, hi):
    rng = np.random.default_rng(hi)
    a = rand_seqs(rng, 45, lo, hi, alphabet)
    b = rand_seqs(rng, 301, lo, hi, alphabet)
    assert np.array_equal(as_np(dist.levenshtein_matrix(a, b)),
                          oracle.levenshtein_matrix(a, b, threads=os.cpu_count() or 1))


@pytest.mark.parametrize("alphabet,lo,hi,kernel", [
    ("ACGT", 65, 128, "levenshtein_kernel"),     # two 64-bit words per ref
    ("ACGT", 100, 256, "levenshtein_kernel"),    # four words, up to the last bit
    (AA20, 129, 200, "levenshtein_kernel"),      # four words, 20 symbols
    ("ACGT", 0, 140, "levenshtein_kernel"),      # empty and one-word refs beside four-word ones
    ("ACGT", 257, 512, "levenshtein_kernel"),    # eight words (small alphabets only)
    (AA20, 257, 300, "levenshtein_dp_kernel"),   # eight words of 20 symbols exceed the table
    ("ACGT", 513, 560, "levenshtein_dp_kernel"),  # past eight words: the DP kernel
])
def test_long_refs_take_the_blocked_bit_vector(dist, alphabet, lo, hi, kernel):
    """Refs longer than one 64-bit word run the blocked bit-vector form (each word hands its
    bottom horizontal step to the next); results equal the reference's two-row DP."""
    from seqtree_b200 import _lib
    rng = np.random.default_rng(lo * 1000 + hi)
    a = rand_seqs(rng, 23, lo, hi, alphabet)
    b = rand_seqs(rng, 77, lo, hi, alphabet)
    got = as_np(dist.levenshtein_matrix(a, b))
    assert _lib.last_kernel_name() == kernel
    assert np.array_equal(got, oracle.levenshtein_matrix(a, b, threads=os.cpu_count() or 1))


def test_many_distinct_bytes_take_the_dp_path(dist):
    rng = np.random.default_rng(9)
    alpha = "".join(chr(c) for c in range(33, 127))  # 94 distinct symbols
    a, b = rand_seqs(rng, 21, 0, 30, alpha), rand_seqs(rng, 37, 0, 30, alpha)
    assert np.array_equal(as_np(dist.levenshtein_matrix(a, b)), oracle.levenshtein_matrix(a, b))


def test_self_matrices_zero_diagonal_symmetric(dist):
    rng = np.random.default_rng(7)
    seqs = rand_seqs(rng, 20, 10, 10)
    h = as_np(dist.hamming_matrix(seqs, seqs))
    assert (h.diagonal() == 0).all() and (h == h.T).all()
    lev = rand_seqs(rng, 20, 0, 14)
    lv = as_np(dist.levenshtein_matrix(lev, lev))
    assert (lv.diagonal() == 0).all() and (lv == lv.T).all()


def test_bounds_property_at_full_size_rows(dist):
    """20,000 x 20,000 ACGT, lengths 30-60: a slice of rows checked exactly, every row checked
    against |m - n| <= lev <= max(m, n)."""
    rng = np.random.default_rng(0)
    b = rand_seqs(rng, 20000, 30, 60, "ACGT")
    a = rand_seqs(np.random.default_rng(1), 64, 30, 60, "ACGT")
    D = as_np(dist.levenshtein_matrix(a, b))
    la = np.array([len(s) for s in a])[:, None]
    lb = np.array([len(s) for s in b])[None, :]
    assert (D >= np.abs(la - lb)).all() and (D <= np.maximum(la, lb)).all()
    assert np.array_equal(D[:8], oracle.levenshtein_matrix(a[:8], b, threads=os.cpu_count() or 1))


def test_empty_inputs(dist):
    assert as_np(dist.hamming_matrix([], ["A"])).shape == (0, 1)
    assert as_np(dist.hamming_matrix(["A"], [])).shape == (1, 0)
    assert as_np(dist.levenshtein_matrix([], [])).shape == (0, 0)


def test_shared_memory_limit_only_grows_across_calls(dist):
    """The bit-vector kernel's shared memory grows with the alphabet.  A call on a large alphabet,
    then a small one, then the large one again must all launch (the per-kernel limit is raised,
    never lowered under a later, larger launch) -- the reference's own symmetric/bounds tests
    hit this order with random amino-acid strings."""
    rng = np.random.default_rng(44)
    big = AA20 + AA20.lower() + "0123456789"
    for alphabet in (big, "AC", big, "ACGT", big):
        a, b = rand_seqs(rng, 9, 0, 40, alphabet), rand_seqs(rng, 11, 0, 40, alphabet)
        assert np.array_equal(as_np(dist.levenshtein_matrix(a, b)), oracle.levenshtein_matrix(a, b))
    for _ in range(50):
        a, b = rand_seqs(rng, 1, 0, 15, AA20)[0], rand_seqs(rng, 1, 0, 15, AA20)[0]
        assert dist.levenshtein(a, b) == dist.levenshtein(b, a)
