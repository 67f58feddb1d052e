"""Gotoh NW / SW score and distance matrices on the GPU, mirroring the invariant and known-answer
tests of the reference's tests/test_pairwise.py (its BioPython comparisons are replaced by the
reference's own C++ through the golden vectors)."""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
from conftest import as_np, rand_seqs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pw(cuda_ready):
    from seqtree_b200 import pairwise
    return pairwise


@pytest.fixture(scope="module")
def B62(cuda_ready):
    from seqtree_b200 import SubstitutionMatrix
    return SubstitutionMatrix.blosum62()


def test_golden_vectors(pw, golden_align):
    from seqtree_b200 import SubstitutionMatrix
    for case in golden_align:
        m = getattr(SubstitutionMatrix, case["matrix"])()
        fn = pw.dist_matrix if case["dist"] else pw.score_matrix
        if case["overflow"]:
            with pytest.raises(OverflowError, match="distance" if case["dist"] else "score"):
                fn(case["queries"], case["refs"], m, mode=case["mode"], gap_open=case["gap_open"],
                   gap_extend=case["gap_extend"])
            continue
        got = as_np(fn(case["queries"], case["refs"], m, mode=case["mode"],
                       gap_open=case["gap_open"], gap_extend=case["gap_extend"]))
        assert got.tolist() == case["expected"], case["name"]


def test_known_answers(pw, B62):
    assert pw.score("CASSLGQAYEQYF", "CASSPGQAYEQF", B62) == 45
    assert pw.score("CASSLGQAYEQYF", "CASSPGQAYEQF", B62, gap_open=12) == 44
    for L in (1, 2, 3, 5):
        assert pw.score("AAA", "AAA" + "A" * L, B62) == 12 - (11 + (L - 1))
    for L in (1, 2, 3):
        assert pw.score("AAA", "AAA" + "A" * L, B62, gap_open=5, gap_extend=5) == 12 - 5 * L
    assert pw.score("AAA", "KKAAA", B62) == 0
    assert pw.score("WWW", "KKK", B62, mode="local") == 0
    assert pw.score("WWWAAAWWW", "KKKAAAKKK", B62, mode="local") == 12
    assert pw.score("WWWAAAWWW", "KKKAAAKKK", B62, mode="global") < 0
    s = "CASSLGQAYEQYF"
    assert pw.score(s, s, B62, mode="local") == pw.score(s, s, B62, mode="global")


def test_huge_gaps_do_not_wrap(pw, B62):
    q, r = "CASSLGQAYEQYF", "CASSPGQAYEQF"
    assert pw.score(q, r, B62, gap_open=10 ** 8) == -99_999_944
    assert pw.score(q, r, B62, gap_open=2 ** 30) == -1_073_741_768
    assert pw.score(q, r, B62, gap_open=2 ** 31 - 1) == -2_147_483_591


def test_overflow_is_refused(pw, B62):
    with pytest.raises(OverflowError, match="32 bits"):
        pw.score("A" * 400, "W" * 600, B62, gap_open=2 ** 31 - 1, gap_extend=2 ** 31 - 1)
    for threads in (1, 0, 4):
        with pytest.raises(OverflowError):
            pw.score_matrix(["A" * 100], ["C"], B62, gap_open=10 ** 8, gap_extend=10 ** 8,
                            threads=threads)
        with pytest.raises(OverflowError):
            pw.dist_matrix(["A" * 100], ["C"], B62, gap_open=10 ** 8, gap_extend=10 ** 8,
                           threads=threads)
    with pytest.raises(OverflowError, match="distance"):
        pw.dist_matrix(["AAA"], ["C"], B62, gap_open=2 ** 31 - 1, gap_extend=2 ** 31 - 1)


def test_dist_is_a_distance_and_equals_the_gram_transform(pw, B62):
    rng = np.random.default_rng(19)
    seqs = rand_seqs(rng, 15, 10, 20)
    D = as_np(pw.dist_matrix(seqs, seqs, B62))
    assert (np.diagonal(D) == 0).all() and (D >= 0).all() and (D == D.T).all()
    q, r = rand_seqs(rng, 6, 8, 16), rand_seqs(rng, 5, 8, 16)
    D = as_np(pw.dist_matrix(q, r, B62))
    for i, a in enumerate(q):
        for j, b in enumerate(r):
            assert D[i, j] == pw.score(a, a, B62) + pw.score(b, b, B62) - 2 * pw.score(a, b, B62)


@pytest.mark.parametrize("mode", ["global", "local"])
@pytest.mark.parametrize("go,ge", [(11, 1), (5, 5), (1, 3), (0, 0), (1, 10)])
def test_against_oracle(pw, B62, mode, go, ge):
    rng = np.random.default_rng(hash((mode, go, ge)) & 0xFFFF)
    q, r = rand_seqs(rng, 23, 1, 40), rand_seqs(rng, 67, 1, 40)
    for dist in (False, True):
        fn = pw.dist_matrix if dist else pw.score_matrix
        got = as_np(fn(q, r, B62, mode=mode, gap_open=go, gap_extend=ge))
        exp = oracle.align_matrix(q, r, B62.similarity_grid, mode=mode, gap_open=go,
                                  gap_extend=ge, dist=dist, threads=os.cpu_count() or 1)
        assert np.array_equal(got, exp)


@pytest.mark.parametrize("mode", ["global", "local"])
def test_protein_lengths_against_oracle(pw, B62, mode):
    """Log-normal protein lengths (median 180, clipped 50-500), a block of the workload."""
    rng = np.random.default_rng(2)
    lens = np.clip(np.round(rng.lognormal(np.log(180), 0.5, size=40)), 50, 500).astype(int)
    seqs = ["".join(rng.choice(list("ACDEFGHIKLMNPQRSTVWY"), size=int(L))) for L in lens]
    q, r = seqs[:16], seqs[16:]
    got = as_np(pw.dist_matrix(q, r, B62, mode=mode))
    exp = oracle.align_matrix(q, r, B62.similarity_grid, mode=mode, dist=True,
                              threads=os.cpu_count() or 1)
    assert np.array_equal(got, exp)


def test_bad_arguments_raise(pw, B62):
    with pytest.raises(ValueError, match="gap_open"):
        pw.score("AA", "AA", B62, gap_open=-1)
    with pytest.raises(ValueError, match="mode"):
        pw.score("AA", "AA", B62, mode="semiglobal")
    with pytest.raises(ValueError, match="alphabet|symbol"):
        pw.score("AA#", "AA", B62)
    assert pw.score_matrix([], ["A"], B62).shape == (0, 1)
    assert pw.score("", "", B62) == 0
    assert pw.score("", "AAA", B62) == -(11 + 2)
    assert pw.score("", "AAA", B62, mode="local") == 0


@pytest.mark.parametrize("mode", ["global", "local"])
@pytest.mark.parametrize("dist", [False, True])
def test_short_pairs_thread_and_wavefront_paths(pw, B62, mode, dist):
    """Junction-length sets (all <= 32) take the one-thread-per-pair kernel or the wavefront,
    whichever the autotuner measured faster; the first call tunes (both run), the second runs
    the cached choice.  Both calls are bit-exact against the oracle, empty strings included, as
    are gap costs the int16 wavefront refuses (only the per-thread path takes those)."""
    from seqtree_b200 import _lib
    rng = np.random.default_rng(77 + dist + 2 * (mode == "local"))
    q = rand_seqs(rng, 300, 1, 30) + [""]
    r = rand_seqs(rng, 400, 1, 16) + ["", "W" * 32]
    fn = pw.dist_matrix if dist else pw.score_matrix
    want = oracle.align_matrix(q, r, B62.similarity_grid, mode=mode, dist=dist)
    for _ in range(2):
        got = as_np(fn(q, r, B62, mode=mode))
        np.testing.assert_array_equal(got, want)
    for go, ge in ((200, 30), (2000, 900)):
        want = oracle.align_matrix(q[:60], r[:70], B62.similarity_grid, mode=mode, gap_open=go,
                                   gap_extend=ge, dist=dist)
        got = as_np(fn(q[:60], r[:70], B62, mode=mode, gap_open=go, gap_extend=ge))
        np.testing.assert_array_equal(got, want)
    assert "align|" in _lib.tuning_table() or os.environ.get("SEQTREE_B200_TUNE") == "0"


_PER_THREAD_SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import oracle
from seqtree_b200 import SubstitutionMatrix, _lib, pairwise
AA20 = "ACDEFGHIKLMNPQRSTVWY"
def rand_seqs(rng, n, lo, hi):
    lens = rng.integers(lo, hi + 1, size=n)
    return ["".join(rng.choice(list(AA20), size=int(L))) for L in lens]
B62 = SubstitutionMatrix.blosum62()
rng = np.random.default_rng(91)
q = rand_seqs(rng, 120, 1, 32) + [""]
r = rand_seqs(rng, 150, 1, 32) + ["", "W" * 32]
checked = 0
for mode in ("global", "local"):
    for go, ge in ((5, 5), (1, 3), (11, 1), (0, 0)):
        for dist in (False, True):
            fn = pairwise.dist_matrix if dist else pairwise.score_matrix
            got = np.asarray(fn(q, r, B62, mode=mode, gap_open=go, gap_extend=ge))
            assert _lib.last_kernel_name() == "gotoh_thread_kernel", _lib.last_kernel_name()
            want = oracle.align_matrix(q, r, B62.similarity_grid, mode=mode, gap_open=go,
                                       gap_extend=ge, dist=dist)
            assert np.array_equal(got, want), (mode, go, ge, dist)
            checked += 1
print("per-thread checked", checked)
"""


def test_per_thread_kernel_branches_against_oracle(cuda_ready):
    """The one-thread-per-pair kernel on its own (tuning off, so its static choice runs for every
    set of sequences of at most 32 residues): global mode's raised single-H branch
    (gap_extend <= gap_open: 5/5, 11/1, 0/0), its three-state branch (gap_extend > gap_open:
    1/3) and local mode, score and distance, against the oracle."""
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, SEQTREE_B200_TUNE="0")
    res = subprocess.run([sys.executable, "-c", _PER_THREAD_SCRIPT, str(root)], env=env,
                         capture_output=True, text=True, timeout=600, cwd=str(root))
    assert res.returncode == 0, res.stdout + res.stderr
    assert "per-thread checked 16" in res.stdout


def test_gapblock_chunk_width_is_tuned_and_exact(cuda_ready):
    """The dense gap-block call times every chunk width once per shape and caches the fastest;
    every variant gives the same matrix (checked against the oracle on both calls)."""
    import seqtree_b200 as stb
    from conftest import cdr3
    from seqtree_b200 import _lib
    rng = np.random.default_rng(5)
    q, r = cdr3(rng, 257), cdr3(rng, 3001)
    m = stb.SubstitutionMatrix.blosum62()
    prior = stb.central_prior(21)
    width = max(map(len, q + r))
    want = oracle.gapblock_matrix(q, r, m.penalty_grid, gap_open=8,
                                  prior=stb.gapblock.prior_cube(prior, width), prior_width=width)
    for _ in range(2):
        got = np.asarray(stb.score_matrix(q, r, m, gap_open=8, gap_prior=prior))
        np.testing.assert_array_equal(got, want)
    assert "gapblock|" in _lib.tuning_table() or os.environ.get("SEQTREE_B200_TUNE") == "0"


@pytest.mark.parametrize("mode", ["global", "local"])
def test_full_size_protein_configuration(pw, B62, mode):
    """The 4,096 x 4,096 protein configuration (log-normal lengths, median 180, clipped 50-500;
    BLOSUM62, gap 11/1) at full size, distance form: six sampled rows (rows are independent)
    against the oracle, a zero diagonal where a query meets itself, and d >= 0 everywhere."""
    rng = np.random.default_rng(4096)
    lens = np.clip(np.round(rng.lognormal(np.log(180), 0.5, size=8192)), 50, 500).astype(int)
    aa = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", np.uint8)
    raw = aa[rng.integers(0, 20, int(lens.sum()))].tobytes().decode()
    cut = np.concatenate([[0], np.cumsum(lens)])
    seqs = [raw[a:b] for a, b in zip(cut[:-1], cut[1:])]
    q, r = seqs[:4096], seqs[4096:]
    r[17] = q[5]  # one self pair: distance 0
    got = as_np(pw.dist_matrix(q, r, B62, mode=mode))
    assert got.shape == (4096, 4096) and got.min() >= 0 and got[5, 17] == 0
    rows = [0, 5, 1000, 2047, 3333, 4095]
    exp = oracle.align_matrix([q[i] for i in rows], r, B62.similarity_grid, mode=mode, dist=True,
                              threads=os.cpu_count() or 1)
    assert np.array_equal(got[rows], exp)


def test_first_call_of_a_large_shape_tunes_on_a_slice(pw, B62):
    """5,000 x 5,000 junctions (2.5e7 pairs) is beyond the 2e7-pair tuning slice of the
    per-thread / wavefront choice: the first call tunes on the first 4,000 query rows, then runs
    the choice on everything.  Rows inside and past the slice are exact in both modes."""
    from conftest import cdr3
    rng = np.random.default_rng(73)
    q, r = cdr3(rng, 5000), cdr3(rng, 5000)
    for mode in ("global", "local"):
        first = as_np(pw.dist_matrix(q, r, B62, mode=mode))
        rows = [0, 3999, 4000, 4999]
        exp = oracle.align_matrix([q[i] for i in rows], r, B62.similarity_grid, mode=mode,
                                  dist=True, threads=os.cpu_count() or 1)
        assert np.array_equal(first[rows], exp)
        assert np.array_equal(first, as_np(pw.dist_matrix(q, r, B62, mode=mode)))


def test_first_call_of_a_long_shape_tunes_the_bucket_width_on_a_slice(pw, B62):
    """2,500 x 10,000 strings of 40-200 residues (2.5e7 pairs) is beyond the 2e7-pair slice on
    which the wavefront's row-bucket width (32 or 64 rows) is tuned: the first call tunes on the
    first 2,000 query rows, then runs the chosen width on everything.  Rows inside and past the
    slice are exact, and the second call (cached width) repeats the first."""
    rng = np.random.default_rng(79)
    q, r = rand_seqs(rng, 2500, 40, 200), rand_seqs(rng, 10000, 40, 200)
    for mode in ("global", "local"):
        first = as_np(pw.score_matrix(q, r, B62, mode=mode))
        rows = [0, 1999, 2000, 2499]
        exp = oracle.align_matrix([q[i] for i in rows], r, B62.similarity_grid, mode=mode,
                                  threads=os.cpu_count() or 1)
        assert np.array_equal(first[rows], exp)
        assert np.array_equal(first, as_np(pw.score_matrix(q, r, B62, mode=mode)))
    from seqtree_b200 import _lib
    assert "wave|" in _lib.tuning_table() or os.environ.get("SEQTREE_B200_TUNE") == "0"
