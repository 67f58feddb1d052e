"""Alignments with traceback (seqtree's align_pair, src/pairwise.cpp:141-267) on the GPU against
the reference's own C++ align_pair (oracle/_ref): scores, aligned strings and ops, identical."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cdr3, rand_seqs


def test_reference_align_pair_known_answers():
    """The reference's docstring examples (python/seqtree/pairwise.py:34-40, 104-110)."""
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    assert oracle.ref_align_pair("CASSLGQAYEQYF", "CASSPGQAYEQF")[1:3] == ("CASSLGQAYEQYF", "CASSPGQAYEQ-F")
    assert oracle.ref_align_pair("WWWAAAWWW", "KKKAAAKKK", mode="local")[:3] == (12, "AAA", "AAA")


def _check(pw, q, r, matrix, name, mode, go, ge, alphabet="aa"):
    got = pw.align_batch(q, r, matrix, mode=mode, gap_open=go, gap_extend=ge, alphabet=alphabet)
    for a, b, g in zip(q, r, got):
        want = oracle.ref_align_pair(a, b, name, mode=mode, gap_open=go, gap_extend=ge,
                                     alphabet=alphabet)
        assert (g.score, g.aligned_query, g.aligned_ref, g.ops) == want, (a, b)


@pytest.mark.gpu
def test_known_answers(cuda_ready):
    import seqtree_b200 as stb
    from seqtree_b200 import pairwise as pw
    m = stb.SubstitutionMatrix.blosum62()
    a = pw.align("CASSLGQAYEQYF", "CASSPGQAYEQF", m)
    assert (a.aligned_query, a.aligned_ref, a.score) == ("CASSLGQAYEQYF", "CASSPGQAYEQ-F", 45)
    a = pw.align("WWWAAAWWW", "KKKAAAKKK", m, mode="local")
    assert (a.score, a.aligned_query, a.aligned_ref) == (12, "AAA", "AAA")
    assert repr(a) == "Alignment(score=12, ops='MMM')"
    a = pw.align("WWW", "KKK", m, mode="local")
    assert (a.score, a.aligned_query, a.ops) == (0, "", "")


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["global", "local"])
@pytest.mark.parametrize("name,go,ge", [("blosum62", 11, 1), ("blosum45", 5, 5), ("pam250", 0, 0),
                                        ("blosum62", 1, 9), ("blosum80", 100000000, 1)])
def test_matches_the_reference(cuda_ready, mode, name, go, ge):
    import seqtree_b200 as stb
    from seqtree_b200 import pairwise as pw
    m = getattr(stb.SubstitutionMatrix, name)()
    rng = np.random.default_rng(hash((mode, name, go, ge)) & 0xFFFF)
    q = cdr3(rng, 120, 8, 25) + rand_seqs(rng, 20, 40, 160) + ["", "c", "CASS"]
    r = cdr3(rng, 120, 8, 25) + rand_seqs(rng, 20, 40, 160) + ["KKK", "", "cass"]
    ok, over = [], []
    for i in range(len(q)):
        try:
            oracle.ref_align_pair(q[i], r[i], name, mode=mode, gap_open=go, gap_extend=ge)
            ok.append(i)
        except OverflowError:
            over.append(i)
    for i in over[:5]:  # the reference refuses these; so must the GPU path
        with pytest.raises(OverflowError, match="32 bits"):
            pw.align(q[i], r[i], m, mode=mode, gap_open=go, gap_extend=ge)
    q, r = [q[i] for i in ok], [r[i] for i in ok]
    _check(pw, q, r, m, name, mode, go, ge)


@pytest.mark.gpu
def test_nucleotides_lowercase_and_pair_lists(cuda_ready):
    import seqtree_b200 as stb
    from seqtree_b200 import pairwise as pw
    rng = np.random.default_rng(12)
    nt = stb.SubstitutionMatrix.unit(4) if hasattr(stb.SubstitutionMatrix, "unit") else None
    if nt is not None:
        q = [s.lower() for s in rand_seqs(rng, 40, 5, 30, "ACGT")]
        r = rand_seqs(rng, 40, 5, 30, "ACGT")
        got = pw.align_batch(q, r, nt, gap_open=2, gap_extend=1, alphabet="nt")
        for a, b, g in zip(q, r, got):
            want = oracle.ref_align_pair(a, b, ("unit", 4), gap_open=2, gap_extend=1, alphabet="nt")
            assert (g.score, g.aligned_query, g.aligned_ref, g.ops) == want
    m = stb.SubstitutionMatrix.blosum62()
    qs, rs = cdr3(rng, 30), cdr3(rng, 50)
    qi = rng.integers(0, 30, 200)
    ri = rng.integers(0, 50, 200)
    got = pw.align_pairs(qs, rs, qi, ri, m)
    for i, k, g in zip(qi, ri, got):
        assert (g.score, g.aligned_query, g.aligned_ref, g.ops) == oracle.ref_align_pair(qs[i], rs[k])
    with pytest.raises(ValueError, match="gap_open"):
        pw.align("AAA", "AAA", m, gap_open=-1)
    with pytest.raises(ValueError):
        pw.align("AAJ", "AAA", m)


# --- penalty alignment: Index::align (src/index.cpp:105-179) --------------------------------

@pytest.mark.gpu
def test_penalty_align_matches_the_reference_golden_vectors(cuda_ready):
    """Every golden case of the reference's Index::align (tests/golden/index_align.json), one
    batched GPU call per setting: score, aligned strings and ops identical."""
    from conftest import load_golden
    from seqtree_b200.matrix import SubstitutionMatrix
    from seqtree_b200.pairwise import penalty_align_pairs
    g = load_golden("index_align")
    refs = g["refs"]
    for case in g["cases"]:
        mat = None if case["matrix"] is None else getattr(SubstitutionMatrix, case["matrix"])()
        qs = [p[0] for p in case["pairs"]]
        ks = [p[1] for p in case["pairs"]]
        got = penalty_align_pairs(qs, refs, np.arange(len(qs)), ks, mat,
                                  gap_open=case["gap_open"], gap_extend=case["gap_extend"])
        for (q, k, score, aq, ar, ops), a in zip(case["pairs"], got):
            assert (a.score, a.aligned_query, a.aligned_ref, a.ops) == (score, aq, ar, ops), \
                (case["matrix"], case["gap_open"], q, refs[k])


@pytest.mark.gpu
def test_penalty_align_known_answers_and_errors(cuda_ready):
    """The reference's tests of Index.align (tests/python/test_engine_guards.py:53-107,
    test_sanity.py:80-98, test_matrix.py:27-40), through the GPU entry point."""
    from seqtree_b200.matrix import SubstitutionMatrix
    from seqtree_b200.pairwise import penalty_align, penalty_align_pairs
    ref = "CASSLGQAYEQYF"
    two_gaps = "CASSLGYEQYF"
    cheap = penalty_align(two_gaps, ref, "BLOSUM62", gap_open=11, gap_extend=1)
    dear = penalty_align(two_gaps, ref, "BLOSUM62", gap_open=11, gap_extend=9)
    assert dear.score - cheap.score == 8
    lin = penalty_align(two_gaps, ref, gap_open=1, gap_extend=1)
    assert lin.score == 2 and lin.ops.count("I") + lin.ops.count("D") == 2
    m = SubstitutionMatrix.blosum62()
    assert "I" in penalty_align("CASSIRSSYEQYF", ref, m, gap_open=1).ops
    assert penalty_align("CASSIRSSYEQYF", ref, m, gap_open=m.scale()).ops == "M" * 4 + "S" * 4 + "M" * 5
    for mat in (m, None):
        a = penalty_align("casspgqayeqf", "CASSPGQAYEQF", mat)
        assert (a.score, a.ops, a.aligned_query) == (0, "M" * 12, "casspgqayeqf")
    assert penalty_align("CASSPGQAYEQY", "CASSPGQAYEQF", m, gap_open=2 * m.scale()).ops == "M" * 11 + "S"
    scores = {"identity": 2, "structural": 18, "PAM250": 24, "BLOSUM62": 28, "PAM100": 30}
    for name, want in scores.items():
        assert penalty_align("CASSLAPGATNEKLFF", "CASSLELGATNEKLFF", name, gap_open=100).score == want
    with pytest.raises(ValueError, match="invalid symbol '!' in query"):
        penalty_align("CASS!GQAYEQYF", ref)
    with pytest.raises(ValueError, match=">= 0"):
        penalty_align(two_gaps, ref, gap_open=-1)
    with pytest.raises(ValueError, match=r"invalid symbol '#' in reference #1"):
        penalty_align_pairs(["CASS"], ["CASS", "CA#S"], [0], [0])
    with pytest.raises(ValueError, match="matrix size does not match the alphabet"):
        penalty_align("ACGT", "ACGA", m, alphabet="nt")
    with pytest.raises(ValueError, match="unknown matrix"):
        penalty_align("CASS", "CASS", "BLOSUM99")
    with pytest.raises(IndexError):
        penalty_align_pairs(["CASS"], ["CASS"], [0], [1])
    assert penalty_align_pairs(["CASS"], ["CASS"], [], []) == []


@pytest.mark.gpu
def test_penalty_align_batches_match_the_port_and_the_reference(cuda_ready):
    """A seeded batch of junction pairs against the Python port, and long proteins (100-400
    residues, nucleotides too) against the reference's own Index::align."""
    from seqtree_b200.matrix import SubstitutionMatrix
    from seqtree_b200.pairwise import penalty_align_pairs
    rng = np.random.default_rng(31)
    qs, rs = cdr3(rng, 120, 6, 24), cdr3(rng, 90, 6, 24)
    qi = rng.integers(0, len(qs), 300)
    ri = rng.integers(0, len(rs), 300)
    pen = SubstitutionMatrix.pam250().penalty_grid
    got = penalty_align_pairs(qs, rs, qi, ri, SubstitutionMatrix.pam250(), gap_open=9, gap_extend=2)
    for a, i, k in zip(got, qi, ri):
        assert (a.score, a.aligned_query, a.aligned_ref, a.ops) == \
            oracle.penalty_align(qs[i], rs[k], pen, 9, 2)
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    for alphabet, pool, name in (("aa", None, "blosum62"), ("nt", "ACGTacgt", None)):
        if pool is None:
            lq, lr = rand_seqs(rng, 6, 100, 400), rand_seqs(rng, 5, 100, 400)
        else:
            lq, lr = rand_seqs(rng, 6, 100, 400, pool), rand_seqs(rng, 5, 100, 400, pool)
        mat = None if name is None else SubstitutionMatrix.blosum62()
        pi, pk = np.repeat(np.arange(6), 5), np.tile(np.arange(5), 6)
        got = penalty_align_pairs(lq, lr, pi, pk, mat, gap_open=11, gap_extend=1, alphabet=alphabet)
        for a, i, k in zip(got, pi, pk):
            want = oracle.ref_index_align(lr, k, lq[i], matrix=name, gap_open=11, gap_extend=1,
                                          alphabet=alphabet)
            assert (a.score, a.aligned_query, a.aligned_ref, a.ops) == want
