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
