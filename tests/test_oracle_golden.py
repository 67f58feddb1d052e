"""The CPU oracle, pinned: against golden vectors produced by the reference's own C++ and
against the known answers the reference's tests hold for this path."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import load_golden, prior_by_name
from seqtree_b200.gapblock import prior_cube
from seqtree_b200.matrix import SubstitutionMatrix

MATRICES = ["blosum62", "blosum45", "blosum80", "pam250", "pam100", "structural"]


def _pen(name):
    if name is None:
        return None
    return getattr(SubstitutionMatrix, name)().penalty_grid


# --- tables --------------------------------------------------------------------------------

@pytest.mark.parametrize("name", MATRICES)
def test_package_tables_match_reference(golden_tables, name):
    m = getattr(SubstitutionMatrix, name)()
    g = golden_tables[name]
    assert m.similarity_grid.tolist() == g["sim"]
    assert m.penalty_grid.tolist() == g["pen"]
    assert m.scale() == g["scale"]


def test_oracle_gram_transform_matches_reference(golden_tables):
    for name in MATRICES:
        g = golden_tables[name]
        pen = oracle.penalty_from_similarity(np.array(g["sim"]), 24)
        assert pen.tolist() == g["pen"]
    u = golden_tables["unit4"]
    assert oracle.penalty_from_similarity(None, 4).tolist() == u["pen"]
    assert SubstitutionMatrix.unit(4).penalty_grid.tolist() == u["pen"]
    assert SubstitutionMatrix.unit(4).similarity_grid.tolist() == u["sim"]


def test_penalty_known_answers():
    """tests/cpp/test_matrix.cpp:13-39 and the documented scale() values."""
    b62 = SubstitutionMatrix.blosum62()
    assert b62.penalty("A", "R") == 11 and b62.penalty("W", "Y") == 14
    assert b62.penalty("A", "R") == b62.penalty("R", "A")
    assert SubstitutionMatrix.pam250().penalty("A", "E") == 6
    assert SubstitutionMatrix.pam100().penalty("A", "E") == 9
    assert SubstitutionMatrix.structural().penalty("A", "E") == 6
    assert b62.scale() == 14 and SubstitutionMatrix.structural().scale() == 7
    assert (b62.similarity("A", "A"), b62.similarity("W", "W")) == (4, 11)
    assert (SubstitutionMatrix.blosum45().similarity("A", "A"),
            SubstitutionMatrix.blosum45().similarity("W", "W")) == (5, 15)
    assert (SubstitutionMatrix.blosum80().similarity("A", "A"),
            SubstitutionMatrix.blosum80().similarity("W", "W")) == (7, 16)


def test_prior_known_answers():
    """python/seqtree/gapblock.py priors: test_gapblock.py known values."""
    from seqtree_b200.gapblock import central_prior, frame_prior, gap_cost, positions_prior
    cp = central_prior(21)
    assert cp(0, 1, 6) == 52 and cp(0, 2, 6) == 42 and cp(3, 0, 6) == 0
    assert frame_prior(21, 5)(2, 1, 10) == 63
    pp = positions_prior((3, 4, -4, -3))
    assert pp(3, 2, 12) == 0 and pp(5, 2, 12) == 1 << 20 and pp(6, 2, 12) == 0
    assert gap_cost(0, 1, 9) == 0 and gap_cost(1, 11, 1) == 11 and gap_cost(3, 11, 1) == 13
    with pytest.raises(ValueError):
        gap_cost(-1, 1, 1)


# --- gap block ------------------------------------------------------------------------------

def test_oracle_gapblock_golden(golden_gapblock):
    for case in golden_gapblock:
        q, r = case["queries"], case["refs"]
        width = max(map(len, q + r))
        prior = prior_by_name(case["prior"])
        cube = prior_cube(prior, width) if prior else None
        mat = case["matrix"]
        A = {"aa": 24, "nt": 4, "iupac": 15}[case["alphabet"]]
        pen = _pen(mat) if mat else oracle.penalty_from_similarity(None, A)
        got = oracle.gapblock_matrix(q, r, pen, alphabet=case["alphabet"],
                                     gap_open=case["gap_open"], gap_extend=case["gap_extend"],
                                     prior=cube, prior_width=width, threads=2)
        assert got.tolist() == case["expected"], case["name"]


def test_oracle_gapblock_brute_force():
    """Every layout enumerated independently (test_gapblock.py:36-54 restated) on small pairs."""
    rng = np.random.default_rng(7)
    pen = _pen("blosum62")
    AA = "ACDEFGHIKLMNPQRSTVWY"
    idx = {c: i for i, c in enumerate("ARNDCQEGHILKMFPSTWYVBZX*")}
    for _ in range(300):
        m = int(rng.integers(1, 16))
        n = int(rng.integers(1, 16))
        q = "".join(rng.choice(list(AA), m))
        r = "".join(rng.choice(list(AA), n))
        go, ge = [(1, 1), (4, 1), (28, 1), (0, 3), (2, 5)][int(rng.integers(0, 5))]
        d, L = abs(m - n), min(m, n)
        best = None
        for i in range(L + 1):
            head = sum(pen[idx[q[j]], idx[r[j]]] for j in range(i))
            if m >= n:
                tail = sum(pen[idx[q[j + d]], idx[r[j]]] for j in range(i, n))
            else:
                tail = sum(pen[idx[q[j]], idx[r[j + d]]] for j in range(i, m))
            best = head + tail if best is None else min(best, head + tail)
        expect = best + (0 if d == 0 else go + (d - 1) * ge)
        got = oracle.gapblock_matrix([q], [r], pen, gap_open=go, gap_extend=ge, threads=1)
        assert got[0, 0] == expect


def test_oracle_encode_errors():
    with pytest.raises(ValueError, match="alphabet"):
        oracle.encode(["CAS#"], "aa")
    codes, off = oracle.encode(["acgt", "ACGT"], "nt")
    assert codes[:8].tolist() == [0, 1, 2, 3, 0, 1, 2, 3]


# --- Gotoh ------------------------------------------------------------------------------------

def test_oracle_align_golden(golden_align):
    for case in golden_align:
        sim = getattr(SubstitutionMatrix, case["matrix"])().similarity_grid
        if case["overflow"]:
            with pytest.raises(OverflowError):
                oracle.align_matrix(case["queries"], case["refs"], sim, mode=case["mode"],
                                    gap_open=case["gap_open"], gap_extend=case["gap_extend"],
                                    dist=case["dist"], threads=2)
            continue
        got = oracle.align_matrix(case["queries"], case["refs"], sim, mode=case["mode"],
                                  gap_open=case["gap_open"], gap_extend=case["gap_extend"],
                                  dist=case["dist"], threads=2)
        assert got.tolist() == case["expected"], case["name"]


def test_oracle_align_known_answers():
    """test_pairwise.py:112-140, :213-226 and the pairwise.py doctests."""
    sim = SubstitutionMatrix.blosum62().similarity_grid

    def score(q, r, mode="global", go=11, ge=1):
        return int(oracle.align_matrix([q], [r], sim, mode=mode, gap_open=go, gap_extend=ge)[0, 0])

    assert score("CASSLGQAYEQYF", "CASSPGQAYEQF") == 45
    assert score("CASSLGQAYEQYF", "CASSPGQAYEQF", go=12) == 44
    assert score("WWWAAAWWW", "KKKAAAKKK", "local") == 12
    for L in (1, 2, 3, 5):
        assert score("AAA", "AAA" + "A" * L) == 12 - (11 + (L - 1))
        if L <= 3:
            assert score("AAA", "AAA" + "A" * L, go=5, ge=5) == 12 - 5 * L
    assert score("AAA", "KKAAA") == 12 - 12
    assert score("WWW", "KKK", "local") == 0
    assert score("CASSLGQAYEQYF", "CASSPGQAYEQF", go=10 ** 8) == -99_999_944
    assert score("CASSLGQAYEQYF", "CASSPGQAYEQF", go=2 ** 30) == -1_073_741_768
    assert score("CASSLGQAYEQYF", "CASSPGQAYEQF", go=2 ** 31 - 1) == -2_147_483_591
    assert score("", "") == 0 and score("", "AAA") == -(11 + 2) and score("", "AAA", "local") == 0
    with pytest.raises(OverflowError):
        oracle.align_matrix(["A" * 400], ["W" * 600], sim, gap_open=2 ** 31 - 1,
                            gap_extend=2 ** 31 - 1)


# --- distances -------------------------------------------------------------------------------

def test_oracle_distance_golden(golden_distance):
    for case in golden_distance:
        fn = oracle.levenshtein_matrix if case["kind"] == "levenshtein" else oracle.hamming_matrix
        assert fn(case["a"], case["b"], threads=2).tolist() == case["expected"], case["name"]


def test_oracle_distance_known_answers():
    """test_distance.py:40-71."""
    lev = lambda a, b: int(oracle.levenshtein_matrix([a], [b])[0, 0])  # noqa: E731
    ham = lambda a, b: int(oracle.hamming_matrix([a], [b])[0, 0])  # noqa: E731
    for a, b, d in [("kitten", "sitting", 3), ("flaw", "lawn", 2),
                    ("CASSLGQAYEQYF", "CASSPGQAYEQF", 2), ("", "", 0), ("abc", "", 3),
                    ("", "abc", 3), ("abc", "abc", 0), ("ABC", "abc", 3)]:
        assert lev(a, b) == d
    for a, b, d in [("AAAA", "AAAA", 0), ("AAAA", "ATAT", 2), ("CASSLGQYF", "CASSPGQYF", 1),
                    ("ABC", "abc", 3)]:
        assert ham(a, b) == d


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build not present")
def test_port_matches_reference_build_on_fresh_inputs():
    """The restatement and the reference C++ agree on inputs outside the fixtures."""
    rng = np.random.default_rng(2024)
    from conftest import cdr3, rand_seqs
    q, r = cdr3(rng, 30), cdr3(rng, 70)
    width = max(map(len, q + r))
    cube = prior_cube(prior_by_name("central21"), width)
    a = oracle.ref_gapblock_matrix(q, r, matrix="blosum62", gap_open=8, prior=cube,
                                   prior_width=width)
    b = oracle.gapblock_matrix(q, r, _pen("blosum62"), gap_open=8, prior=cube, prior_width=width)
    assert (a == b).all()
    q, r = rand_seqs(rng, 8, 20, 90), rand_seqs(rng, 9, 20, 90)
    sim = SubstitutionMatrix.blosum62().similarity_grid
    for mode in ("global", "local"):
        assert (oracle.ref_align_matrix(q, r, "blosum62", mode=mode, dist=True) ==
                oracle.align_matrix(q, r, sim, mode=mode, dist=True)).all()


# --- penalty alignment (Index::align) ------------------------------------------------------

def _index_pen(name):
    if name is None:
        return None
    return getattr(SubstitutionMatrix, name)().penalty_grid


def test_oracle_index_align_golden():
    """The port of Index::align (src/index.cpp:105-179) against the reference's own output on
    seeded pairs: unit cost and five matrices, gaps from free to 4e8, mixed case, empty sides."""
    g = load_golden("index_align")
    refs = g["refs"]
    for case in g["cases"]:
        pen = _index_pen(case["matrix"])
        for q, k, score, aq, ar, ops in case["pairs"]:
            got = oracle.penalty_align(q, refs[k], pen, case["gap_open"], case["gap_extend"])
            assert got == (score, aq, ar, ops), (case["matrix"], case["gap_open"], q, refs[k])


def test_oracle_index_align_known_answers():
    """Known answers of the reference's tests: tests/python/test_engine_guards.py:53-79,
    test_sanity.py:80-98 and test_matrix.py:27-40."""
    b62 = _index_pen("blosum62")
    ref = "CASSLGQAYEQYF"
    two_gaps = "CASSLGYEQYF"
    cheap = oracle.penalty_align(two_gaps, ref, b62, 11, 1)[0]
    dear = oracle.penalty_align(two_gaps, ref, b62, 11, 9)[0]
    assert dear - cheap == 8
    s, _, _, ops = oracle.penalty_align(two_gaps, ref, None, 1, 1)
    assert s == 2 and ops.count("I") + ops.count("D") == 2
    assert "I" in oracle.penalty_align("CASSIRSSYEQYF", ref, b62, 1, 1)[3]
    assert oracle.penalty_align("CASSIRSSYEQYF", ref, b62, 14, 1)[3] == "M" * 4 + "S" * 4 + "M" * 5
    for pen in (b62, None):
        assert oracle.penalty_align("casspgqayeqf", "CASSPGQAYEQF", pen, 1, 1)[0::3] == (0, "M" * 12)
    assert oracle.penalty_align("CASSPGQAYEQY", "CASSPGQAYEQF", b62, 28, 1)[3] == "M" * 11 + "S"
    with pytest.raises(ValueError, match=">= 0"):
        oracle.penalty_align("CASS", "CASS", None, -1, 1)


@pytest.mark.parametrize("name,expected", [("identity", 2), ("structural", 18), ("pam250", 24),
                                           ("blosum62", 28), ("pam100", 30)])
def test_oracle_index_align_matrix_scores(name, expected):
    """tests/python/test_matrix.py:27-40: with gap_open 100 the global alignment is the
    substitution-only score of the two junctions."""
    pen = SubstitutionMatrix.unit(24).penalty_grid if name == "identity" else _index_pen(name)
    assert oracle.penalty_align("CASSLAPGATNEKLFF", "CASSLELGATNEKLFF", pen, 100, 1)[0] == expected


# --- prior cubes (built by the reference's own Python) -------------------------------------

def _reachable(cube, width):
    w1 = width + 1
    return [cube[(m * w1 + d) * w1 + i] for m in range(w1) for d in range(1, m + 1)
            for i in range(m - d + 1)]


def _unreachable_zero(cube, width):
    w1 = width + 1
    live = {(m * w1 + d) * w1 + i for m in range(w1) for d in range(1, m + 1)
            for i in range(m - d + 1)}
    return all(v == 0 for k, v in enumerate(cube) if k not in live)


def test_prior_cubes_match_the_reference_python():
    """The library's prior_cube (every prior) and the oracle's restatement (central_prior)
    against cubes made by the reference's own central/frame/positions/profile priors and
    _prior_cube (python/seqtree/gapblock.py:79-185, 492-509)."""
    from seqtree_b200.gapblock import central_prior
    lams = {"central0": 0, "central1": 1, "central21": 21, "central33": 33}
    cases = load_golden("prior_cubes")
    assert len(cases) == 3 * 7
    for case in cases:
        name, width = case["prior"], case["width"]
        prior = central_prior(lams[name]) if name in lams else prior_by_name(name)
        cube = prior_cube(prior, width)
        assert len(cube) == (width + 1) ** 3
        assert _reachable(cube, width) == case["cells"], (name, width)
        assert _unreachable_zero(cube, width)
        if name in lams:
            ocube = oracle.prior_cube(oracle.central_prior(lams[name]), width)
            assert list(ocube) == list(cube), (name, width)
