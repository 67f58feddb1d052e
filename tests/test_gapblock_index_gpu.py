"""GapBlockIndex on the GPU against the reference's own index tests
(tests/python/test_gapblock.py:335-415 of seqtree) and against the oracle on random batches.

The reference's index returns, per ref within the budget and within d_max of the query's
length, the closed-form gap-block score (its test checks exactly that against the scorer), the
block length |m - n| and the block position; these tests check the same against the oracle's
dense matrix, and the position against a brute force over every block layout."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cdr3

pytestmark = pytest.mark.gpu

REFS = ["CASSLGQAYEQYF", "CASSLGQAYEQYFF", "CASSLGQAYEQY", "CASRQGAWDTQYF",
        "CAWSVSGGGTDTQYF", "CASSIRSSYEQYF", "CSARDRTGNGYTF", "CASSLAPGATNEKLF"]


@pytest.fixture(scope="module")
def gb(cuda_ready):
    import seqtree_b200 as stb
    return stb


def _closed_form(gb, q, r, pen, go, ge, prior):
    width = max(len(q), len(r))
    cube = gb.gapblock.prior_cube(prior, width) if prior is not None else []
    return int(oracle.gapblock_matrix([q], [r], pen, gap_open=go, gap_extend=ge, prior=cube,
                                      prior_width=width if prior is not None else 0)[0, 0])


def _brute_pos(q, r, pen_of, prior):
    """Smallest block position attaining the minimum (every layout enumerated)."""
    m, n = len(q), len(r)
    d = abs(m - n)
    if d == 0:
        return 0
    short = min(m, n)
    best, at = None, 0
    for i in range(short + 1):
        head = sum(pen_of(q[j], r[j]) for j in range(i))
        tail = (sum(pen_of(q[j + d], r[j]) for j in range(i, n)) if m > n
                else sum(pen_of(q[j], r[j + d]) for j in range(i, m)))
        v = head + tail + (prior(i, d, max(m, n)) if prior is not None else 0)
        if best is None or v < best:
            best, at = v, i
    return at


@pytest.mark.parametrize("with_prior", [False, True])
def test_index_search_matches_the_scorer_on_every_ref(gb, with_prior):
    B = gb.SubstitutionMatrix.blosum62()
    prior = gb.central_prior(20) if with_prior else None
    gbi = gb.GapBlockIndex(REFS, "aa", d_max=1)
    budget = 120
    for q in REFS + ["CASSLGQAYEQYW", "CASSLGQYEQYF", "CASSLGQAYEQYFFF"]:
        got = {rid: s for rid, s, _, _ in gbi.search(q, budget, B, gap_open=28, gap_prior=prior)}
        want = {}
        for rid, r in enumerate(REFS):
            if abs(len(q) - len(r)) > 1:
                continue
            s = _closed_form(gb, q, r, B.penalty_grid, 28, 1, prior)
            if s <= budget:
                want[rid] = s
        assert got == want, q


def test_index_finds_refs_both_shorter_and_longer(gb):
    B = gb.SubstitutionMatrix.blosum62()
    gbi = gb.GapBlockIndex(REFS, "aa", d_max=1)
    hits = {gbi.refs[rid]: (s, d) for rid, s, d, _ in gbi.search("CASSLGQAYEQYF", 200, B, gap_open=28)}
    assert hits["CASSLGQAYEQYF"] == (0, 0)
    assert hits["CASSLGQAYEQYFF"][1] == 1
    assert hits["CASSLGQAYEQY"][1] == 1


def test_index_zero_budget_returns_only_exact_matches(gb):
    B = gb.SubstitutionMatrix.blosum62()
    gbi = gb.GapBlockIndex(REFS, "aa", d_max=1)
    hits = gbi.search("CASSLGQAYEQYF", 0, B, gap_open=28)
    assert [gbi.refs[rid] for rid, *_ in hits] == ["CASSLGQAYEQYF"]


def test_index_dmax_zero_is_hamming(gb):
    B = gb.SubstitutionMatrix.blosum62()
    gbi = gb.GapBlockIndex(REFS, "aa", d_max=0)
    hits = gbi.search("CASSLGQAYEQYF", 200, B, gap_open=28)
    assert hits and all(len(gbi.refs[rid]) == 13 for rid, *_ in hits)


def test_index_rejects_bad_arguments(gb):
    B = gb.SubstitutionMatrix.blosum62()
    with pytest.raises(ValueError, match="d_max"):
        gb.GapBlockIndex(REFS, "aa", d_max=-1)
    with pytest.raises(ValueError, match="max_penalty"):
        gb.GapBlockIndex(REFS, "aa").search("CASSLGQAYEQYF", -1, B)


def test_index_len_and_unit_cost_default(gb):
    gbi = gb.GapBlockIndex(REFS, "aa", d_max=1)
    assert len(gbi) == len(REFS)
    hits = gbi.search("CASSLGQAYEQYF", 3, None)
    assert any(gbi.refs[rid] == "CASSLGQAYEQYF" and s == 0 for rid, s, _, _ in hits)


def test_index_skips_refs_shorter_than_the_block(gb):
    B = gb.SubstitutionMatrix.blosum62()
    gbi = gb.GapBlockIndex(["A", "CASSLGQAYEQYF"], "aa", d_max=2)
    hits = gbi.search("CASSLGQAYEQYF", 60, B, gap_open=28)
    assert [gbi.refs[rid] for rid, *_ in hits] == ["CASSLGQAYEQYF"]


def test_index_handles_short_refs_and_large_dmax(gb):
    gbi = gb.GapBlockIndex(["AC", "AG"], "aa", d_max=3)
    hits = gbi.search("AC", 5, None)
    assert hits[0][1] == 0 and gbi.refs[hits[0][0]] == "AC"


@pytest.mark.parametrize("d_max,with_prior", [(0, False), (2, False), (3, True)])
def test_search_batch_matches_the_oracle(gb, d_max, with_prior):
    """200 junction queries x 3,000 refs: every (ref, score) within the budget and d_max, in the
    reference's order (score, then ref id), block length |m - n|, block position the smallest
    minimising layout."""
    B = gb.SubstitutionMatrix.blosum62()
    rng = np.random.default_rng(d_max * 10 + with_prior)
    q, r = cdr3(rng, 200, 8, 22), cdr3(rng, 3000, 8, 22)
    prior = gb.central_prior(21) if with_prior else None
    budget = 40
    gbi = gb.GapBlockIndex(r, "aa", d_max=d_max)
    got = gbi.search_batch(q, budget, B, gap_open=8, gap_prior=prior)
    width = max(map(len, q + r))
    cube = gb.gapblock.prior_cube(prior, width) if prior is not None else []
    dense = oracle.gapblock_matrix(q, r, B.penalty_grid, gap_open=8, gap_extend=1, prior=cube,
                                   prior_width=width if prior is not None else 0)
    ql = np.array([len(s) for s in q])[:, None]
    rl = np.array([len(s) for s in r])[None, :]
    ok = (dense <= budget) & (np.abs(ql - rl) <= d_max)
    pen_of = lambda a, b: B.penalty(a, b)  # noqa: E731
    checked = 0
    for i in range(len(q)):
        ks = np.flatnonzero(ok[i])
        want = sorted(((int(k), int(dense[i, k])) for k in ks), key=lambda t: (t[1], t[0]))
        assert [(a, b) for a, b, _, _ in got[i]] == want, i
        for rid, s, d, p in got[i]:
            assert d == abs(len(q[i]) - len(r[rid]))
            if checked < 300:
                assert p == _brute_pos(q[i], r[rid], pen_of, prior), (q[i], r[rid])
                checked += 1
    assert checked > 0
