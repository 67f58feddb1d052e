"""Per-query E-value cutoffs (thetas_from_scores, seqtree python/seqtree/evalue.py:102-143): the
oracle against the reference's docstring example and rules on CPU; the GPU kernel against the
oracle on random rows, on a SparseScores and on the device rows of the sparse gap-block kernel."""
from __future__ import annotations

import numpy as np
import pytest

import oracle


def test_oracle_known_answers():
    # the reference docstring: E(4) = (100/100)*1 = 1.0 is allowed; E(5) = 2.0 is not
    assert oracle.thetas_from_scores([[2, 5, 9]], 100, 100, 1.0, 10) == [4]
    # k < 1: one control hit already overshoots
    assert oracle.thetas_from_scores([[2, 5]], 100, 100, 0.5, 10) == [-1]
    # fewer than k + 1 hits: the ceiling itself
    assert oracle.thetas_from_scores([[1]], 10, 100, 1.0, 7) == [7]
    # exclude_exact drops the zero before counting
    assert oracle.thetas_from_scores([[0, 3, 4]], 100, 100, 1.0, 10, exclude_exact=True) == [3]
    assert oracle.thetas_from_scores([[0, 3, 4]], 100, 100, 1.0, 10) == [2]
    for bad, msg in [((0, 1, 1.0, 1), "n_target"), ((1, 1, 0.0, 1), "e_target"),
                     ((1, 1, 1.0, -1), "theta_max")]:
        with pytest.raises(ValueError, match=msg):
            oracle.thetas_from_scores([[1]], *bad)


@pytest.mark.gpu
def test_gpu_matches_the_oracle(cuda_ready):
    from seqtree_b200 import evalue
    rng = np.random.default_rng(3)
    rows = [list(rng.integers(0, 40, size=int(rng.integers(0, 400)))) for _ in range(700)]
    rows += [[], [0, 0, 0], [5] * 1000, [39, 38]]
    for n, m, e, tmax in [(100, 100, 1.0, 10), (88, 250000, 0.05, 24), (20000, 250000, 0.05, 24),
                          (10, 100, 2.5, 30), (1, 1000, 0.001, 39)]:
        for ex in (False, True):
            want = oracle.thetas_from_scores(rows, n, m, e, tmax, exclude_exact=ex)
            assert evalue.thetas_from_scores(rows, n, m, e, tmax, exclude_exact=ex) == want
    assert evalue.thetas_from_scores([[2, 5, 9]], 100, 100, 1.0, 10) == [4]
    with pytest.raises(ValueError, match="e_target"):
        evalue.thetas_from_scores([[1]], 1, 1, -1.0, 1)


@pytest.mark.gpu
def test_gpu_cutoffs_from_sparse_gapblock_rows(cuda_ready):
    """Cutoffs straight from the sparse kernel's device rows equal the oracle's on the same
    (exact) control scores."""
    import seqtree_b200 as stb
    from conftest import cdr3
    from seqtree_b200 import device, evalue
    rng = np.random.default_rng(8)
    q, ctrl = cdr3(rng, 150, 9, 18), cdr3(rng, 5000, 9, 18)
    B = stb.SubstitutionMatrix.blosum62()
    hits = device.Hits()
    device.gapblock_sparse_into(device.SeqSet(q), device.SeqSet(ctrl), hits, max_penalty=40,
                                matrix=B, gap_open=8)
    got = evalue.thetas_from_hits(hits, 200, 5000, 2.0, 40).cpu().numpy().tolist()
    ip, _, sc = hits.to_host()
    rows = [sc[a:b].tolist() for a, b in zip(ip[:-1], ip[1:])]
    assert got == oracle.thetas_from_scores(rows, 200, 5000, 2.0, 40)
    sp = stb.score_sparse(q, ctrl, 40, B, gap_open=8)
    assert evalue.thetas_from_scores(sp, 200, 5000, 2.0, 40) == got
