"""IslandProfile (seqtree python/seqtree/gapblock.py:208-380) and embed_in_frame: the host fit
and the oracle against golden vectors made by the reference's own Python
(tests/golden/gen_profiles.py), the reference's own profile tests
(tests/python/test_gapblock.py:283-291, 558-640), and the GPU scorer against both."""
from __future__ import annotations

import json
from pathlib import Path

import pytest

import oracle

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "profiles.json").read_text())
ISLAND = ["CASSLGQAYEQYF", "CASSLGQGYEQYF", "CASSPGQAYEQYF", "CASSLGQAYEQYF", "CASSLGKAYEQYF"]


def test_fit_reproduces_the_reference_profiles():
    from seqtree_b200.gapblock import IslandProfile
    for case in GOLDEN["profiles"]:
        p = IslandProfile.fit(case["members"], **case["kwargs"])
        assert (p.width, p.c) == (case["width"], case["c"])
        assert p.penalties == case["penalties"]
        assert p.consensus() == case["consensus"]


def test_oracle_scores_match_the_reference():
    for case in GOLDEN["profiles"]:
        got = [oracle.profile_score(case["penalties"], case["width"], case["c"], q)
               for q in case["queries"]]
        assert got == case["scores"]


def test_oracle_thetas_match_the_reference():
    rows = GOLDEN["control_rows"]
    for t in GOLDEN["thetas"]:
        assert oracle.thetas_from_scores(rows, t["n_target"], t["m_control"], t["e_target"],
                                         t["theta_max"], exclude_exact=t["exclude_exact"]) == t["expected"]


def test_embed_in_frame_round_trips():
    from seqtree_b200.gapblock import embed_in_frame
    assert embed_in_frame("CASSLF", 6, 3) == "CASSLF"
    assert embed_in_frame("CASLF", 6, 3) == "CAS-LF"
    for s, w, c in (("CASSLF", 5, 3), ("CASSLF", 8, 9)):
        with pytest.raises(ValueError):
            embed_in_frame(s, w, c)


def test_fit_rejects_bad_arguments_and_names_its_frame():
    from seqtree_b200.gapblock import IslandProfile
    with pytest.raises(ValueError, match="empty"):
        IslandProfile.fit([])
    with pytest.raises(ValueError, match="lam"):
        IslandProfile.fit(ISLAND, lam=-1)
    with pytest.raises(ValueError, match="pseudocount"):
        IslandProfile.fit(ISLAND, pseudocount=0)
    with pytest.raises(ValueError, match="outside"):
        IslandProfile.fit(ISLAND, c=99)
    p = IslandProfile.fit(ISLAND, c=4)
    assert repr(p) == "IslandProfile(width=13, c=4)"
    hub = "CASSLGQAYEQYF"
    assert IslandProfile.fit([hub] * 4 + [hub[:6] + hub[7:]]).c == 6


@pytest.mark.gpu
def test_gpu_scores_match_the_reference(cuda_ready):
    from seqtree_b200.gapblock import IslandProfile
    for case in GOLDEN["profiles"]:
        p = IslandProfile(case["penalties"], case["width"], case["c"])
        assert p.score_batch(case["queries"]) == case["scores"]


@pytest.mark.gpu
def test_gpu_thetas_match_the_reference(cuda_ready):
    from seqtree_b200 import evalue
    rows = GOLDEN["control_rows"]
    for t in GOLDEN["thetas"]:
        assert evalue.thetas_from_scores(rows, t["n_target"], t["m_control"], t["e_target"],
                                         t["theta_max"], exclude_exact=t["exclude_exact"]) == t["expected"]


@pytest.mark.gpu
def test_reference_profile_properties_on_the_gpu(cuda_ready):
    from seqtree_b200.gapblock import UNREACHABLE, IslandProfile
    p = IslandProfile.fit(ISLAND)
    assert p.score(p.consensus()) == 0
    assert all(p.score(s) >= 0 for s in ISLAND)
    assert IslandProfile.fit(["CASSLGQAYEQYF"]).score("CASSLGQAYEQYF") == 0
    m = IslandProfile.fit(["CASSA"] * 4 + ["CASSG"])
    assert m.score("CASSA") == 0 < m.score("CASSG") < m.score("CASSW")
    p4 = IslandProfile.fit(ISLAND, c=4)
    assert p4.score("CASSLGQAYEQYFFFFF") == UNREACHABLE
    assert p4.score("CAS") == UNREACHABLE
    assert p4.score("CASSLGQAYEQY") < UNREACHABLE
    big = IslandProfile.fit(ISLAND, lam=10 ** 9)
    assert 0 <= big.score("W" * big.width) < UNREACHABLE
    hub = "CASSLGQAYEQYF"
    assert IslandProfile.fit([hub] * 4 + [hub[:6] + hub[7:]]).score(hub) == 0
    seqs = ISLAND + ["CCCCCCCCCCCCC", "CASSLGQAYEQYFFF"]
    assert p.score_batch(seqs) == [p.score(s) for s in seqs]
