"""Generate the golden vectors under tests/golden/ from the REFERENCE's own C++.

Run in a checkout next to the reference tree (it needs oracle/_ref/libseqtree_ref.so, which
oracle/Makefile builds from the reference sources, and the reference's Python package for the
gap-block priors):

    make -C oracle REF=<reference tree> && python tests/golden/gen_golden.py <reference tree>

Every expected matrix below is the output of seqtree 0.6.0's C++ (gapblock_matrix,
align_score_matrix / align_dist_matrix, hamming_matrix / levenshtein_matrix) on seeded inputs;
the inputs are stored beside it.  The tests compare both the CPU oracle and the CUDA library
with these files, so neither needs the reference tree at test time.

The prior cubes passed to the reference are built by the reference's own Python
(``python/seqtree/gapblock.py``: ``central_prior``, ``frame_prior``, ``positions_prior``,
``profile_prior`` and ``_prior_cube``), loaded from the reference tree with a stub in place of
its compiled ``_core``; ``prior_cubes.json`` keeps their reachable cells so that the library's
own ``prior_cube`` and the oracle's restatement are pinned against them.
"""
from __future__ import annotations

import importlib.util
import json
import sys
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

if len(sys.argv) != 2:
    raise SystemExit("usage: gen_golden.py <reference source tree>")
REF = Path(sys.argv[1])
OUT = Path(__file__).resolve().parent
AA20 = "ACDEFGHIKLMNPQRSTVWY"


def load_reference_gapblock():
    """The reference's python/seqtree/gapblock.py with a stub for its compiled ``_core`` (the
    priors and ``_prior_cube`` use none of its names)."""
    pkg = types.ModuleType("seqtree")
    pkg.__path__ = [str(REF / "python" / "seqtree")]
    core = types.ModuleType("seqtree._core")
    for name in ("Index", "ScoreMatrix", "SearchParams", "SubstitutionMatrix", "gapblock_matrix"):
        setattr(core, name, object)
    sys.modules["seqtree"] = pkg
    sys.modules["seqtree._core"] = core
    spec = importlib.util.spec_from_file_location("seqtree.gapblock",
                                                  REF / "python" / "seqtree" / "gapblock.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["seqtree.gapblock"] = mod
    spec.loader.exec_module(mod)
    return mod


GB = load_reference_gapblock()
prior_cube = GB._prior_cube


def rand_seqs(rng, n, lo, hi, alphabet=AA20):
    lens = rng.integers(lo, hi + 1, size=n)
    return ["".join(rng.choice(list(alphabet), size=int(L))) for L in lens]


def cdr3(rng, n, lo=10, hi=20):
    """'CASS' + uniform middle + 'F', total length uniform in [lo, hi]."""
    lens = rng.integers(lo, hi + 1, size=n)
    return ["CASS" + "".join(rng.choice(list(AA20), size=int(L) - 5)) + "F" for L in lens]


def tables():
    out = {}
    for name in ["blosum62", "blosum45", "blosum80", "pam250", "pam100", "structural"]:
        sim, pen, scale = oracle.ref_tables(name)
        out[name] = {"sim": sim.tolist(), "pen": pen.tolist(), "scale": int(scale)}
    sim, pen, scale = oracle.ref_tables(("unit", 4))
    out["unit4"] = {"sim": sim.tolist(), "pen": pen.tolist(), "scale": int(scale)}
    return out


PRIORS = {
    "none": None,
    "central21": GB.central_prior(21),
    "frame21_5": GB.frame_prior(21, 5),
    "positions": GB.positions_prior((3, 4, -4, -3)),
    "profile21": GB.profile_prior(21, lambda j, m: 1.0 - abs(2 * j + 1 - m) / m),
}


def reachable(cube, width):
    """The cells _prior_cube fills ([m][d][i], d >= 1, i <= m - d), in that order."""
    w1 = width + 1
    return [cube[(m * w1 + d) * w1 + i] for m in range(w1) for d in range(1, m + 1)
            for i in range(m - d + 1)]


def prior_cube_cases():
    """The reference's cubes for every prior at the widths the gap-block cases use, plus the
    CDR3 workloads' widths (20 and 25) and central_prior at lam 0, 1 and 33."""
    cases = []
    extra = {"central0": GB.central_prior(0), "central1": GB.central_prior(1),
             "central33": GB.central_prior(33)}
    for width in (7, 20, 25):
        for name, prior in list(PRIORS.items()) + list(extra.items()):
            if prior is None:
                continue
            cases.append({"prior": name, "width": width,
                          "cells": reachable(prior_cube(prior, width), width)})
    return cases


def gapblock_cases():
    cases = []
    rng = np.random.default_rng(7)
    seqs = rand_seqs(rng, 40, 4, 20)
    width = max(map(len, seqs))
    for pname, prior in PRIORS.items():
        cube = prior_cube(prior, width) if prior else []
        exp = oracle.ref_gapblock_matrix(seqs, seqs, matrix="blosum62", gap_open=28, gap_extend=1,
                                         prior=cube, prior_width=width)
        cases.append({"name": f"self40_{pname}", "queries": seqs, "refs": seqs,
                      "matrix": "blosum62", "alphabet": "aa", "gap_open": 28, "gap_extend": 1,
                      "prior": pname, "expected": exp.tolist()})
    # the workload shape: CDR3-like junctions, BLOSUM62, gap_open 8, central prior
    rng = np.random.default_rng(1)
    q = cdr3(rng, 48)
    r = cdr3(np.random.default_rng(0), 200)
    width = max(map(len, q + r))
    for pname in ("none", "central21", "positions"):
        prior = PRIORS[pname]
        cube = prior_cube(prior, width) if prior else []
        for mat, go in (("blosum62", 8), ("structural", 8)):
            exp = oracle.ref_gapblock_matrix(q, r, matrix=mat, gap_open=go, gap_extend=1,
                                             prior=cube, prior_width=width)
            cases.append({"name": f"cdr3_{mat}_{pname}", "queries": q, "refs": r, "matrix": mat,
                          "alphabet": "aa", "gap_open": go, "gap_extend": 1, "prior": pname,
                          "expected": exp.tolist()})
    # gap costs that exercise the d == 0 guard and gap_open < gap_extend
    rng = np.random.default_rng(11)
    q = rand_seqs(rng, 24, 1, 22)
    r = rand_seqs(rng, 30, 1, 22)
    for go, ge in ((0, 3), (2, 5), (5, 5), (0, 0), (1, 1)):
        exp = oracle.ref_gapblock_matrix(q, r, matrix="blosum62", gap_open=go, gap_extend=ge)
        cases.append({"name": f"gaps_{go}_{ge}", "queries": q, "refs": r, "matrix": "blosum62",
                      "alphabet": "aa", "gap_open": go, "gap_extend": ge, "prior": "none",
                      "expected": exp.tolist()})
    # unit cost on nucleotides and IUPAC, lower case mixed in (the codec folds case)
    rng = np.random.default_rng(5)
    q = rand_seqs(rng, 20, 0, 18, "ACGTacgt")
    r = rand_seqs(rng, 25, 0, 18, "ACGT")
    exp = oracle.ref_gapblock_matrix(q, r, alphabet="nt", matrix=None, gap_open=1, gap_extend=1)
    cases.append({"name": "unit_nt", "queries": q, "refs": r, "matrix": None, "alphabet": "nt",
                  "gap_open": 1, "gap_extend": 1, "prior": "none", "expected": exp.tolist()})
    q = rand_seqs(rng, 16, 1, 14, "ACGTRYSWKMBDHVN")
    r = rand_seqs(rng, 18, 1, 14, "ACGTRYSWKMBDHVN")
    exp = oracle.ref_gapblock_matrix(q, r, alphabet="iupac", matrix=None, gap_open=2, gap_extend=1)
    cases.append({"name": "unit_iupac", "queries": q, "refs": r, "matrix": None,
                  "alphabet": "iupac", "gap_open": 2, "gap_extend": 1, "prior": "none",
                  "expected": exp.tolist()})
    # long sequences (beyond the 64-residue fast path) and heavy penalties
    rng = np.random.default_rng(13)
    q = rand_seqs(rng, 10, 40, 120)
    r = rand_seqs(rng, 12, 30, 130)
    width = max(map(len, q + r))
    cube = prior_cube(PRIORS["central21"], width)
    exp = oracle.ref_gapblock_matrix(q, r, matrix="pam250", gap_open=30, gap_extend=2, prior=cube,
                                     prior_width=width)
    cases.append({"name": "long_pam250_central", "queries": q, "refs": r, "matrix": "pam250",
                  "alphabet": "aa", "gap_open": 30, "gap_extend": 2, "prior": "central21",
                  "expected": exp.tolist()})
    return cases


def align_cases():
    cases = []
    rng = np.random.default_rng(29)
    q = rand_seqs(rng, 14, 5, 25)
    r = rand_seqs(rng, 11, 5, 25)
    settings = [("global", 11, 1), ("global", 5, 5), ("global", 1, 3), ("global", 0, 0),
                ("global", 100, 5), ("local", 11, 1), ("local", 1, 10), ("local", 5, 5),
                ("global", 10 ** 8, 1), ("global", 2 ** 30, 1)]
    for mat in ("blosum62", "blosum45", "blosum80"):
        for mode, go, ge in settings:
            for dist in (False, True):
                try:
                    exp = oracle.ref_align_matrix(q, r, mat, mode=mode, gap_open=go,
                                                  gap_extend=ge, dist=dist).tolist()
                    err = None
                except OverflowError as e:
                    exp, err = None, str(e)
                cases.append({"name": f"{mat}_{mode}_{go}_{ge}_{'dist' if dist else 'score'}",
                              "queries": q, "refs": r, "matrix": mat, "mode": mode,
                              "gap_open": go, "gap_extend": ge, "dist": dist, "expected": exp,
                              "overflow": err})
    # protein-length sequences (the long path), both modes, score and distance
    rng = np.random.default_rng(3)
    q = rand_seqs(rng, 6, 50, 240)
    r = rand_seqs(rng, 7, 50, 240)
    for mode in ("global", "local"):
        for dist in (False, True):
            exp = oracle.ref_align_matrix(q, r, "blosum62", mode=mode, gap_open=11, gap_extend=1,
                                          dist=dist).tolist()
            cases.append({"name": f"protein_{mode}_{'dist' if dist else 'score'}", "queries": q,
                          "refs": r, "matrix": "blosum62", "mode": mode, "gap_open": 11,
                          "gap_extend": 1, "dist": dist, "expected": exp, "overflow": None})
    # empty sequences
    q = ["", "A", "CASSLGQAYEQYF"]
    r = ["", "AAA", "CASSPGQAYEQF"]
    for mode in ("global", "local"):
        exp = oracle.ref_align_matrix(q, r, "blosum62", mode=mode).tolist()
        cases.append({"name": f"empty_{mode}", "queries": q, "refs": r, "matrix": "blosum62",
                      "mode": mode, "gap_open": 11, "gap_extend": 1, "dist": False,
                      "expected": exp, "overflow": None})
    return cases


def distance_cases():
    cases = []
    rng = np.random.default_rng(5)
    a = rand_seqs(rng, 40, 12, 12)
    b = rand_seqs(rng, 30, 12, 12)
    cases.append({"name": "hamming_aa12", "kind": "hamming", "a": a, "b": b,
                  "expected": oracle.ref_distance_matrix(a, b, False).tolist()})
    a = rand_seqs(rng, 33, 12, 12, "ACGT")
    b = rand_seqs(rng, 37, 12, 12, "ACGT")
    cases.append({"name": "hamming_nt12", "kind": "hamming", "a": a, "b": b,
                  "expected": oracle.ref_distance_matrix(a, b, False).tolist()})
    a = rand_seqs(rng, 9, 70, 70, "ACGTacgtN-")
    b = rand_seqs(rng, 11, 70, 70, "ACGTacgtN-")
    cases.append({"name": "hamming_mixed70", "kind": "hamming", "a": a, "b": b,
                  "expected": oracle.ref_distance_matrix(a, b, False).tolist()})
    rng = np.random.default_rng(6)
    a = rand_seqs(rng, 35, 0, 15, "ACGT")
    b = rand_seqs(rng, 25, 0, 15, "ACGT")
    cases.append({"name": "lev_nt15", "kind": "levenshtein", "a": a, "b": b,
                  "expected": oracle.ref_distance_matrix(a, b, True).tolist()})
    a = rand_seqs(rng, 20, 30, 60, "ACGT")
    b = rand_seqs(rng, 24, 30, 60, "ACGT")
    cases.append({"name": "lev_nt30_60", "kind": "levenshtein", "a": a, "b": b,
                  "expected": oracle.ref_distance_matrix(a, b, True).tolist()})
    a = rand_seqs(rng, 12, 0, 80, AA20 + AA20.lower())
    b = rand_seqs(rng, 10, 50, 140, AA20 + AA20.lower())
    cases.append({"name": "lev_aa_long", "kind": "levenshtein", "a": a, "b": b,
                  "expected": oracle.ref_distance_matrix(a, b, True).tolist()})
    return cases


def main() -> None:
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libseqtree_ref.so is missing; run `make -C oracle` first")
    (OUT / "tables.json").write_text(json.dumps(tables()))
    (OUT / "gapblock.json").write_text(json.dumps(gapblock_cases()))
    (OUT / "align.json").write_text(json.dumps(align_cases()))
    (OUT / "distance.json").write_text(json.dumps(distance_cases()))
    (OUT / "prior_cubes.json").write_text(json.dumps(prior_cube_cases()))
    for f in sorted(OUT.glob("*.json")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
