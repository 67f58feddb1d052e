"""Generate tests/golden/index_align.json from the REFERENCE's own Index::align.

    make -C oracle && python tests/golden/gen_index_align.py

seqtree 0.6.0's Index::build + Index::align (src/index.cpp:91-179), compiled from its sources
by oracle/Makefile, aligns seeded queries (mixed case, ambiguity codes, empty strings) to
seeded references under unit cost and the built-in matrices, for gap settings from free gaps
to 4 x 10^8.  (Near 10^9 the reference's int32 recurrence overflows its INT32_MAX / 4 borders
and its traceback reads outside the strings, so no golden vector is taken there.)  Each case
stores its inputs and the reference's (score, aligned_query, aligned_ref, ops), so the tests
need no reference tree.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent
AA = "ACDEFGHIKLMNPQRSTVWY"


def junction(rng, lo, hi):
    L = int(rng.integers(lo, hi + 1))
    mid = "".join(rng.choice(list(AA), size=max(L - 5, 0)))
    return ("CASS" + mid + "F")[:L]


def mutate(rng, s):
    s = list(s)
    for _ in range(int(rng.integers(0, 4))):
        op = rng.integers(0, 3)
        if op == 0 and s:
            s[int(rng.integers(0, len(s)))] = str(rng.choice(list(AA + "BZX*")))
        elif op == 1:
            s.insert(int(rng.integers(0, len(s) + 1)), str(rng.choice(list(AA))))
        elif s:
            del s[int(rng.integers(0, len(s)))]
    out = "".join(s)
    return out.lower() if rng.random() < 0.15 else out


def main():
    rng = np.random.default_rng(2024)
    refs = [junction(rng, 6, 22) for _ in range(40)] + ["", "C", "cassLGQAYEQYF"]
    settings = [(None, 1, 1), (None, 11, 1), ("blosum62", 11, 1), ("blosum62", 28, 1),
                ("blosum62", 11, 9), ("pam250", 8, 3), ("structural", 0, 0), ("blosum45", 1, 1),
                ("blosum80", 100, 1), ("pam100", 20, 20), (None, 100000000, 1),
                ("blosum62", 400000000, 7)]
    cases = []
    for mat, go, ge in settings:
        pairs = []
        for _ in range(30):
            k = int(rng.integers(0, len(refs)))
            q = mutate(rng, refs[k]) if rng.random() < 0.7 else junction(rng, 0, 20)
            pairs.append((q, k))
        pairs.append(("", 0))
        pairs.append(("CASS", len(refs) - 3))  # against the empty reference
        out = []
        for q, k in pairs:
            out.append([q, k] + list(oracle.ref_index_align(refs, k, q, matrix=mat, gap_open=go,
                                                            gap_extend=ge)))
        cases.append({"matrix": mat, "gap_open": go, "gap_extend": ge, "pairs": out})
    (OUT / "index_align.json").write_text(json.dumps({"refs": refs, "cases": cases}, indent=0))


if __name__ == "__main__":
    main()
