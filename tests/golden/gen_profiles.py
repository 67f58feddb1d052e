"""Golden vectors for the island-profile and E-value-cutoff rows, from the REFERENCE's own Python.

seqtree's IslandProfile (python/seqtree/gapblock.py) and thetas_from_scores
(python/seqtree/evalue.py) are pure Python; gapblock.py imports the compiled ``_core`` only for
names these functions do not use, so the module is loaded from the reference tree with a stub in
its place.  Run next to the reference tree:

    python tests/golden/gen_profiles.py [/path/to/seqtree]

It writes tests/golden/profiles.json: seeded islands with the reference's fitted profile
(penalties, width, c) and its scores for seeded query sets, plus seeded control-score rows with
the reference's per-query cutoffs.
"""
from __future__ import annotations

import importlib.util
import json
import sys
import types
from pathlib import Path

import numpy as np

if len(sys.argv) != 2:
    raise SystemExit("usage: gen_profiles.py <reference source tree>")
REF = Path(sys.argv[1])
OUT = Path(__file__).resolve().parent / "profiles.json"
AA20 = "ACDEFGHIKLMNPQRSTVWY"


def load_reference():
    pkg = types.ModuleType("seqtree")
    pkg.__path__ = [str(REF / "python" / "seqtree")]
    core = types.ModuleType("seqtree._core")
    for name in ("Index", "ScoreMatrix", "SearchParams", "SubstitutionMatrix", "gapblock_matrix"):
        setattr(core, name, object)
    sys.modules["seqtree"] = pkg
    sys.modules["seqtree._core"] = core
    mods = {}
    for name in ("gapblock", "evalue"):
        spec = importlib.util.spec_from_file_location(f"seqtree.{name}",
                                                      REF / "python" / "seqtree" / f"{name}.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[f"seqtree.{name}"] = mod
        spec.loader.exec_module(mod)
        mods[name] = mod
    return mods["gapblock"], mods["evalue"]


def junction(rng, lo, hi):
    L = int(rng.integers(lo, hi + 1))
    return "CASS" + "".join(rng.choice(list(AA20), size=L - 5)) + "F"


def island(rng, hub, n):
    out = []
    for _ in range(n):
        s = list(hub)
        for _ in range(int(rng.integers(0, 3))):
            s[int(rng.integers(4, len(s) - 1))] = AA20[int(rng.integers(0, 20))]
        if rng.random() < 0.3 and len(s) > 8:
            del s[int(rng.integers(4, len(s) - 1))]
        out.append("".join(s))
    return out


def main():
    gb, ev = load_reference()
    rng = np.random.default_rng(2024)
    cases = []
    for t in range(12):
        hub = junction(rng, 11, 18)
        members = island(rng, hub, int(rng.integers(1, 30)))
        kw = {}
        if t % 3 == 1:
            kw["c"] = int(rng.integers(0, min(map(len, members)) + 1))
        if t % 4 == 2:
            kw["lam"] = int(rng.integers(1, 5000))
            kw["pseudocount"] = float(rng.choice([0.1, 0.5, 2.0]))
        p = gb.IslandProfile.fit(members, **kw)
        queries = island(rng, hub, 40) + [junction(rng, 6, 24) for _ in range(40)] + \
            ["", "W" * 30, "CASSXZF", p.consensus()]
        cases.append({"members": members, "kwargs": kw, "width": p.width, "c": p.c,
                      "penalties": p.penalties, "consensus": p.consensus(), "queries": queries,
                      "scores": p.score_batch(queries)})
    rows = [sorted(int(x) for x in rng.integers(0, 60, size=int(rng.integers(0, 300))))
            for _ in range(200)] + [[], [0, 0, 3], [7] * 50]
    thetas = []
    for n, m, e, tmax in [(100, 100, 1.0, 10), (88, 250000, 0.05, 24), (20000, 250000, 0.05, 24),
                          (10, 100, 2.5, 30), (1, 1000, 0.004, 59)]:
        for ex in (False, True):
            thetas.append({"n_target": n, "m_control": m, "e_target": e, "theta_max": tmax,
                           "exclude_exact": ex,
                           "expected": ev.thetas_from_scores(rows, n, m, e, tmax, exclude_exact=ex)})
    OUT.write_text(json.dumps({"profiles": cases, "control_rows": rows, "thetas": thetas}))
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
