"""Concurrent calls from several host threads.

The reference's matrix functions are reentrant and may be called from many threads at once
(`include/seqtree/seqtree.hpp:186-242`; the binding releases the GIL, `src/_bindings.cpp:
501-615`).  The drop-in keeps that contract: every C-ABI call owns its error record, and calls
on one device are serialised inside the library, so results and error messages must be the
ones a single-threaded caller sees.  ctypes releases the GIL around each call, so the threads
here really do enter the library together.
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

from conftest import AA20, as_np, cdr3, rand_seqs

pytestmark = pytest.mark.gpu


def _jobs(stb):
    from seqtree_b200 import distance, gapblock, pairwise
    rng = np.random.default_rng(41)
    q, r = cdr3(rng, 60), cdr3(rng, 90)
    b62 = stb.SubstitutionMatrix.blosum62()
    nt_a, nt_b = rand_seqs(rng, 50, 8, 40, "ACGT"), rand_seqs(rng, 70, 8, 40, "ACGT")
    ham_a, ham_b = rand_seqs(rng, 40, 12, 12, "ACGT"), rand_seqs(rng, 55, 12, 12, "ACGT")
    prot_a, prot_b = rand_seqs(rng, 12, 30, 120, AA20), rand_seqs(rng, 9, 30, 120, AA20)
    qi, ri = rng.integers(0, len(q), 40), rng.integers(0, len(r), 40)
    sparse = lambda: gapblock.score_sparse(q, r, 24, b62, gap_open=8)  # noqa: E731
    return {
        "gapblock": lambda: as_np(gapblock.score_matrix(q, r, b62, gap_open=8,
                                                        gap_prior=gapblock.central_prior(21))).copy(),
        "sparse": lambda: (lambda s: (s.indptr.copy(), s.ref_ids.copy(), s.scores.copy()))(sparse()),
        "levenshtein": lambda: as_np(distance.levenshtein_matrix(nt_a, nt_b)).copy(),
        "hamming": lambda: as_np(distance.hamming_matrix(ham_a, ham_b)).copy(),
        "nw_dist": lambda: as_np(pairwise.dist_matrix(prot_a, prot_b, b62)).copy(),
        "sw_score": lambda: as_np(pairwise.score_matrix(prot_a, prot_b, b62, mode="local")).copy(),
        "penalty_align": lambda: [(a.aligned_query, a.aligned_ref, a.ops, a.score) for a in
                                  pairwise.penalty_align_pairs(q, r, qi, ri, "blosum62", 8, 1)],
        "bad_symbol": lambda: _error_text(lambda: gapblock.score_matrix(q[:3] + ["CAS#F"], r[:4], b62)),
        "unequal_hamming": lambda: _error_text(lambda: distance.hamming_matrix(["ACGT"], ["ACG"])),
    }


def _error_text(call):
    try:
        call()
    except ValueError as e:
        return ("ValueError", str(e))
    return ("no error", "")


def _same(a, b) -> bool:
    if isinstance(a, np.ndarray):
        return isinstance(b, np.ndarray) and a.dtype == b.dtype and np.array_equal(a, b)
    if isinstance(a, tuple) and a and isinstance(a[0], np.ndarray):
        return all(_same(x, y) for x, y in zip(a, b))
    return a == b


def test_threads_get_the_single_threaded_results_and_errors(cuda_ready):
    import seqtree_b200 as stb
    jobs = _jobs(stb)
    want = {name: fn() for name, fn in jobs.items()}
    assert want["bad_symbol"][0] == "ValueError" and "'#'" in want["bad_symbol"][1]
    assert want["unequal_hamming"][0] == "ValueError" and "equal-length" in want["unequal_hamming"][1]

    names = list(jobs)
    failures: list[str] = []
    done = []

    def worker(t: int):
        try:
            for it in range(3):
                # each thread walks the jobs in its own rotation, so different kinds overlap
                for j in range(len(names)):
                    name = names[(j + 3 * t + it) % len(names)]
                    got = jobs[name]()
                    if not _same(want[name], got):
                        failures.append(f"thread {t} iteration {it}: {name} differs")
            done.append(t)
        except Exception as e:  # recorded and reported by the main thread
            failures.append(f"thread {t}: {type(e).__name__}: {e}")

    threads = [threading.Thread(target=worker, args=(t,), daemon=True) for t in range(6)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    assert not any(th.is_alive() for th in threads), "a thread did not finish within 300 s"
    assert not failures, failures[:5]
    assert sorted(done) == list(range(6))
