"""Needleman-Wunsch / Smith-Waterman with affine (Gotoh) gaps, maximising the raw similarity.

Mirrors seqtree's ``python/seqtree/pairwise.py`` (``score`` ``:53-85``, ``score_matrix``
``:119-136``, ``dist_matrix`` ``:139-167``).  Conventions: a gap run of length L costs
``gap_open + (L-1) * gap_extend``; ``gap_open == gap_extend`` is linear; global mode charges end
gaps; local mode floors the match state at 0 and takes the best cell anywhere.  Gap costs are
positive magnitudes that are subtracted.
"""
from __future__ import annotations

from collections.abc import Sequence

from ._core import align_dist_matrix as _dist_matrix
from ._core import align_score as _align_score
from ._core import align_score_matrix as _score_matrix
from .matrix import ScoreMatrix, SubstitutionMatrix

__all__ = ["score", "score_matrix", "dist_matrix"]


def score(query: str, ref: str, matrix: SubstitutionMatrix, mode: str = "global",
          gap_open: int = 11, gap_extend: int = 1, alphabet: str = "aa") -> int:
    """Optimal alignment score of ``query`` against ``ref`` (signed; higher is more similar)."""
    return _align_score(query, ref, matrix, mode=mode, gap_open=gap_open,
                        gap_extend=gap_extend, alphabet=alphabet)


def score_matrix(queries: Sequence[str], refs: Sequence[str], matrix: SubstitutionMatrix,
                 mode: str = "global", gap_open: int = 11, gap_extend: int = 1,
                 alphabet: str = "aa", threads: int = 0) -> ScoreMatrix:
    """Every query against every reference: a (len(queries), len(refs)) similarity matrix."""
    return _score_matrix(list(queries), list(refs), matrix, mode=mode, gap_open=gap_open,
                         gap_extend=gap_extend, alphabet=alphabet, threads=threads)


def dist_matrix(queries: Sequence[str], refs: Sequence[str], matrix: SubstitutionMatrix,
                mode: str = "global", gap_open: int = 11, gap_extend: int = 1,
                alphabet: str = "aa", threads: int = 0) -> ScoreMatrix:
    """Alignment distances ``d(a, b) = s(a,a) + s(b,b) - 2 s(a,b)``; zero on the diagonal."""
    return _dist_matrix(list(queries), list(refs), matrix, mode=mode, gap_open=gap_open,
                        gap_extend=gap_extend, alphabet=alphabet, threads=threads)
