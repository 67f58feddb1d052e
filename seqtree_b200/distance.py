"""Plain string edit distances: Hamming and Levenshtein, byte for byte, case-sensitive.

Mirrors seqtree's ``python/seqtree/distance.py`` (``hamming`` ``:37-58``, ``levenshtein``
``:61-78``, ``hamming_matrix`` ``:81-102``, ``levenshtein_matrix`` ``:105-119``).  Unit costs, no
substitution matrix, no alphabet.
"""
from __future__ import annotations

from collections.abc import Sequence

from ._core import hamming as _hamming
from ._core import hamming_matrix as _hamming_matrix
from ._core import levenshtein as _levenshtein
from ._core import levenshtein_matrix as _levenshtein_matrix
from .matrix import ScoreMatrix

__all__ = ["hamming", "levenshtein", "hamming_matrix", "levenshtein_matrix"]


def hamming(a: str, b: str) -> int:
    """Number of positions at which equal-length ``a`` and ``b`` differ (ValueError otherwise)."""
    return _hamming(a, b)


def levenshtein(a: str, b: str) -> int:
    """Fewest single-character insert / delete / substitute steps from ``a`` to ``b``."""
    return _levenshtein(a, b)


def hamming_matrix(a: Sequence[str], b: Sequence[str], threads: int = 0) -> ScoreMatrix:
    """Hamming distance of every ``a`` against every ``b``."""
    return _hamming_matrix(list(a), list(b), threads=threads)


def levenshtein_matrix(a: Sequence[str], b: Sequence[str], threads: int = 0) -> ScoreMatrix:
    """Levenshtein distance of every ``a`` against every ``b``; lengths may differ freely."""
    return _levenshtein_matrix(list(a), list(b), threads=threads)
