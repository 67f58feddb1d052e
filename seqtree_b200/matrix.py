"""Substitution matrices and the zero-copy result matrix.

``SubstitutionMatrix`` mirrors seqtree's class of the same name (``include/seqtree/seqtree.hpp:43-75``,
``src/substitution_matrix.cpp``, binding ``src/_bindings.cpp:240-317``): two views of one grid,
the raw signed similarity (maximised by Needleman-Wunsch / Smith-Waterman) and the non-negative
Gram penalty ``pen = s(a,a) + s(b,b) - 2 s(a,b)`` clamped at 0 (minimised by the gap-block score).

``ScoreMatrix`` mirrors the binding's result type (``src/_bindings.cpp:206-209,470-499``): a
read-only (rows, cols) int32 row-major block exported through the buffer protocol (format
``'i'``, C-contiguous), so ``numpy.asarray`` and ``memoryview`` wrap it without copying.
"""
from __future__ import annotations

import operator

import numpy as np

from ._tables import SIMILARITY

AMINO_ACIDS = "ARNDCQEGHILKMFPSTWYVBZX*"  # src/codec.cpp:9
ALPHABET_SYMBOLS = {0: AMINO_ACIDS, 1: "ACGT", 2: "ACGTRYSWKMBDHVN"}  # src/codec.cpp:9-11


def parse_alphabet(a: str) -> int:
    """The binding's alphabet names (src/_bindings.cpp:34-40)."""
    low = a.lower()
    if low in ("aa", "amino", "protein"):
        return 0
    if low in ("nt", "dna", "nucleotide"):
        return 1
    if low in ("nt_iupac", "iupac"):
        return 2
    raise ValueError(f"unknown alphabet '{a}' (use 'aa', 'nt', or 'iupac')")


def parse_align_mode(m: str) -> int:
    """The binding's mode names (src/_bindings.cpp:211-216)."""
    low = m.lower()
    if low in ("global", "nw", "needleman-wunsch"):
        return 0
    if low in ("local", "sw", "smith-waterman"):
        return 1
    raise ValueError(f"unknown mode '{m}' (use 'global' or 'local')")


def amino_acids() -> str:
    return AMINO_ACIDS


def alphabet_symbols(alphabet: str) -> str:
    return ALPHABET_SYMBOLS[parse_alphabet(alphabet)]


class SubstitutionMatrix:
    """Non-negative substitution penalties (penalty(a,a) == 0) plus the raw similarity."""

    __slots__ = ("_sim", "_pen")

    def __init__(self, sim: np.ndarray, pen: np.ndarray):
        self._sim = np.ascontiguousarray(sim, dtype=np.int32)
        self._pen = np.ascontiguousarray(pen, dtype=np.int32)

    # -- factories ---------------------------------------------------------------------------
    @classmethod
    def from_similarity(cls, grid) -> "SubstitutionMatrix":
        """Gram / squared-distance transform of a square similarity grid, clamped at 0."""
        rows = [list(r) for r in grid]
        n = len(rows)
        if n == 0 or n > 32:
            raise ValueError("matrix size must be 1..32")
        if any(len(r) != n for r in rows):
            raise ValueError("similarity matrix must be square")
        sim = np.array(rows, dtype=np.int64)
        if sim.min() < -(2 ** 31) or sim.max() >= 2 ** 31:
            raise TypeError("similarity entries must fit int32")
        sim = sim.astype(np.int32)
        d = np.diagonal(sim).astype(np.int64)
        pen = d[:, None] + d[None, :] - 2 * sim.astype(np.int64)
        pen = np.where(pen < 0, 0, pen).astype(np.int32)  # int32 wrap as in the reference
        return cls(sim, pen)

    @classmethod
    def unit(cls, size: int) -> "SubstitutionMatrix":
        """0 for a match, 1 for a mismatch; similarity +1/0 (src/substitution_matrix.cpp:15-27)."""
        eye = np.eye(size, dtype=np.int32)
        return cls(eye, 1 - eye)

    @classmethod
    def _named(cls, name: str) -> "SubstitutionMatrix":
        return cls.from_similarity(SIMILARITY[name])

    @classmethod
    def blosum62(cls):
        return cls._named("blosum62")

    @classmethod
    def blosum45(cls):
        return cls._named("blosum45")

    @classmethod
    def blosum80(cls):
        return cls._named("blosum80")

    @classmethod
    def pam250(cls):
        return cls._named("pam250")

    @classmethod
    def pam100(cls):
        return cls._named("pam100")

    @classmethod
    def structural(cls):
        return cls._named("structural")

    # -- views -------------------------------------------------------------------------------
    def size(self) -> int:
        return int(self._sim.shape[0])

    def _index(self, a: str, b: str, what: str) -> tuple[int, int]:
        if len(a) != 1 or len(b) != 1:
            raise ValueError(f"{what}() takes two single amino-acid characters")
        ia, ib = AMINO_ACIDS.find(a), AMINO_ACIDS.find(b)
        if ia < 0 or ib < 0:
            raise ValueError("unknown amino acid; expected one of " + AMINO_ACIDS)
        if ia >= self.size() or ib >= self.size():
            raise ValueError("residue out of range for this matrix's alphabet")
        return ia, ib

    def penalty(self, a: str, b: str) -> int:
        ia, ib = self._index(a, b, "penalty")
        return int(self._pen[ia, ib])

    def similarity(self, a: str, b: str) -> int:
        ia, ib = self._index(a, b, "similarity")
        return int(self._sim[ia, ib])

    def scale(self) -> int:
        """Median off-diagonal penalty (src/substitution_matrix.cpp:76-86): element n/2 of the
        sorted off-diagonal penalties."""
        n = self.size()
        if n < 2:
            return 0
        off = self._pen[~np.eye(n, dtype=bool)]
        return int(np.partition(off, off.size // 2)[off.size // 2])

    @property
    def penalty_grid(self) -> np.ndarray:
        return self._pen

    @property
    def similarity_grid(self) -> np.ndarray:
        return self._sim

    def __repr__(self) -> str:
        return f"SubstitutionMatrix(size={self.size()})"


def _unsigned_index(v) -> int:
    """``v`` as a size_t index: an integer (or an object with ``__index__``) that is not
    negative; a float, a string or a negative number is a TypeError, the way the reference's
    binding rejects an argument it cannot convert to ``size_t``."""
    try:
        i = operator.index(v)
    except TypeError:
        raise TypeError(f"index must be a non-negative integer, not {type(v).__name__}") from None
    if i < 0:
        raise TypeError("index must be a non-negative integer")
    return i


class ScoreMatrix:
    """A read-only (n_queries, n_refs) int32 matrix, row-major, exported by buffer protocol."""

    __slots__ = ("_a", "__weakref__")

    def __init__(self, array: np.ndarray):
        assert array.dtype == np.int32 and array.ndim == 2 and array.flags.c_contiguous
        array.flags.writeable = False
        self._a = array

    def __buffer__(self, flags):
        return memoryview(self._a)

    def __release_buffer__(self, view):
        pass

    def __array__(self, dtype=None, copy=None):
        if dtype is not None and np.dtype(dtype) != np.int32:
            return self._a.astype(dtype)
        return self._a

    @property
    def shape(self) -> tuple[int, int]:
        return (int(self._a.shape[0]), int(self._a.shape[1]))

    def __len__(self) -> int:
        return int(self._a.shape[0])

    def row(self, i: int) -> list[int]:
        i = _unsigned_index(i)
        if i >= self._a.shape[0]:
            raise IndexError("row out of range")
        return self._a[i].tolist()

    def __getitem__(self, ik):
        # a pair of unsigned indices, as the reference's std::pair<size_t, size_t> argument
        # takes: anything else (a scalar, three indices, a float, a negative) is a TypeError
        if isinstance(ik, (str, bytes)) or not hasattr(ik, "__len__") or len(ik) != 2:
            raise TypeError("ScoreMatrix indices must be a pair (i, k) of non-negative integers")
        i, k = (_unsigned_index(v) for v in ik)
        if i >= self._a.shape[0] or k >= self._a.shape[1]:
            raise IndexError("index out of range")
        return int(self._a[i, k])

    def __repr__(self) -> str:
        return f"ScoreMatrix({self._a.shape[0]}, {self._a.shape[1]})"
