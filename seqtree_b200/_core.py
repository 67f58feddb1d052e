"""Drop-in for the hot-path functions of seqtree's compiled module ``_core``.

Same names, argument names, defaults, return types and exceptions as the reference binding
(seqtree ``src/_bindings.cpp:501-615``), computed on the GPU through the C ABI of
``libseqtree_b200.so``.  ``threads`` is accepted and ignored: the work runs on the current CUDA
device.  The scalar helpers (``align_score``, ``hamming``, ``levenshtein``) are 1 x 1 matrix
calls on the same kernels.
"""
from __future__ import annotations

import ctypes
import operator

import numpy as np

from . import _lib
from .matrix import ScoreMatrix, SubstitutionMatrix, parse_align_mode, parse_alphabet

__all__ = ["gapblock_matrix", "gapblock_sparse", "align_score_matrix", "align_dist_matrix", "hamming_matrix",
           "levenshtein_matrix", "align_score", "hamming", "levenshtein", "ScoreMatrix",
           "SubstitutionMatrix"]

_INT32 = (-(2 ** 31), 2 ** 31 - 1)


def _i32(name: str, v) -> int:
    """``v`` converted the way the reference binding's int32_t argument is: an integer or an
    object with ``__index__`` in range, else TypeError (a float or a string is never truncated
    or parsed)."""
    try:
        v = operator.index(v)
    except TypeError:
        raise TypeError(f"{name} must be an integer, not {type(v).__name__}") from None
    if not _INT32[0] <= v <= _INT32[1]:
        raise TypeError(f"{name} must fit a 32-bit signed integer")
    return v


def _u32(name: str, v) -> int:
    """As :func:`_i32` for a uint32_t argument: a negative value is a TypeError."""
    try:
        v = operator.index(v)
    except TypeError:
        raise TypeError(f"{name} must be an integer, not {type(v).__name__}") from None
    if not 0 <= v <= 0xFFFFFFFF:
        raise TypeError(f"{name} must fit a 32-bit unsigned integer")
    return v


def _result(rows: int, cols: int) -> np.ndarray:
    return _lib.pinned_int32(rows, cols)


def gapblock_matrix(queries, refs, alphabet: str = "aa", matrix: SubstitutionMatrix | None = None,
                    gap_open: int = 1, gap_extend: int = 1, prior=(), prior_width: int = 0,
                    threads: int = 0) -> ScoreMatrix:
    """Exhaustive single-gap-block penalties for every (query, ref) pair (GIL released).

    ``prior`` is the gap prior flattened to ``[m][d][i]``; see :func:`seqtree_b200.gapblock.score_matrix`,
    which builds it.
    """
    alph = parse_alphabet(alphabet)
    q, r = _lib.pack(queries), _lib.pack(refs)
    pen = None if matrix is None else np.ascontiguousarray(matrix.penalty_grid, np.int32)
    pr32 = _prior32(prior)
    out = _result(q.count, r.count)
    err = _lib.st_error()
    code = _lib.lib.st_gapblock_matrix(
        q.ref(), r.ref(), alph, _lib.i32_ptr(pen), 0 if pen is None else pen.shape[0],
        _i32("gap_open", gap_open), _i32("gap_extend", gap_extend),
        _lib.i32_ptr(pr32) if pr32.size else None, int(pr32.size), _u32("prior_width", prior_width),
        _i32("threads", threads), out.ctypes.data, ctypes.byref(err))
    _lib.check(code, err)
    return ScoreMatrix(out)


def _prior32(prior) -> np.ndarray:
    if isinstance(prior, np.ndarray) and prior.dtype == np.int32:
        return np.ascontiguousarray(prior).ravel()
    pr = np.ascontiguousarray(np.asarray(prior, dtype=np.int64), dtype=np.int64).ravel()
    if pr.size and (pr.min() < _INT32[0] or pr.max() > _INT32[1]):
        raise TypeError("prior entries must fit a 32-bit signed integer")
    return pr.astype(np.int32)


def gapblock_sparse(queries, refs, max_penalty: int, alphabet: str = "aa",
                    matrix: SubstitutionMatrix | None = None, gap_open: int = 1,
                    gap_extend: int = 1, prior=(), prior_width: int = 0, threads: int = 0):
    """The cells of :func:`gapblock_matrix` with score <= ``max_penalty``, as CSR arrays
    ``(indptr int64[N+1], ref_ids int32[nnz], scores int32[nnz])``; refs ascend within a row."""
    alph = parse_alphabet(alphabet)
    q, r = _lib.pack(queries), _lib.pack(refs)
    pen = None if matrix is None else np.ascontiguousarray(matrix.penalty_grid, np.int32)
    pr32 = _prior32(prior)
    res = _lib.st_sparse()
    err = _lib.st_error()
    code = _lib.lib.st_gapblock_sparse(
        q.ref(), r.ref(), alph, _lib.i32_ptr(pen), 0 if pen is None else pen.shape[0],
        _i32("gap_open", gap_open), _i32("gap_extend", gap_extend),
        _lib.i32_ptr(pr32) if pr32.size else None, int(pr32.size), _u32("prior_width", prior_width),
        _i32("max_penalty", max_penalty), _i32("threads", threads), ctypes.byref(res), ctypes.byref(err))
    _lib.check(code, err)
    # the arrays take over the library's pinned blocks (no copy of a possibly huge result)
    n, nnz = int(res.rows), int(res.nnz)
    indptr = _lib.adopt_pinned(res.indptr, n + 1, ctypes.c_int64, np.int64)
    ref_ids = _lib.adopt_pinned(res.ref_ids, nnz, ctypes.c_int32, np.int32)
    scores = _lib.adopt_pinned(res.scores, nnz, ctypes.c_int32, np.int32)
    return indptr, ref_ids, scores


def _align(queries, refs, matrix: SubstitutionMatrix, mode: str, gap_open: int, gap_extend: int,
           alphabet: str, dist: bool) -> ScoreMatrix:
    if not isinstance(matrix, SubstitutionMatrix):
        raise TypeError("matrix must be a SubstitutionMatrix")
    alph = parse_alphabet(alphabet)
    md = parse_align_mode(mode)
    q, r = _lib.pack(queries), _lib.pack(refs)
    sim = np.ascontiguousarray(matrix.similarity_grid, np.int32)
    out = _result(q.count, r.count)
    err = _lib.st_error()
    fn = _lib.lib.st_align_dist_matrix if dist else _lib.lib.st_align_score_matrix
    code = fn(q.ref(), r.ref(), _lib.i32_ptr(sim), sim.shape[0], alph, md,
              _i32("gap_open", gap_open), _i32("gap_extend", gap_extend), 0, out.ctypes.data,
              ctypes.byref(err))
    _lib.check(code, err)
    return ScoreMatrix(out)


def align_score_matrix(queries, refs, matrix: SubstitutionMatrix, mode: str = "global",
                       gap_open: int = 11, gap_extend: int = 1, alphabet: str = "aa",
                       threads: int = 0) -> ScoreMatrix:
    """Dense (n_queries, n_refs) similarity matrix, GIL released."""
    _i32("threads", threads)
    return _align(queries, refs, matrix, mode, gap_open, gap_extend, alphabet, False)


def align_dist_matrix(queries, refs, matrix: SubstitutionMatrix, mode: str = "global",
                      gap_open: int = 11, gap_extend: int = 1, alphabet: str = "aa",
                      threads: int = 0) -> ScoreMatrix:
    """Dense distance matrix d = s(a,a) + s(b,b) - 2*s(a,b); non-negative, zero on identity."""
    _i32("threads", threads)
    return _align(queries, refs, matrix, mode, gap_open, gap_extend, alphabet, True)


def _distance(a, b, lev: bool) -> ScoreMatrix:
    pa, pb = _lib.pack(a), _lib.pack(b)
    out = _result(pa.count, pb.count)
    err = _lib.st_error()
    fn = _lib.lib.st_levenshtein_matrix if lev else _lib.lib.st_hamming_matrix
    code = fn(pa.ref(), pb.ref(), 0, out.ctypes.data, ctypes.byref(err))
    _lib.check(code, err)
    return ScoreMatrix(out)


def hamming_matrix(a, b, threads: int = 0) -> ScoreMatrix:
    """Dense (len(a), len(b)) int32 Hamming matrix; ValueError if any pair differs in length."""
    _i32("threads", threads)
    return _distance(a, b, False)


def levenshtein_matrix(a, b, threads: int = 0) -> ScoreMatrix:
    """Dense (len(a), len(b)) int32 Levenshtein matrix."""
    _i32("threads", threads)
    return _distance(a, b, True)


def align_score(query: str, ref: str, matrix: SubstitutionMatrix, mode: str = "global",
                gap_open: int = 11, gap_extend: int = 1, alphabet: str = "aa") -> int:
    """Optimal similarity score of one pair ('global' NW, 'local' SW)."""
    return align_score_matrix([query], [ref], matrix, mode, gap_open, gap_extend, alphabet)[0, 0]


def hamming(a: str, b: str) -> int:
    """Number of differing positions of two equal-length sequences; case-sensitive."""
    return hamming_matrix([a], [b])[0, 0]


def levenshtein(a: str, b: str) -> int:
    """Unit-cost edit distance; case-sensitive."""
    return levenshtein_matrix([a], [b])[0, 0]


class Alignment:
    """An optimal alignment (seqtree's ``Alignment``, ``include/seqtree/types.hpp:67-72``):
    ``aligned_query`` / ``aligned_ref`` with ``-`` for gaps, ``ops`` per column ('M' match,
    'S' substitution, 'D' gap in the ref, 'I' gap in the query) and the similarity ``score``."""

    __slots__ = ("aligned_query", "aligned_ref", "ops", "score")

    def __init__(self, aligned_query: str, aligned_ref: str, ops: str, score: int):
        self.aligned_query, self.aligned_ref, self.ops, self.score = aligned_query, aligned_ref, ops, score

    def __repr__(self) -> str:
        return f"Alignment(score={self.score}, ops='{self.ops}')"


def align_pair(query: str, ref: str, matrix: SubstitutionMatrix, mode: str = "global",
               gap_open: int = 11, gap_extend: int = 1, alphabet: str = "aa") -> Alignment:
    """Optimal alignment of one pair with its traceback (``_core.align_pair``,
    src/_bindings.cpp:515-525), GIL released."""
    if not isinstance(matrix, SubstitutionMatrix):
        raise TypeError("matrix must be a SubstitutionMatrix")
    alph = parse_alphabet(alphabet)
    md = parse_align_mode(mode)
    qb, rb = query.encode("utf-8"), ref.encode("utf-8")
    sim = np.ascontiguousarray(matrix.similarity_grid, np.int32)
    cap = len(qb) + len(rb) + 1
    bufs = [ctypes.create_string_buffer(cap) for _ in range(3)]
    score = ctypes.c_int32(0)
    err = _lib.st_error()
    code = _lib.lib.st_align_pair(qb, len(qb), rb, len(rb), _lib.i32_ptr(sim), sim.shape[0], alph,
                                  md, _i32("gap_open", gap_open), _i32("gap_extend", gap_extend),
                                  ctypes.byref(score), bufs[0], bufs[1], bufs[2], cap,
                                  ctypes.byref(err))
    _lib.check(code, err)
    aq, ar, ops = (b.value.decode("utf-8") for b in bufs)
    return Alignment(aq, ar, ops, int(score.value))
