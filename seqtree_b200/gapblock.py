"""Single-gap-block scoring for anchored loops (CDR3 / junction) -- the dense matrix path.

Mirrors the matrix-facing part of seqtree's ``python/seqtree/gapblock.py``: ``score_matrix``
(``:512-564``), the gap-prior builders ``central_prior`` (``:79-94``), ``profile_prior``
(``:97-125``), ``frame_prior`` (``:128-146``), ``positions_prior`` (``:149-185``), ``gap_cost``
(``:60-76``) and the ``[m][d][i]`` prior cube (``_prior_cube``, ``:492-509``).  The matrix itself
is computed by the CUDA library.

The score of a pair is a non-negative penalty: the block of length ``d = |len(q) - len(r)|`` is
placed at whichever of the ``min(len) + 1`` positions minimises substitution cost plus prior,
plus ``gap_open + (d-1) * gap_extend``; equal lengths score the plain substitution sum.
"""
from __future__ import annotations

from collections.abc import Callable, Iterable, Sequence

import numpy as np

from ._core import gapblock_matrix as _gapblock_matrix
from ._core import gapblock_sparse as _gapblock_sparse
from .matrix import ScoreMatrix, SubstitutionMatrix

__all__ = ["score_matrix", "score_sparse", "SparseScores", "central_prior", "profile_prior",
           "frame_prior", "positions_prior", "gap_cost", "ScoreMatrix", "UNREACHABLE"]

#: A prior large enough that no layout carrying it wins, small enough not to overflow int32
#: once a substitution cost is added (python/seqtree/gapblock.py:48-50).
UNREACHABLE = 1 << 20

#: ``prior(block_start, block_length, longer_length) -> int``; must be >= 0 and 0 at d == 0.
GapPrior = Callable[[int, int, int], int]


def gap_cost(d: int, gap_open: int, gap_extend: int) -> int:
    """Affine cost of one gap block of length ``d``; ``d == 0`` costs nothing."""
    if d < 0:
        raise ValueError("gap length must be >= 0")
    return 0 if d == 0 else gap_open + (d - 1) * gap_extend


def _cube_index(width: int):
    """(i, d, m) grids of the reachable cells of a width-``width`` cube (d >= 1, i <= m - d)."""
    w1 = width + 1
    m, d, i = np.meshgrid(np.arange(w1), np.arange(w1), np.arange(w1), indexing="ij")
    return i, d, m, (d >= 1) & (i <= m - d)


def central_prior(lam: int) -> GapPrior:
    """``lam * |block midpoint - m/2|`` as ``int(lam * |2i + d - m| // 2)``; 0 at d == 0."""
    if lam < 0:
        raise ValueError("lam must be >= 0")

    def prior(i: int, d: int, m: int) -> int:
        return 0 if d == 0 else int(lam * abs(2 * i + d - m) // 2)

    def cube(width: int) -> np.ndarray:
        # Same arithmetic as prior() in int64 (an int lam) or float64 (a float lam): a floor
        # division of a non-negative value, then truncation, exactly as int(...) of it.
        i, d, m, ok = _cube_index(width)
        x = np.abs(2 * i + d - m)
        v = (lam * x) // 2 if isinstance(lam, (int, np.integer)) else np.floor_divide(lam * x, 2)
        return np.where(ok, v, 0).astype(np.int64)

    prior.cube = cube
    return prior


def profile_prior(lam: int, w: Callable[[int, int], float] | Sequence[float]) -> GapPrior:
    """``int(lam * sum(w(j, m) for j in block))``: lam per unit of positional weight deleted."""
    if lam < 0:
        raise ValueError("lam must be >= 0")
    wfn = w if callable(w) else (lambda j, m: w[j])

    def prior(i: int, d: int, m: int) -> int:
        return int(lam * sum(wfn(j, m) for j in range(i, i + d)))

    return prior


def frame_prior(lam: int, c: int) -> GapPrior:
    """Pin the block to frame column ``c``: ``lam * |i - c|`` (0 at d == 0)."""
    if lam < 0:
        raise ValueError("lam must be >= 0")
    if c < 0:
        raise ValueError("c must be >= 0")

    def prior(i: int, d: int, m: int) -> int:
        return 0 if d == 0 else lam * abs(i - c)

    def cube(width: int) -> np.ndarray:
        i, d, m, ok = _cube_index(width)
        return np.where(ok, lam * np.abs(i - c), 0).astype(np.int64)

    if isinstance(lam, (int, np.integer)) and isinstance(c, (int, np.integer)):
        prior.cube = cube
    return prior


def positions_prior(starts: Iterable[int]) -> GapPrior:
    """Allow the block only at ``starts`` (negative = from the end of the shorter sequence,
    clamped into range); 0 at a permitted start, :data:`UNREACHABLE` elsewhere."""
    ss = tuple(starts)
    if not ss:
        raise ValueError("need at least one start position")

    def prior(i: int, d: int, m: int) -> int:
        if d == 0:
            return 0
        shorter = m - d
        for p in ss:
            allowed = min(p, shorter) if p >= 0 else max(0, shorter + p)
            if i == allowed:
                return 0
        return UNREACHABLE

    return prior


def _default_gap_open(matrix: SubstitutionMatrix | None) -> int:
    return 2 * matrix.scale() if matrix is not None else 1


def prior_cube(prior: GapPrior, width: int):
    """Flatten ``prior`` to ``[m][d][i]`` with stride ``width + 1``.

    Only reachable cells are filled -- ``d >= 1`` and ``i <= m - d`` -- the rest stay zero and
    are never read.  A negative prior value raises ValueError naming the cell.  The built-in
    central and frame priors fill the cube with numpy (same values); any other callable is
    evaluated cell by cell.
    """
    fast = getattr(prior, "cube", None)
    if fast is not None:
        c = fast(width)
        if (c < 0).any():
            mm, dd, ii = (int(x[0]) for x in np.nonzero(c < 0))
            raise ValueError(f"gap_prior({ii}, {dd}, {mm}) = {int(c[mm, dd, ii])} is negative")
        if c.max(initial=0) >= 2 ** 31:
            raise TypeError("prior entries must fit a 32-bit signed integer")
        return c.astype(np.int32).ravel()
    w1 = width + 1
    cube = [0] * (w1 * w1 * w1)
    for m in range(w1):
        for d in range(1, m + 1):
            base = (m * w1 + d) * w1
            for i in range(m - d + 1):
                v = int(prior(i, d, m))
                if v < 0:
                    raise ValueError(f"gap_prior({i}, {d}, {m}) = {v} is negative")
                cube[base + i] = v
    return cube


_prior_cube = prior_cube


def score_matrix(queries: Sequence[str], refs: Sequence[str],
                 matrix: SubstitutionMatrix | None = None, gap_open: int | None = None,
                 gap_extend: int = 1, gap_prior: GapPrior | None = None, alphabet: str = "aa",
                 threads: int = 0) -> ScoreMatrix:
    """Gap-block penalty of every query against every reference, on the GPU.

    ``gap_open`` defaults to ``2 * matrix.scale()`` (1 for unit cost).  ``gap_prior`` is
    materialised once into a lookup cube.  Returns a (len(queries), len(refs)) int32
    :class:`ScoreMatrix`; ``numpy.asarray`` wraps it without copying.
    """
    q, r = list(queries), list(refs)
    if gap_open is None:
        gap_open = _default_gap_open(matrix)
    if gap_open < 0 or gap_extend < 0:
        raise ValueError("gap_open and gap_extend must be >= 0")
    width = max(max(map(len, q), default=0), max(map(len, r), default=0))
    cube = prior_cube(gap_prior, width) if gap_prior is not None else []
    return _gapblock_matrix(q, r, alphabet, matrix, gap_open, gap_extend, cube, width, threads)


class SparseScores:
    """Thresholded gap-block matrix in CSR form: row ``i`` lists the refs ``k`` (ascending) whose
    score against query ``i`` is <= ``max_penalty``, with those scores.

    ``indptr`` (int64, rows + 1), ``ref_ids`` and ``scores`` (int32, nnz) are numpy arrays, the
    layout of ``scipy.sparse.csr_matrix((scores, ref_ids, indptr), shape)``.
    """

    def __init__(self, indptr, ref_ids, scores, shape, max_penalty: int):
        self.indptr, self.ref_ids, self.scores = indptr, ref_ids, scores
        self.shape = tuple(shape)
        self.max_penalty = max_penalty

    @property
    def nnz(self) -> int:
        return int(self.ref_ids.size)

    def row(self, i: int):
        """(ref_ids, scores) of query ``i``."""
        if not -self.shape[0] <= i < self.shape[0]:
            raise IndexError("row index out of range")
        i %= self.shape[0]
        a, b = int(self.indptr[i]), int(self.indptr[i + 1])
        return self.ref_ids[a:b], self.scores[a:b]

    def to_dense(self, fill: int = -1):
        """The (rows, cols) int32 matrix with ``fill`` where a cell did not pass."""
        out = np.full(self.shape, fill, np.int32)
        rows = np.repeat(np.arange(self.shape[0]), np.diff(self.indptr))
        out[rows, self.ref_ids] = self.scores
        return out

    def __repr__(self) -> str:
        return (f"SparseScores(shape={self.shape}, nnz={self.nnz}, "
                f"max_penalty={self.max_penalty})")


def score_sparse(queries: Sequence[str], refs: Sequence[str], max_penalty: int,
                 matrix: SubstitutionMatrix | None = None, gap_open: int | None = None,
                 gap_extend: int = 1, gap_prior: GapPrior | None = None, alphabet: str = "aa",
                 threads: int = 0) -> SparseScores:
    """Every (query, ref) pair with gap-block penalty <= ``max_penalty``, on the GPU.

    The same scores as :func:`score_matrix` (same arguments and defaults), keeping only the cells
    that pass the threshold, the way ``GapBlockIndex.search`` keeps its hits; nothing of size
    ``len(queries) * len(refs)`` is ever materialised, so it runs on sets whose dense matrix
    would not fit in memory (1e5 x 1e6 and beyond).  Raises ``ValueError`` when
    ``max_penalty < 0``.
    """
    if max_penalty < 0:
        raise ValueError("max_penalty must be >= 0")
    q, r = list(queries), list(refs)
    if gap_open is None:
        gap_open = _default_gap_open(matrix)
    if gap_open < 0 or gap_extend < 0:
        raise ValueError("gap_open and gap_extend must be >= 0")
    width = max(max(map(len, q), default=0), max(map(len, r), default=0))
    cube = prior_cube(gap_prior, width) if gap_prior is not None else []
    indptr, ref_ids, scores = _gapblock_sparse(q, r, max_penalty, alphabet, matrix, gap_open,
                                              gap_extend, cube, width, threads)
    return SparseScores(indptr, ref_ids, scores, (len(q), len(r)), max_penalty)
