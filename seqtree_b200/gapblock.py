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

from . import _lib
from ._core import gapblock_matrix as _gapblock_matrix
from ._core import gapblock_sparse as _gapblock_sparse
from .matrix import ScoreMatrix, SubstitutionMatrix

__all__ = ["score_matrix", "score_sparse", "SparseScores", "central_prior", "profile_prior",
           "frame_prior", "positions_prior", "gap_cost", "gapblock_score", "deletion_variants",
           "ScoreMatrix", "UNREACHABLE"]

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
        # The built-in priors are pure functions of their parameters, so a cube is built and
        # checked once per width and kept on the prior (read-only).
        memo = prior.__dict__.setdefault("_cube_memo", {})
        hit = memo.get(width)
        if hit is not None:
            return hit
        c = fast(width)
        if (c < 0).any():
            mm, dd, ii = (int(x[0]) for x in np.nonzero(c < 0))
            raise ValueError(f"gap_prior({ii}, {dd}, {mm}) = {int(c[mm, dd, ii])} is negative")
        if c.max(initial=0) >= 2 ** 31:
            raise TypeError("prior entries must fit a 32-bit signed integer")
        out = c.astype(np.int32).ravel()
        out.flags.writeable = False
        if len(memo) < 16:
            memo[width] = out
        return out
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


def deletion_variants(q: str, d: int) -> list[tuple[int, str]]:
    """``q`` with one contiguous run of ``d`` residues removed, for every start of the run, as
    ``(block_position, variant)`` (python/seqtree/gapblock.py:383-400).  ``d == 0`` removes
    nothing and gives the single pair ``(0, q)``; ``d`` outside ``[0, len(q)]`` raises
    ValueError."""
    if not 0 <= d <= len(q):
        raise ValueError(f"cannot delete {d} residues from a length-{len(q)} sequence")
    if d == 0:
        return [(0, q)]
    return [(start, q[:start] + q[start + d:]) for start in range(len(q) + 1 - d)]


_PAIR_SYMBOLS = "ARNDCQEGHILKMFPSTWYVBZX*"  # the amino-acid codec's 24 symbols


def gapblock_score(q: str, r: str, matrix: SubstitutionMatrix | None = None,
                   gap_open: int | None = None, gap_extend: int = 1,
                   gap_prior: GapPrior | None = None,
                   _pen: dict | None = None) -> tuple[int, int]:
    """``(score, block_position)`` of one pair (python/seqtree/gapblock.py:413-489), from the exact
    pair kernel on the GPU.

    Penalties are looked up on the characters themselves, as the reference's scalar scorer does:
    ``_pen[(a, b)]`` when given, else ``matrix.penalty(a, b)``, else unit cost ``a != b``
    (case-sensitive).  The pair's distinct characters (at most 24) are renamed to codec symbols
    and scored with that table.  ``block_position`` indexes the shorter sequence (0 to
    ``min(m, n)``) and is the first position that attains the minimum; it is 0 for equal
    lengths.
    """
    import ctypes

    import torch

    from . import device
    if gap_open is None:
        gap_open = _default_gap_open(matrix)
    if gap_open < 0 or gap_extend < 0:
        raise ValueError("gap_open and gap_extend must be >= 0")
    syms = sorted(set(q) | set(r))
    if len(syms) > len(_PAIR_SYMBOLS):
        raise ValueError("gapblock_score: more than 24 distinct symbols in one pair")
    if _pen is not None:
        pen = lambda a, b: _pen[a, b]  # noqa: E731
    elif matrix is not None:
        pen = matrix.penalty
    else:
        pen = lambda a, b: int(a != b)  # noqa: E731
    grid = np.zeros((24, 24), np.int32)
    for i, a in enumerate(syms):
        for j, b in enumerate(syms):
            grid[i, j] = pen(a, b)
    rename = str.maketrans({c: _PAIR_SYMBOLS[i] for i, c in enumerate(syms)})
    width = max(len(q), len(r))
    cube = np.asarray(prior_cube(gap_prior, width) if gap_prior is not None else [],
                      dtype=np.int64).astype(np.int32).ravel()
    qs = device.SeqSet([q.translate(rename)], "aa")
    rs = device.SeqSet([r.translate(rename)], "aa")
    idx = torch.zeros(2, dtype=torch.int32, device="cuda")
    res = torch.empty(2, dtype=torch.int32, device="cuda")
    err = _lib.st_error()
    _lib.check(_lib.lib.st_gapblock_pairs_pos_sets(
        qs.handle, rs.handle, ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(idx.data_ptr() + 4),
        1, _lib.i32_ptr(grid), 24, gap_open, gap_extend,
        _lib.i32_ptr(cube) if cube.size else None, int(cube.size), width if cube.size else 0,
        ctypes.c_void_p(res.data_ptr()), ctypes.c_void_p(res.data_ptr() + 4),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(err)), err)
    score, pos = res.tolist()
    return int(score), int(pos)


def score_matrix(queries: Sequence[str], refs: Sequence[str],
                 matrix: SubstitutionMatrix | None = None, gap_open: int | None = None,
                 gap_extend: int = 1, gap_prior: GapPrior | None = None, alphabet: str = "aa",
                 threads: int = 0) -> ScoreMatrix:
    """Gap-block penalty of every query against every reference, on the GPU.

    ``gap_open`` defaults to ``2 * matrix.scale()`` (1 for unit cost).  ``gap_prior`` is
    materialised once into a lookup cube.  Returns a (len(queries), len(refs)) int32
    :class:`ScoreMatrix`; ``numpy.asarray`` wraps it without copying.
    """
    if gap_open is None:
        gap_open = _default_gap_open(matrix)
    if gap_open < 0 or gap_extend < 0:
        raise ValueError("gap_open and gap_extend must be >= 0")
    q, r = _lib.pack(queries), _lib.pack(refs)
    width = max(q.max_len, r.max_len)
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
    if gap_open is None:
        gap_open = _default_gap_open(matrix)
    if gap_open < 0 or gap_extend < 0:
        raise ValueError("gap_open and gap_extend must be >= 0")
    q, r = _lib.pack(queries), _lib.pack(refs)
    width = max(q.max_len, r.max_len)
    cube = prior_cube(gap_prior, width) if gap_prior is not None else []
    indptr, ref_ids, scores = _gapblock_sparse(q, r, max_penalty, alphabet, matrix, gap_open,
                                              gap_extend, cube, width, threads)
    return SparseScores(indptr, ref_ids, scores, (q.count, r.count), max_penalty)


class GapBlockIndex:
    """Thresholded single-gap-block search over a reference set, on the GPU.

    The reference's ``GapBlockIndex`` (``python/seqtree/gapblock.py:567-673``) reaches refs of
    length ``len(query) +- d`` for ``d <= d_max`` through Hamming searches over deletion
    variants, and returns every ref within ``max_penalty`` with its best gap-block score.  That
    score is the closed form of ``score_matrix`` (one block of ``|m - n|`` residues in the longer
    sequence, prior only when ``d > 0``), so here a search is the exhaustive sparse kernel over
    the batch (``score_sparse``), restricted to ``|m - n| <= d_max``, with the block position
    taken from the exact pair kernel.  Build once, search many -- ``search_batch`` answers many
    queries in one pass, which is where the GPU pays.

    Results per query are ``(ref_id, score, block_length, block_position)`` sorted by ascending
    score then ref id, as in the reference.  ``block_length`` is ``|len(query) - len(ref)|``;
    ``block_position`` indexes the shorter sequence and, where several positions attain the
    minimum, is the smallest (the reference reports the first position its traversal meets).
    With ``max_penalty`` 0 only score-0 refs pass: identical sequences for matrices whose
    penalties between different residues are positive (all the built-ins; the reference asks its
    Hamming engine for zero substitutions in that case).
    """

    def __init__(self, refs: Iterable[str], alphabet: str = "aa", d_max: int = 1):
        if d_max < 0:
            raise ValueError("d_max must be >= 0")
        from . import device
        self.refs = list(refs)
        self.d_max = d_max
        self.alphabet = alphabet
        self._set = device.SeqSet(self.refs, alphabet)
        self._lens = np.fromiter(map(len, self.refs), np.int32, len(self.refs))

    def __len__(self) -> int:
        return len(self.refs)

    def search(self, query: str, max_penalty: int, matrix: SubstitutionMatrix | None = None,
               gap_open: int | None = None, gap_extend: int = 1,
               gap_prior: GapPrior | None = None) -> list[tuple[int, int, int, int]]:
        """All refs within ``max_penalty`` under the gap-block score (see the class docs)."""
        return self.search_batch([query], max_penalty, matrix, gap_open, gap_extend, gap_prior)[0]

    def search_batch(self, queries: Sequence[str], max_penalty: int,
                     matrix: SubstitutionMatrix | None = None, gap_open: int | None = None,
                     gap_extend: int = 1, gap_prior: GapPrior | None = None
                     ) -> list[list[tuple[int, int, int, int]]]:
        """``search`` for every query of the batch, in one GPU pass."""
        import ctypes

        import torch

        from . import _lib, device
        if gap_open is None:
            gap_open = _default_gap_open(matrix)
        if max_penalty < 0:
            raise ValueError("max_penalty must be >= 0")
        if gap_open < 0 or gap_extend < 0:
            raise ValueError("gap_open and gap_extend must be >= 0")
        q = list(queries)
        if not q:
            return []
        if not self.refs:
            return [[] for _ in q]
        width = max(max(map(len, q)), int(self._lens.max()))
        cube = np.asarray(prior_cube(gap_prior, width) if gap_prior is not None else [],
                          dtype=np.int64).astype(np.int32).ravel()
        qset = device.SeqSet(q, self.alphabet)
        stream = torch.cuda.current_stream().cuda_stream
        hits = device.Hits()
        device.gapblock_sparse_into(qset, self._set, hits, stream, max_penalty=max_penalty,
                                    matrix=matrix, gap_open=gap_open, gap_extend=gap_extend,
                                    prior=cube, prior_width=width if cube.size else 0)
        ip, rid, sc = device.hits_tensors(hits)
        rows = device.torch_rows(ip)
        qlen = torch.from_numpy(np.fromiter(map(len, q), np.int32, len(q))).cuda()
        rlen = torch.from_numpy(self._lens).cuda()
        d = (qlen[rows] - rlen[rid.long()]).abs()
        keep = d <= self.d_max
        rows, rid, sc, d = rows[keep], rid[keep], sc[keep], d[keep]
        n = int(rows.numel())
        pos = torch.empty(n, dtype=torch.int32, device="cuda")
        if n:
            qi = rows.to(torch.int32)
            again = torch.empty(n, dtype=torch.int32, device="cuda")
            pen = None if matrix is None else np.ascontiguousarray(matrix.penalty_grid, np.int32)
            err = _lib.st_error()
            _lib.check(_lib.lib.st_gapblock_pairs_pos_sets(
                qset.handle, self._set.handle, ctypes.c_void_p(qi.data_ptr()),
                ctypes.c_void_p(rid.data_ptr()), n, _lib.i32_ptr(pen),
                0 if pen is None else pen.shape[0], gap_open, gap_extend,
                _lib.i32_ptr(cube) if cube.size else None, int(cube.size),
                width if cube.size else 0, ctypes.c_void_p(again.data_ptr()),
                ctypes.c_void_p(pos.data_ptr()), ctypes.c_void_p(stream), ctypes.byref(err)), err)
            if not torch.equal(again, sc):
                raise RuntimeError("seqtree_b200: pair rescore disagrees with the sparse kernel")
        # order: query, then score, then ref id (stable sorts, least significant key first)
        order = torch.argsort(rid, stable=True)
        order = order[torch.argsort(sc[order], stable=True)]
        order = order[torch.argsort(rows[order], stable=True)]
        rows, rid, sc, d, pos = (t[order].cpu().numpy() for t in (rows, rid, sc, d, pos))
        bounds = np.searchsorted(rows, np.arange(len(q) + 1))
        out = []
        for a, b in zip(bounds[:-1], bounds[1:]):
            out.append([(int(r), int(s), int(dd), int(p))
                        for r, s, dd, p in zip(rid[a:b], sc[a:b], d[a:b], pos[a:b])])
        return out


# ------------------------------------------------------------------ island profiles --------
UNREACHABLE = 1 << 20
_AA = "ACDEFGHIKLMNPQRSTVWY"


def embed_in_frame(seq: str, width: int, c: int, gap: str = "-") -> str:
    """Place ``seq`` into a ``width``-column frame with its gap block at column ``c``: the first
    ``c`` symbols, ``width - len(seq)`` gaps, then the rest (seqtree
    ``python/seqtree/gapblock.py:186-205``; same errors)."""
    d = width - len(seq)
    if d < 0:
        raise ValueError(f"sequence of length {len(seq)} does not fit a width-{width} frame")
    if not 0 <= c <= len(seq):
        raise ValueError(f"frame column {c} outside [0, {len(seq)}]")
    return seq[:c] + gap * d + seq[c:]


class IslandProfile:
    """Column penalties over a frame -- seqtree's ``IslandProfile``
    (``python/seqtree/gapblock.py:208-380``) with the same constructor, ``fit``, ``consensus``,
    ``score`` and ``score_batch``.  Fitting is host statistics over an island's members (the
    reference's arithmetic, so the integer penalties are identical); scoring runs on the GPU
    (``st_profile_scores_sets``), one thread per sequence, and is meant for whole controls or
    repertoires.  Penalties are ``round(lam * log(p_max_j / p_j(a)))``, zero on each column's
    consensus symbol, capped so that a full-width score stays below :data:`UNREACHABLE`.
    Sequences are taken as ASCII text (one byte per residue)."""

    def __init__(self, penalties: list[dict[str, int]], width: int, c: int) -> None:
        self.penalties = penalties
        self.width = width
        self.c = c

    @classmethod
    def fit(cls, members: Sequence[str], c: int | None = None, lam: int = 1000,
            pseudocount: float = 0.5, gap: str = "-") -> "IslandProfile":
        import collections
        import math
        members = list(members)
        if not members:
            raise ValueError("cannot fit a profile to an empty island")
        if lam < 0:
            raise ValueError("lam must be >= 0")
        if pseudocount <= 0:
            raise ValueError("pseudocount must be > 0")
        width = max(len(s) for s in members)
        shortest = min(len(s) for s in members)
        if c is None:
            c = min(range(shortest + 1), key=lambda k: cls._entropy(members, width, k, gap))
        elif not 0 <= c <= shortest:
            raise ValueError(f"frame column {c} outside [0, {shortest}]")
        alpha = _AA + gap
        cap = UNREACHABLE // (width + 1)
        framed = [embed_in_frame(s, width, c, gap) for s in members]
        penalties = []
        for j in range(width):
            counts = collections.Counter(f[j] for f in framed)
            denom = sum(counts.values()) + pseudocount * len(alpha)
            probs = {a: (counts.get(a, 0) + pseudocount) / denom for a in alpha}
            p_max = max(probs.values())
            penalties.append({a: min(cap, int(round(lam * math.log(p_max / p))))
                              for a, p in probs.items()})
        return cls(penalties, width, c)

    @staticmethod
    def _entropy(members: Sequence[str], width: int, c: int, gap: str) -> float:
        import collections
        import math
        total = 0.0
        framed = [embed_in_frame(s, width, c, gap) for s in members]
        for j in range(width):
            counts = collections.Counter(f[j] for f in framed)
            n = sum(counts.values())
            total -= sum((v / n) * math.log(v / n) for v in counts.values() if v)
        return total

    def consensus(self, gap: str = "-") -> str:
        """The zero-penalty sequence: each column's cheapest symbol, gaps stripped."""
        return "".join(min(col, key=col.get) for col in self.penalties).replace(gap, "")

    def _table(self, gap: str) -> np.ndarray:
        cap = UNREACHABLE // (self.width + 1)
        t = np.full((max(self.width, 1), 256), cap, np.int32)
        for j, col in enumerate(self.penalties):
            for sym, v in col.items():
                b = sym.encode()
                if len(b) == 1:
                    t[j, b[0]] = v
        return t

    def score(self, seq: str, gap: str = "-") -> int:
        """Penalty of ``seq`` in this island's frame; :data:`UNREACHABLE` when it does not fit."""
        return self.score_batch([seq], gap)[0]

    def score_batch(self, seqs: Iterable[str], gap: str = "-") -> list[int]:
        """:meth:`score` for many sequences, on the GPU."""
        out = self.score_batch_np(seqs, gap)
        return [int(x) for x in out]

    def score_batch_np(self, seqs: Iterable[str], gap: str = "-") -> np.ndarray:
        """:meth:`score_batch` as an int32 numpy array."""
        import ctypes

        import torch

        from . import _lib, device
        seqs = list(seqs)
        g = gap.encode()
        if len(g) != 1:
            raise ValueError("gap must be a single ASCII symbol")
        if not all(s.isascii() for s in seqs):
            raise ValueError("profile scoring takes ASCII sequences")
        if not seqs:
            return np.zeros(0, np.int32)
        table = np.ascontiguousarray(self._table(gap))
        ss = device.SeqSet(seqs, None)
        out = torch.empty(len(seqs), dtype=torch.int32, device="cuda")
        err = _lib.st_error()
        _lib.check(_lib.lib.st_profile_scores_sets(
            _lib.i32_ptr(table), int(self.width), int(self.c), g[0], UNREACHABLE, ss.handle,
            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
            ctypes.byref(err)), err)
        return out.cpu().numpy()

    def __repr__(self) -> str:
        return f"IslandProfile(width={self.width}, c={self.c})"
