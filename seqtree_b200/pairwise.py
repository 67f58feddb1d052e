"""Needleman-Wunsch / Smith-Waterman with affine (Gotoh) gaps, maximising the raw similarity.

Mirrors seqtree's ``python/seqtree/pairwise.py`` (``score`` ``:53-85``, ``score_matrix``
``:119-136``, ``dist_matrix`` ``:139-167``).  Conventions: a gap run of length L costs
``gap_open + (L-1) * gap_extend``; ``gap_open == gap_extend`` is linear; global mode charges end
gaps; local mode floors the match state at 0 and takes the best cell anywhere.  Gap costs are
positive magnitudes that are subtracted.
"""
from __future__ import annotations

from collections.abc import Sequence

import ctypes

import numpy as np

from . import _lib
from ._core import Alignment, _i32
from ._core import align_pair as _align_pair
from ._core import align_dist_matrix as _dist_matrix
from ._core import align_score as _align_score
from ._core import align_score_matrix as _score_matrix
from .matrix import ScoreMatrix, SubstitutionMatrix, alphabet_symbols, parse_align_mode, parse_alphabet

__all__ = ["score", "align", "align_batch", "align_pairs", "Alignment", "score_matrix",
           "dist_matrix", "penalty_align", "penalty_align_pairs"]


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


def align(query: str, ref: str, matrix: SubstitutionMatrix, mode: str = "global",
          gap_open: int = 11, gap_extend: int = 1, alphabet: str = "aa") -> Alignment:
    """As :func:`score`, but also returns the aligned strings and the edit ops (seqtree's
    ``pairwise.align`` / ``align_pair``, ``src/pairwise.cpp:141-267``).  In local mode the aligned
    strings are the matched sub-sequences only."""
    return _align_pair(query, ref, matrix, mode=mode, gap_open=gap_open, gap_extend=gap_extend,
                       alphabet=alphabet)


def align_batch(queries: Sequence[str], refs: Sequence[str], matrix: SubstitutionMatrix,
                mode: str = "global", gap_open: int = 11, gap_extend: int = 1,
                alphabet: str = "aa") -> list[Alignment]:
    """``align(queries[p], refs[p])`` for every p, in one GPU launch."""
    q, r = list(queries), list(refs)
    if len(q) != len(r):
        raise ValueError("queries and refs must pair up (equal lengths)")
    idx = np.arange(len(q), dtype=np.int32)
    return align_pairs(q, r, idx, idx, matrix, mode, gap_open, gap_extend, alphabet)


def align_pairs(queries: Sequence[str], refs: Sequence[str], query_idx, ref_idx,
                matrix: SubstitutionMatrix, mode: str = "global", gap_open: int = 11,
                gap_extend: int = 1, alphabet: str = "aa") -> list[Alignment]:
    """Alignments of the listed pairs ``(queries[query_idx[p]], refs[ref_idx[p]])`` -- e.g. the
    hits of a sparse search -- one thread per pair on the GPU, exact for any gap cost."""
    import torch

    from .device import SeqSet
    if not isinstance(matrix, SubstitutionMatrix):
        raise TypeError("matrix must be a SubstitutionMatrix")
    alph = parse_alphabet(alphabet)
    md = parse_align_mode(mode)
    go, ge = _i32("gap_open", gap_open), _i32("gap_extend", gap_extend)
    if go < 0 or ge < 0:
        raise ValueError("seqtree: gap_open and gap_extend must be >= 0 (they are magnitudes, and "
                         "are subtracted)")
    sim = np.ascontiguousarray(matrix.similarity_grid, np.int32)
    if sim.shape[0] != len(alphabet_symbols(alphabet)):
        raise ValueError("matrix size does not match the alphabet")
    q, r = list(queries), list(refs)
    qi = np.ascontiguousarray(query_idx, np.int32).ravel()
    ri = np.ascontiguousarray(ref_idx, np.int32).ravel()
    if qi.size != ri.size:
        raise ValueError("query_idx and ref_idx must have the same length")
    n = int(qi.size)
    if n == 0:
        return []
    if qi.min() < 0 or qi.max() >= len(q) or ri.min() < 0 or ri.max() >= len(r):
        raise IndexError("pair index out of range")
    qs, rs = SeqSet(q, alphabet), SeqSet(r, alphabet)
    slot = max(max(map(len, q)) + max(map(len, r)), 1)
    dev = "cuda"
    tq, tr = torch.from_numpy(qi).to(dev), torch.from_numpy(ri).to(dev)
    score = torch.empty(n, dtype=torch.int64, device=dev)
    start = torch.empty(n, dtype=torch.int32, device=dev)
    bufs = [torch.empty(n * slot, dtype=torch.uint8, device=dev) for _ in range(3)]
    err = _lib.st_error()
    _lib.check(_lib.lib.st_align_pairs_sets(
        qs.handle, rs.handle, ctypes.c_void_p(tq.data_ptr()), ctypes.c_void_p(tr.data_ptr()), n,
        _lib.i32_ptr(sim), sim.shape[0], md, go, ge, ctypes.c_void_p(score.data_ptr()),
        ctypes.c_void_p(start.data_ptr()), ctypes.c_void_p(bufs[0].data_ptr()),
        ctypes.c_void_p(bufs[1].data_ptr()), ctypes.c_void_p(bufs[2].data_ptr()), slot,
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(err)), err)
    sc, st = score.cpu().numpy(), start.cpu().numpy()
    if sc.size and (sc.max() > 2**31 - 1 or sc.min() < -2**31):
        raise OverflowError("seqtree: the alignment score does not fit in 32 bits -- the gap costs "
                            "are absurdly large for these sequences")
    qa, ra, ops = (b.cpu().numpy().reshape(n, slot) for b in bufs)
    local = md == 1
    out = []
    for p in range(n):
        s = int(st[p])
        if s < 0:  # an empty side: the reference writes the raw input (global) or nothing (local)
            a, b = q[qi[p]], r[ri[p]]
            if local:
                out.append(Alignment("", "", "", int(sc[p])))
            else:
                out.append(Alignment(a + "-" * len(b), "-" * len(a) + b,
                                     "D" * len(a) + "I" * len(b), int(sc[p])))
            continue
        out.append(Alignment(qa[p, s:].tobytes().decode(), ra[p, s:].tobytes().decode(),
                             ops[p, s:].tobytes().decode(), int(sc[p])))
    return out


# ------------------------------------------------------------ penalty alignment (Index.align)
_MATRIX_NAMES = ("identity", "blosum62", "blosum45", "blosum80", "pam250", "pam100", "structural")


def _penalty_grid(matrix, alphabet: str) -> np.ndarray | None:
    """The penalty grid of ``matrix`` as seqtree's SearchParams takes it (src/_bindings.cpp:
    67-119): None or '' is unit cost, a name is a built-in matrix ('identity' is unit cost of the
    alphabet's size; the others need amino acids), or a SubstitutionMatrix."""
    if matrix is None:
        return None
    if isinstance(matrix, str):
        name = matrix.lower()
        if name and name not in _MATRIX_NAMES:
            raise ValueError(f"unknown matrix '{matrix}' (use '', 'identity', 'BLOSUM62', "
                             "'BLOSUM45', 'BLOSUM80', 'PAM250', 'PAM100', 'structural', or a "
                             "SubstitutionMatrix)")
        if not name:
            return None
        if name == "identity":
            matrix = SubstitutionMatrix.unit(len(alphabet_symbols(alphabet)))
        elif parse_alphabet(alphabet) != 0:
            raise ValueError(f"{name} requires the amino-acid alphabet")
        else:
            matrix = SubstitutionMatrix._named(name)
    if not isinstance(matrix, SubstitutionMatrix):
        raise TypeError("matrix must be a name string or a SubstitutionMatrix")
    return np.ascontiguousarray(matrix.penalty_grid, np.int32)


def penalty_align_pairs(queries: Sequence[str], refs: Sequence[str], query_idx, ref_idx,
                        matrix=None, gap_open: int = 1, gap_extend: int = 1,
                        alphabet: str = "aa") -> list[Alignment]:
    """Penalty-minimising global alignments of the listed pairs ``(queries[query_idx[p]],
    refs[ref_idx[p]])`` on the GPU, one thread per pair: seqtree's ``Index.align(ref_id, query,
    SearchParams(matrix=..., gap_open=..., gap_extend=...))`` (src/index.cpp:105-179) with
    ``refs`` as the index's references.  ``score`` is the summed substitution penalty plus
    ``gap_open + (L-1) * gap_extend`` per gap run (lower is closer); unit cost when ``matrix``
    is None.  The aligned strings keep the caller's characters (case included)."""
    alph = parse_alphabet(alphabet)
    pen = _penalty_grid(matrix, alphabet)
    go, ge = _i32("gap_open", gap_open), _i32("gap_extend", gap_extend)
    qi = np.ascontiguousarray(query_idx, np.int32).ravel()
    ri = np.ascontiguousarray(ref_idx, np.int32).ravel()
    if qi.size != ri.size:
        raise ValueError("query_idx and ref_idx must have the same length")
    q, r = _lib.pack(queries), _lib.pack(refs)
    n = int(qi.size)
    if n and (qi.min() < 0 or qi.max() >= q.count or ri.min() < 0 or ri.max() >= r.count):
        raise IndexError("pair index out of range")
    stride = q.max_len + r.max_len + 1
    scores = np.zeros(n, np.int32)
    lengths = np.zeros(n, np.int32)
    bufs = [ctypes.create_string_buffer(max(n * stride, 1)) for _ in range(3)]
    err = _lib.st_error()
    _lib.check(_lib.lib.st_penalty_align_pairs(
        q.ref(), r.ref(), _lib.i32_ptr(qi), _lib.i32_ptr(ri), n, alph, _lib.i32_ptr(pen),
        0 if pen is None else pen.shape[0], go, ge, _lib.i32_ptr(scores), bufs[0], bufs[1],
        bufs[2], stride, _lib.i32_ptr(lengths), ctypes.byref(err)), err)
    raw = [b.raw for b in bufs]
    out = []
    for p in range(n):
        a, L = p * stride, int(lengths[p])
        out.append(Alignment(raw[0][a:a + L].decode("latin-1"), raw[1][a:a + L].decode("latin-1"),
                             raw[2][a:a + L].decode("latin-1"), int(scores[p])))
    return out


def penalty_align(query: str, ref: str, matrix=None, gap_open: int = 1, gap_extend: int = 1,
                  alphabet: str = "aa") -> Alignment:
    """One pair of :func:`penalty_align_pairs`: what ``Index.build(refs).align(k, query,
    params)`` returns for ``ref = refs[k]``."""
    return penalty_align_pairs([query], [ref], [0], [0], matrix, gap_open, gap_extend,
                               alphabet)[0]
