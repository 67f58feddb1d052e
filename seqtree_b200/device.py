"""Device-resident form of the matrix calls: sequence sets uploaded once, results in HBM.

A :class:`SeqSet` is uploaded and encoded once (``st_seqset_create``); the ``*_into`` calls
write a dense int32 matrix into caller-provided DEVICE memory on a caller-provided CUDA stream
with no host round trip (``st_*_matrix_sets`` in ``include/seqtree_b200.h``).  Pointers and
streams are plain integers, so any allocator works; with PyTorch pass ``t.data_ptr()`` and
``torch.cuda.current_stream().cuda_stream``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .matrix import SubstitutionMatrix, parse_align_mode, parse_alphabet


class SeqSet:
    """Sequences resident on the current CUDA device (encoded, or raw bytes when alphabet=None)."""

    def __init__(self, seqs, alphabet: str | None = "aa"):
        packed = _lib.Packed(seqs)
        self.alphabet = None if alphabet is None else parse_alphabet(alphabet)
        self._h = ctypes.c_void_p()
        err = _lib.st_error()
        code = _lib.lib.st_seqset_create(packed.ref(), -1 if self.alphabet is None else self.alphabet,
                                         ctypes.byref(self._h), ctypes.byref(err))
        _lib.check(code, err)
        self.count = packed.count

    @property
    def handle(self):
        return self._h

    def __len__(self) -> int:
        return self.count

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib.st_seqset_destroy(h)
            self._h = ctypes.c_void_p()


def gapblock_into(queries: SeqSet, refs: SeqSet, out_ptr: int, stream: int = 0,
                  matrix: SubstitutionMatrix | None = None, gap_open: int = 1,
                  gap_extend: int = 1, prior=(), prior_width: int = 0) -> None:
    pen = None if matrix is None else np.ascontiguousarray(matrix.penalty_grid, np.int32)
    pr = np.ascontiguousarray(np.asarray(prior, dtype=np.int64).astype(np.int32)).ravel()
    err = _lib.st_error()
    code = _lib.lib.st_gapblock_matrix_sets(
        queries.handle, refs.handle, _lib.i32_ptr(pen), 0 if pen is None else pen.shape[0],
        gap_open, gap_extend, _lib.i32_ptr(pr) if pr.size else None, int(pr.size),
        int(prior_width), ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream), ctypes.byref(err))
    _lib.check(code, err)


def align_into(queries: SeqSet, refs: SeqSet, out_ptr: int, stream: int = 0, *,
               matrix: SubstitutionMatrix, mode: str = "global", gap_open: int = 11,
               gap_extend: int = 1, dist: bool = False) -> None:
    sim = np.ascontiguousarray(matrix.similarity_grid, np.int32)
    err = _lib.st_error()
    code = _lib.lib.st_align_matrix_sets(queries.handle, refs.handle, _lib.i32_ptr(sim),
                                         sim.shape[0], parse_align_mode(mode), gap_open,
                                         gap_extend, int(dist), ctypes.c_void_p(out_ptr),
                                         ctypes.c_void_p(stream), ctypes.byref(err))
    _lib.check(code, err)


def hamming_into(a: SeqSet, b: SeqSet, out_ptr: int, stream: int = 0) -> None:
    err = _lib.st_error()
    code = _lib.lib.st_hamming_matrix_sets(a.handle, b.handle, ctypes.c_void_p(out_ptr),
                                           ctypes.c_void_p(stream), ctypes.byref(err))
    _lib.check(code, err)


def levenshtein_into(a: SeqSet, b: SeqSet, out_ptr: int, stream: int = 0) -> None:
    err = _lib.st_error()
    code = _lib.lib.st_levenshtein_matrix_sets(a.handle, b.handle, ctypes.c_void_p(out_ptr),
                                               ctypes.c_void_p(stream), ctypes.byref(err))
    _lib.check(code, err)
