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
        self._free = _lib.lib.st_seqset_destroy  # kept: module globals are gone at exit
        packed = seqs if isinstance(seqs, _lib.Packed) else _lib.Packed(seqs)
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
            self._free(h)
            self._h = None


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


class Hits:
    """A thresholded sparse result kept on the current CUDA device (``st_hits``): CSR rows of
    device pointers, refilled in place by :func:`gapblock_sparse_into`."""

    def __init__(self):
        self._free = _lib.lib.st_hits_destroy
        self._h = ctypes.c_void_p()
        err = _lib.st_error()
        _lib.check(_lib.lib.st_hits_create(ctypes.byref(self._h), ctypes.byref(err)), err)

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        """rows, cols, nnz and the device pointers of indptr / ref_ids / scores."""
        rows, cols, nnz = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        ip, ri, sc = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        code = _lib.lib.st_hits_info(self._h, ctypes.byref(rows), ctypes.byref(cols),
                                     ctypes.byref(nnz), ctypes.byref(ip), ctypes.byref(ri),
                                     ctypes.byref(sc))
        if code:
            raise ValueError("invalid hits handle")
        return {"rows": rows.value, "cols": cols.value, "nnz": nnz.value,
                "indptr": ip.value or 0, "ref_ids": ri.value or 0, "scores": sc.value or 0}

    def to_host(self):
        """(indptr int64[rows+1], ref_ids int32[nnz], scores int32[nnz]) as numpy arrays."""
        info = self.info()
        indptr = np.zeros(info["rows"] + 1, np.int64)
        ref_ids = np.zeros(info["nnz"], np.int32)
        scores = np.zeros(info["nnz"], np.int32)
        err = _lib.st_error()
        code = _lib.lib.st_hits_download(self._h, indptr.ctypes.data, ref_ids.ctypes.data,
                                         scores.ctypes.data, ctypes.byref(err))
        _lib.check(code, err)
        return indptr, ref_ids, scores

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._free(h)
            self._h = None


def gapblock_sparse_into(queries: SeqSet, refs: SeqSet, hits: Hits, stream: int = 0, *,
                         max_penalty: int, matrix: SubstitutionMatrix | None = None,
                         gap_open: int = 1, gap_extend: int = 1, prior=(),
                         prior_width: int = 0) -> int:
    """Fill ``hits`` with the cells of the gap-block matrix scoring <= ``max_penalty``; returns
    the hit count.  Synchronises ``stream`` once (to size the sort)."""
    pen = None if matrix is None else np.ascontiguousarray(matrix.penalty_grid, np.int32)
    pr = np.ascontiguousarray(np.asarray(prior, dtype=np.int64).astype(np.int32)).ravel()
    err = _lib.st_error()
    code = _lib.lib.st_gapblock_sparse_sets(
        queries.handle, refs.handle, _lib.i32_ptr(pen), 0 if pen is None else pen.shape[0],
        gap_open, gap_extend, _lib.i32_ptr(pr) if pr.size else None, int(pr.size),
        int(prior_width), int(max_penalty), hits.handle, ctypes.c_void_p(stream),
        ctypes.byref(err))
    _lib.check(code, err)
    return hits.info()["nnz"]


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


class _DeviceArray:
    """A borrowed device buffer exposed through ``__cuda_array_interface__`` (for torch views)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr or 0, False), "version": 3, "strides": None}


def hits_tensors(hits):
    """(indptr int64, ref_ids int32, scores int32) torch copies of a device ``Hits``."""
    import torch
    info = hits.info()
    rows, nnz = info["rows"], info["nnz"]

    def view(ptr, n, ts, dt):
        if n == 0:
            return torch.zeros(0, dtype=dt, device="cuda")
        return torch.as_tensor(_DeviceArray(ptr, n, ts), device="cuda").clone()

    return (view(info["indptr"], rows + 1, "<i8", torch.int64),
            view(info["ref_ids"], nnz, "<i4", torch.int32),
            view(info["scores"], nnz, "<i4", torch.int32))


def torch_rows(indptr):
    """Row index of every CSR entry."""
    import torch
    n = indptr.numel() - 1
    return torch.arange(n, device=indptr.device).repeat_interleave(indptr[1:] - indptr[:-1])


def hits_rows(hits, rows) -> list:
    """``[(ref_ids int32, scores int32), ...]`` numpy arrays of the listed CSR rows of a device
    ``Hits``; only the row pointers and the listed rows cross to the host."""
    import torch
    info = hits.info()
    rows = [int(i) for i in rows]
    if info["rows"] == 0 or not rows:
        return [(np.zeros(0, np.int32), np.zeros(0, np.int32)) for _ in rows]
    ip = torch.as_tensor(_DeviceArray(info["indptr"], info["rows"] + 1, "<i8"),
                         device="cuda").cpu().numpy()
    out = []
    nnz = info["nnz"]
    ri = sc = None
    if nnz:
        ri = torch.as_tensor(_DeviceArray(info["ref_ids"], nnz, "<i4"), device="cuda")
        sc = torch.as_tensor(_DeviceArray(info["scores"], nnz, "<i4"), device="cuda")
    for i in rows:
        a, b = int(ip[i]), int(ip[i + 1])
        if b > a:
            out.append((ri[a:b].cpu().numpy(), sc[a:b].cpu().numpy()))
        else:
            out.append((np.zeros(0, np.int32), np.zeros(0, np.int32)))
    return out
