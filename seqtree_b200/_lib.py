"""ctypes binding of ``libseqtree_b200.so`` (the C ABI in ``include/seqtree_b200.h``).

The library is the only compute path: importing this module fails loudly when the shared
library is missing, and every call runs on the current CUDA device (there is no CPU fallback).
ctypes releases the GIL for the duration of each foreign call, as the reference's binding does
(seqtree ``src/_bindings.cpp:227,537,558,592,608``).
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libseqtree_b200.so"

ST_OK, ST_EINVAL, ST_EOVERFLOW, ST_ECUDA, ST_ETIMEOUT, ST_ENOMEM, ST_ENODEV = range(7)
ALPHABET_AA, ALPHABET_NT, ALPHABET_IUPAC = 0, 1, 2
MODE_GLOBAL, MODE_LOCAL = 0, 1


class st_strings(ctypes.Structure):
    _fields_ = [("bytes", ctypes.c_void_p), ("offsets", ctypes.c_void_p),
                ("count", ctypes.c_int64)]


class st_error(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int32), ("message", ctypes.c_char * 256)]


class st_peak(ctypes.Structure):
    _fields_ = [("lane_ops_per_s", ctypes.c_double), ("lane_ops_per_sm_clk", ctypes.c_double),
                ("ms", ctypes.c_double), ("sms", ctypes.c_int32), ("threads", ctypes.c_int32)]


PEAK_OPS = {"lop3": 0, "iadd3": 1, "imad": 2, "viaddmin_s16x2": 3, "viaddmax_s32": 4,
            "vimax3_s32": 5, "lds32": 6}


class st_sparse(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_int64), ("cols", ctypes.c_int64), ("nnz", ctypes.c_int64),
                ("indptr", ctypes.POINTER(ctypes.c_int64)),
                ("ref_ids", ctypes.POINTER(ctypes.c_int32)),
                ("scores", ctypes.POINTER(ctypes.c_int32))]


_i32p = ctypes.POINTER(ctypes.c_int32)
_sp = ctypes.POINTER(st_strings)
_ep = ctypes.POINTER(st_error)

# (name, restype, argtypes) of every symbol declared in include/seqtree_b200.h
SIGNATURES = [
    ("st_version", ctypes.c_int32, []),
    ("st_device_count", ctypes.c_int32, []),
    ("st_gapblock_matrix", ctypes.c_int32,
     [_sp, _sp, ctypes.c_int32, _i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p,
      ctypes.c_int64, ctypes.c_uint32, ctypes.c_int32, ctypes.c_void_p, _ep]),
    ("st_align_score_matrix", ctypes.c_int32,
     [_sp, _sp, _i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, _ep]),
    ("st_align_dist_matrix", ctypes.c_int32,
     [_sp, _sp, _i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, _ep]),
    ("st_align_pair", ctypes.c_int32,
     [ctypes.c_char_p, ctypes.c_int64, ctypes.c_char_p, ctypes.c_int64, _i32p, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p, ctypes.c_char_p,
      ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int64, _ep]),
    ("st_penalty_align_pairs", ctypes.c_int32,
     [_sp, _sp, _i32p, _i32p, ctypes.c_int64, ctypes.c_int32, _i32p, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_int32, _i32p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_int64, _i32p, _ep]),
    ("st_hamming_matrix", ctypes.c_int32, [_sp, _sp, ctypes.c_int32, ctypes.c_void_p, _ep]),
    ("st_levenshtein_matrix", ctypes.c_int32, [_sp, _sp, ctypes.c_int32, ctypes.c_void_p, _ep]),
    ("st_gapblock_sparse", ctypes.c_int32,
     [_sp, _sp, ctypes.c_int32, _i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p,
      ctypes.c_int64, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32,
      ctypes.POINTER(st_sparse), _ep]),
    ("st_sparse_free", None, [ctypes.POINTER(st_sparse)]),
    ("st_hits_create", ctypes.c_int32, [ctypes.POINTER(ctypes.c_void_p), _ep]),
    ("st_hits_destroy", None, [ctypes.c_void_p]),
    ("st_hits_info", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
      ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_void_p),
      ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]),
    ("st_hits_download", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_gapblock_sparse_sets", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, _i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
      _i32p, ctypes.c_int64, ctypes.c_uint32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
      _ep]),
    ("st_gapblock_pairs_sets", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, _i32p,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p, ctypes.c_int64, ctypes.c_uint32,
      ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_gapblock_pairs_pos_sets", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, _i32p,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p, ctypes.c_int64, ctypes.c_uint32,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_encoder_param_count", ctypes.c_int64, []),
    ("st_encoder_create", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), _ep]),
    ("st_encoder_destroy", None, [ctypes.c_void_p]),
    ("st_encoder_get_params", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_encoder_set_precision", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, _ep]),
    ("st_encoder_loss_grad", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
      ctypes.POINTER(ctypes.c_float), ctypes.c_void_p, _ep]),
    ("st_encoder_train_step", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_float, ctypes.POINTER(ctypes.c_float), _ep]),
    ("st_encoder_embed", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, _ep]),
    ("st_train_gemm_bf16", ctypes.c_int32,
     [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, _ep]),
    ("st_propose_topk", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_propose_topk_ranges", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_propose_range", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, _ep]),
    ("st_embed_dots", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_stream_status", ctypes.c_int32, [ctypes.c_void_p, _ep]),
    ("st_align_pairs_sets", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, _i32p,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
      ctypes.c_void_p, _ep]),
    ("st_profile_scores_sets", ctypes.c_int32,
     [_i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint8, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_thetas_csr", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
      ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_seqset_create", ctypes.c_int32,
     [_sp, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p), _ep]),
    ("st_seqset_destroy", None, [ctypes.c_void_p]),
    ("st_seqset_count", ctypes.c_int64, [ctypes.c_void_p]),
    ("st_gapblock_matrix_sets", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, _i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
      _i32p, ctypes.c_int64, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_align_matrix_sets", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, _i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_hamming_matrix_sets", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_levenshtein_matrix_sets", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_split_joined", ctypes.c_int64,
     [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]),
    ("st_levenshtein_matrix_noalloc", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, _ep]),
    ("st_builtin_similarity", ctypes.c_int32,
     [ctypes.c_char_p, _i32p, ctypes.c_int32, _i32p, _ep]),
    ("st_measure_peak", ctypes.c_int32,
     [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(st_peak), _ep]),
    ("st_last_launch_count", ctypes.c_int32, []),
    ("st_total_launch_count", ctypes.c_int64, []),
    ("st_tuning_table", ctypes.c_int64, [ctypes.c_char_p, ctypes.c_int64]),
    ("st_last_kernel_name", ctypes.c_char_p, []),
    ("st_host_alloc", ctypes.c_void_p, [ctypes.c_uint64]),
    ("st_host_free", None, [ctypes.c_void_p]),
]


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"seqtree_b200: the CUDA library {LIB_PATH} is not built; run "
            "`python -m seqtree_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def check(code: int, err: st_error) -> None:
    """Raise the Python exception the reference's binding raises for the same failure."""
    if code == ST_OK:
        return
    msg = err.message.decode("utf-8", "replace")
    if code == ST_EINVAL:
        raise ValueError(msg)
    if code == ST_EOVERFLOW:
        raise OverflowError(msg)
    if code == ST_ENOMEM:
        raise MemoryError(msg)
    raise RuntimeError(msg)


try:  # the list packer (csrc/pack_py.c); without it the join-and-split path below packs lists
    from . import _pack
except ImportError:
    _pack = None


def _pack_ascii(seqs: list):
    """(bytes, offsets) of a list of ASCII strings without a per-string Python loop: the list is
    joined with a newline separator, which the library splits (``st_split_joined``).  None when
    that does not apply (non-str items, non-ASCII text, or a newline inside a string), so the
    caller takes the general path."""
    n = len(seqs)
    if n == 0:
        return None
    try:
        buf = "\n".join(seqs).encode("ascii")
    except (TypeError, UnicodeError):
        return None
    data = np.empty(max(len(buf) - (n - 1), 1), dtype=np.uint8)
    off = np.empty(n + 1, dtype=np.int64)
    if lib.st_split_joined(buf, len(buf), n, data.ctypes.data, off.ctypes.data) < 0:
        return None
    return data, off


class Packed:
    """A list of sequences as one byte buffer plus int64 offsets (keeps both alive)."""

    __slots__ = ("data", "offsets", "struct")

    def __init__(self, seqs):
        seqs = seqs if isinstance(seqs, list) else list(seqs)
        packed = _pack.pack(seqs) if _pack is not None else None
        if packed is not None:  # ASCII strings, copied in one pass by the extension
            self.data = np.frombuffer(packed[0], dtype=np.uint8)
            self.offsets = np.frombuffer(packed[1], dtype=np.int64)
            self.struct = st_strings(self.data.ctypes.data, self.offsets.ctypes.data, len(seqs))
            return
        fast = _pack_ascii(seqs)
        if fast is not None:
            self.data, self.offsets = fast
            self.struct = st_strings(self.data.ctypes.data, self.offsets.ctypes.data, len(seqs))
            return
        try:
            data = "".join(seqs).encode("utf-8")
            lens = np.fromiter(map(len, seqs), dtype=np.int64, count=len(seqs))
            if len(data) != int(lens.sum()):  # non-ASCII text: use byte lengths
                raise UnicodeError
        except (TypeError, UnicodeError):
            enc = []
            for s in seqs:
                if isinstance(s, str):
                    enc.append(s.encode("utf-8"))
                elif isinstance(s, (bytes, bytearray)):
                    enc.append(bytes(s))
                else:
                    raise TypeError("sequences must be str") from None
            data = b"".join(enc)
            lens = np.fromiter(map(len, enc), dtype=np.int64, count=len(enc))
        off = np.zeros(len(seqs) + 1, dtype=np.int64)
        np.cumsum(lens, out=off[1:])
        self.data = np.frombuffer(data, dtype=np.uint8) if data else np.zeros(1, np.uint8)
        self.offsets = off
        self.struct = st_strings(self.data.ctypes.data, self.offsets.ctypes.data, len(seqs))

    @classmethod
    def from_arrays(cls, data: np.ndarray, offsets: np.ndarray) -> "Packed":
        """Sequences already concatenated: ``data`` (uint8) and ``offsets`` (int64, count + 1)."""
        self = cls.__new__(cls)
        self.data = np.ascontiguousarray(data, np.uint8) if len(data) else np.zeros(1, np.uint8)
        self.offsets = np.ascontiguousarray(offsets, np.int64)
        self.struct = st_strings(self.data.ctypes.data, self.offsets.ctypes.data,
                                 len(self.offsets) - 1)
        return self

    @property
    def count(self) -> int:
        return int(self.struct.count)

    @property
    def max_len(self) -> int:
        """Length in bytes of the longest sequence (0 when there are none)."""
        return int(np.diff(self.offsets).max()) if self.offsets.size > 1 else 0

    def ref(self):
        return ctypes.byref(self.struct)


class _PinnedOwner:
    """Returns a pinned block to the library's cache when the last view is gone."""

    __slots__ = ("ptr", "_free")

    def __init__(self, ptr: int):
        self.ptr = ptr
        self._free = lib.st_host_free

    def __del__(self):
        if self.ptr:
            self._free(ctypes.c_void_p(self.ptr))
            self.ptr = 0


def pack(seqs) -> "Packed":
    """``seqs`` as a :class:`Packed` (returned as is when it already is one)."""
    return seqs if isinstance(seqs, Packed) else Packed(seqs)


def pinned_int32(rows: int, cols: int) -> np.ndarray:
    """An int32 (rows, cols) array in page-locked host memory from the library's cache.

    Device results copy into it at full PCIe rate.  Falls back to ordinary memory when no
    pinned block can be had (the copy is then slower, the result identical).
    """
    n = rows * cols
    if n == 0:
        return np.zeros((rows, cols), np.int32)
    ptr = lib.st_host_alloc(n * 4)
    if not ptr:
        return np.empty((rows, cols), np.int32)
    buf = (ctypes.c_int32 * n).from_address(ptr)
    buf._owner = _PinnedOwner(ptr)  # the ctypes array is the numpy base; it owns the block
    return np.frombuffer(buf, dtype=np.int32, count=n).reshape(rows, cols)


def pinned_array(n: int, dtype) -> np.ndarray:
    """A 1-d int32 or int64 array of n elements in page-locked host memory from the library's
    cache (ordinary memory when no pinned block can be had)."""
    dtype = np.dtype(dtype)
    ctype = {4: ctypes.c_int32, 8: ctypes.c_int64}[dtype.itemsize]
    if n == 0:
        return np.zeros(0, dtype)
    ptr = lib.st_host_alloc(n * dtype.itemsize)
    if not ptr:
        return np.empty(n, dtype)
    buf = (ctype * n).from_address(ptr)
    buf._owner = _PinnedOwner(ptr)
    return np.frombuffer(buf, dtype=dtype, count=n)


def adopt_pinned(ptr, n: int, ctype, dtype) -> np.ndarray:
    """A numpy view of n elements of a pinned block the library allocated; the view owns the
    block (it returns to the cache when the last view is gone)."""
    addr = ctypes.cast(ptr, ctypes.c_void_p).value
    if not addr:
        return np.zeros(n, dtype)
    buf = (ctype * max(n, 1)).from_address(addr)
    buf._owner = _PinnedOwner(addr)
    return np.frombuffer(buf, dtype=dtype, count=n)


def i32_ptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(_i32p)


def last_launch_count() -> int:
    return int(lib.st_last_launch_count())


def tuning_table() -> str:
    """The autotuner's decisions: one line per tuned shape key."""
    n = int(lib.st_tuning_table(None, 0))
    buf = ctypes.create_string_buffer(n + 1)
    lib.st_tuning_table(buf, n + 1)
    return buf.value.decode()


def total_launch_count() -> int:
    return int(lib.st_total_launch_count())


def last_kernel_name() -> str:
    return (lib.st_last_kernel_name() or b"").decode()


def device_count() -> int:
    return int(lib.st_device_count())


def measure_peak(op: str, all_sms: bool) -> dict:
    """Peak issue rate of one instruction on the current device (``st_measure_peak``)."""
    out, err = st_peak(), st_error()
    check(lib.st_measure_peak(PEAK_OPS[op], int(all_sms), ctypes.byref(out), ctypes.byref(err)),
          err)
    return {"lane_ops_per_s": out.lane_ops_per_s, "per_sm_clk": out.lane_ops_per_sm_clk,
            "ms": out.ms, "sms": out.sms, "threads": out.threads}


def measure_peaks() -> dict:
    """Every probe of :func:`measure_peak`, on one SM and on all SMs."""
    return {op: {"one_sm": measure_peak(op, False), "all_sms": measure_peak(op, True)}
            for op in PEAK_OPS}
