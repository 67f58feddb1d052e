"""Learned candidate proposal for thresholded gap-block search at scales where the exhaustive
kernel's 10^12 pairs are the cost (1e6 x 1e6 CDR3-like junctions).

A small encoder (:class:`Encoder`; 2 conv + 2 attention layers, width 128, 64-d unit-length
output) is trained on pairs scored by the exact gap-block kernel so that squared embedding
distance tracks the score.  Its embeddings feed a BF16 tensor-core product that proposes
candidate refs for every query: the top-k by dot product (``st_propose_topk``), or every ref whose
dot product reaches a threshold chosen per (query length, ref length) cell
(``st_propose_range``).  Every proposal is rescored by the exact kernel, so reported scores are
always exact.  A held-out calibration batch sets the thresholds and routes the query and ref
lengths where proposals cost more than exhaustive scoring to the exhaustive kernel, so that the
estimated recall reaches the bound.

Everything runs through ``libseqtree_b200.so``: the training kernels (forward, backward, Adam),
the embedding, the proposal kernel and the exact scorer.
"""
from __future__ import annotations

import ctypes
import itertools
import json
import os
import struct
import zlib

import numpy as np

from . import _lib
from .device import hits_tensors as _hits_tensors, torch_rows
from .matrix import SubstitutionMatrix
from .workloads import AA20, AA20_CODES as _AA20_CODES, AA24, CODE as _CODE, PAD  # noqa: F401
from .workloads import cdr3_codes, cdr3_lengths, codes_to_letters, codes_to_strings  # noqa: F401


# ------------------------------------------------------------------------ model files -------
# A trained encoder (and, from LearnedIndex, its calibrated fallback) is kept in one versioned
# flat file, little-endian:
#   magic "STBE" | version u32 | parameter count u64 | metadata length u32 | metadata (UTF-8 JSON)
#   | parameters (fp32 x count) | CRC-32 of every preceding byte (u32)
# It is written to a temporary beside the destination and renamed over it, so a concurrent reader
# sees the old file or the new one, never half of one, and a failed write leaves no temporary
# (the reference's src/atomic_write.hpp:47-75 does the same for its index files).
MODEL_MAGIC = b"STBE"
MODEL_VERSION = 1
_tmp_seq = itertools.count()


def encode_model(params: np.ndarray, meta: dict | None = None) -> bytes:
    """The model-file bytes of ``params`` (fp32) and a JSON-serialisable ``meta``."""
    p = np.ascontiguousarray(params, np.float32).ravel()
    m = json.dumps(meta or {}, sort_keys=True).encode()
    body = (MODEL_MAGIC + struct.pack("<IQI", MODEL_VERSION, p.size, len(m)) + m +
            p.astype("<f4").tobytes())
    return body + struct.pack("<I", zlib.crc32(body) & 0xFFFFFFFF)


def decode_model(data: bytes, name: str = "model file") -> tuple[np.ndarray, dict]:
    """(params, meta) of model-file bytes; ValueError when they are not a version-1 file, are
    truncated, or fail the checksum."""
    if len(data) < 20 or data[:4] != MODEL_MAGIC:
        raise ValueError(f"seqtree_b200: '{name}' is not a seqtree_b200 encoder file")
    version, count, mlen = struct.unpack_from("<IQI", data, 4)
    if version != MODEL_VERSION:
        raise ValueError(f"seqtree_b200: '{name}' is a version {version} encoder file; this "
                         f"library reads version {MODEL_VERSION}")
    end = 20 + mlen + 4 * count
    if len(data) != end + 4:
        raise ValueError(f"seqtree_b200: truncated or corrupt encoder file '{name}'")
    (crc,) = struct.unpack_from("<I", data, end)
    if zlib.crc32(data[:end]) & 0xFFFFFFFF != crc:
        raise ValueError(f"seqtree_b200: truncated or corrupt encoder file '{name}' (checksum)")
    meta = json.loads(data[20:20 + mlen].decode())
    params = np.frombuffer(data, dtype="<f4", count=count, offset=20 + mlen).astype(np.float32)
    return params, meta


def atomic_write(path, data: bytes) -> None:
    """Writes ``data`` to a temporary beside ``path`` and renames it over ``path``; on any failure
    the temporary is removed and the error re-raised (``path`` is left as it was)."""
    path = os.fspath(path)
    tmp = f"{path}.tmp.{os.getpid()}.{next(_tmp_seq)}"
    try:
        with open(tmp, "wb") as f:
            f.write(data)
            f.flush()
            os.fsync(f.fileno())
        os.replace(tmp, path)
    except BaseException:
        try:
            os.remove(tmp)
        except FileNotFoundError:
            pass
        raise


def param_count() -> int:
    return int(_lib.lib.st_encoder_param_count())


def init_params(seed: int) -> np.ndarray:
    """Uniform(+-1/sqrt(fan_in)) weights and zero biases, in the flat parameter order."""
    rng = np.random.default_rng(seed)
    W, A, E = 128, 24, 64
    blocks = [((3, A, W), 3), ((W,), 0), ((3 * W, W), 3 * W), ((W,), 0)]
    for _ in range(2):
        blocks += [((W, 3 * W), W), ((3 * W,), 0), ((W, W), W), ((W,), 0)]
    blocks += [((W, E), W), ((E,), 0)]
    parts = []
    for shape, fan in blocks:
        n = int(np.prod(shape))
        parts.append(rng.uniform(-1, 1, n) / np.sqrt(fan) if fan else np.zeros(n))
    out = np.concatenate(parts).astype(np.float32)
    assert out.size == param_count()
    return out


def pad_codes(seqs) -> tuple[np.ndarray, np.ndarray]:
    """Amino-acid codes [S, 32] (zero past each length) and lengths [S]."""
    S = len(seqs)
    codes = np.zeros((S, PAD), np.uint8)
    lens = np.fromiter((len(s) for s in seqs), np.int32, S)
    if S and (lens.min() < 1 or lens.max() > PAD):
        raise ValueError("encoder inputs must have 1..32 residues")
    flat = np.frombuffer("".join(seqs).encode(), np.uint8)
    c = _CODE[flat]
    if (c == 255).any():
        bad = chr(int(flat[np.argmax(c == 255)]))
        raise ValueError(f"symbol '{bad}' is not in the alphabet")
    rows = np.repeat(np.arange(S), lens)
    cols = np.arange(flat.size) - np.repeat(np.cumsum(lens) - lens, lens)
    codes[rows, cols] = c
    return codes, lens


class Encoder:
    """The CUDA encoder (``st_encoder``): parameters, training steps and embeddings."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0, precision: str = "bf16"):
        """``precision`` is that of the training products: "bf16" (tensor cores, fp32
        accumulation) or "fp32" (CUDA cores, the numbers of the float64 checker to fp32
        rounding).  Weights, gradients and optimizer state are fp32 either way."""
        p = init_params(seed) if params is None else np.ascontiguousarray(params, np.float32)
        if p.size != param_count():
            raise ValueError(f"expected {param_count()} parameters, got {p.size}")
        self._free = _lib.lib.st_encoder_destroy
        self._h = ctypes.c_void_p()
        err = _lib.st_error()
        _lib.check(_lib.lib.st_encoder_create(p.ctypes.data, ctypes.byref(self._h),
                                              ctypes.byref(err)), err)
        self.set_precision(precision)

    def set_precision(self, precision: str) -> None:
        code = {"fp32": 0, "bf16": 1}.get(precision)
        if code is None:
            raise ValueError("precision is 'bf16' or 'fp32'")
        err = _lib.st_error()
        _lib.check(_lib.lib.st_encoder_set_precision(self._h, code, ctypes.byref(err)), err)
        self.precision = precision

    def save(self, path, meta: dict | None = None) -> None:
        """Writes the weights (and ``meta``) to a model file, atomically (see ``encode_model``)."""
        atomic_write(path, encode_model(self.params(), meta))

    @classmethod
    def load(cls, path, precision: str = "bf16") -> "Encoder":
        """An encoder with the weights of a model file; its metadata is in ``.meta``.  Raises
        ValueError for a file that is not a version-1 encoder file or is truncated / corrupt."""
        with open(path, "rb") as f:
            params, meta = decode_model(f.read(), os.fspath(path))
        if params.size != param_count():
            raise ValueError(f"seqtree_b200: '{os.fspath(path)}' holds {params.size} parameters; "
                             f"this encoder has {param_count()}")
        enc = cls(params, precision=precision)
        enc.meta = meta
        return enc

    def params(self) -> np.ndarray:
        out = np.empty(param_count(), np.float32)
        err = _lib.st_error()
        _lib.check(_lib.lib.st_encoder_get_params(self._h, out.ctypes.data, ctypes.byref(err)), err)
        return out

    @staticmethod
    def _batch(codes, lens, scores):
        codes = np.ascontiguousarray(codes, np.uint8)
        lens = np.ascontiguousarray(lens, np.int32)
        scores = np.ascontiguousarray(scores, np.int32)
        S = lens.size
        if codes.shape != (S, PAD) or scores.size != S // 2:
            raise ValueError("batch: codes [S, 32], lens [S], scores [S/2]")
        return codes, lens, scores, S

    def loss_grad(self, codes, lens, scores, grad: bool = True):
        codes, lens, scores, S = self._batch(codes, lens, scores)
        loss = ctypes.c_float()
        g = np.empty(param_count(), np.float32) if grad else None
        err = _lib.st_error()
        _lib.check(_lib.lib.st_encoder_loss_grad(
            self._h, codes.ctypes.data, lens.ctypes.data, scores.ctypes.data, S,
            ctypes.byref(loss), None if g is None else g.ctypes.data, ctypes.byref(err)), err)
        return float(loss.value), g

    def train_step(self, codes, lens, scores, lr: float) -> float:
        codes, lens, scores, S = self._batch(codes, lens, scores)
        loss = ctypes.c_float()
        err = _lib.st_error()
        _lib.check(_lib.lib.st_encoder_train_step(
            self._h, codes.ctypes.data, lens.ctypes.data, scores.ctypes.data, S, float(lr),
            ctypes.byref(loss), ctypes.byref(err)), err)
        return float(loss.value)

    def embed_into(self, seqset, out_ptr: int, layout: int = 0, stream: int = 0) -> None:
        """Embeddings of a device set: layout 0 fp32 [n][64] (fp32 forward), 1 bf16 swizzled
        [n][64] (bf16 tensor-core inference), 2 the fp32 forward in layout 1's format."""
        err = _lib.st_error()
        _lib.check(_lib.lib.st_encoder_embed(self._h, seqset.handle, ctypes.c_void_p(out_ptr),
                                             int(layout), ctypes.c_void_p(stream),
                                             ctypes.byref(err)), err)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._free(h)
            self._h = None


def pair_scores(qset, rset, qi_ptr: int, ri_ptr: int, n: int, out_ptr: int, stream: int = 0, *,
                matrix: SubstitutionMatrix | None, gap_open: int, gap_extend: int = 1, prior=(),
                prior_width: int = 0) -> None:
    """Exact gap-block scores of the listed pairs (device int32 index arrays and output)."""
    pen = None if matrix is None else np.ascontiguousarray(matrix.penalty_grid, np.int32)
    pr = np.ascontiguousarray(np.asarray(prior, dtype=np.int64).astype(np.int32)).ravel()
    err = _lib.st_error()
    code = _lib.lib.st_gapblock_pairs_sets(
        qset.handle, rset.handle, ctypes.c_void_p(qi_ptr), ctypes.c_void_p(ri_ptr), int(n),
        _lib.i32_ptr(pen), 0 if pen is None else pen.shape[0], gap_open, gap_extend,
        _lib.i32_ptr(pr) if pr.size else None, int(pr.size), int(prior_width),
        ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream), ctypes.byref(err))
    _lib.check(code, err)


def swizzle_rows(x):
    """bf16 [n][64] rows in the proposal kernel's operand layout: the eight 16-byte chunks of row
    r stored at chunk ^ (r & 7) (what ``Encoder.embed_into(..., layout=1)`` writes)."""
    import torch
    n = x.shape[0]
    if x.dim() != 2 or x.shape[1] != 64:
        raise ValueError("embeddings must be [n, 64]")
    chunks = x.to(torch.bfloat16).reshape(n, 8, 8)
    perm = torch.arange(8, device=x.device)[None, :] ^ (torch.arange(n, device=x.device)[:, None] & 7)
    out = torch.empty_like(chunks)
    out.scatter_(1, perm[:, :, None].expand(n, 8, 8), chunks)
    return out.reshape(n, 64).contiguous()


def propose_topk_into(q_ptr: int, nq: int, r_ptr: int, nr: int, k: int, ids_ptr: int,
                      scores_ptr: int = 0, stream: int = 0, ranges_ptr: int = 0) -> None:
    """``st_propose_topk`` on device pointers (swizzled bf16 embeddings in, [nq][k] out); with
    ``ranges_ptr`` (device int32, two per 256-query tile) ``st_propose_topk_ranges``."""
    err = _lib.st_error()
    if ranges_ptr:
        code = _lib.lib.st_propose_topk_ranges(
            ctypes.c_void_p(q_ptr), int(nq), ctypes.c_void_p(r_ptr), int(nr), int(k),
            ctypes.c_void_p(ranges_ptr), ctypes.c_void_p(ids_ptr),
            ctypes.c_void_p(scores_ptr or None), ctypes.c_void_p(stream), ctypes.byref(err))
    else:
        code = _lib.lib.st_propose_topk(ctypes.c_void_p(q_ptr), int(nq), ctypes.c_void_p(r_ptr),
                                        int(nr), int(k), ctypes.c_void_p(ids_ptr),
                                        ctypes.c_void_p(scores_ptr or None),
                                        ctypes.c_void_p(stream), ctypes.byref(err))
    _lib.check(code, err)


QUERY_TILE, REF_TILE = 256, 128  # the proposal kernel's tile heights


def propose_range_into(q_ptr: int, nq: int, qlens_ptr: int, r_ptr: int, nr: int, rlens_ptr: int,
                       thresholds: np.ndarray, pq_ptr: int, pr_ptr: int, capacity: int,
                       stream: int = 0, ranges_ptr: int = 0) -> int:
    """``st_propose_range`` on device pointers: writes up to ``capacity`` (query, ref) pairs whose
    dot product reaches ``thresholds[qlen, rlen]`` (float32 [33, 33]) and returns how many pass in
    all (synchronous)."""
    thr = np.ascontiguousarray(thresholds, np.float32)
    if thr.shape != (PAD + 1, PAD + 1):
        raise ValueError("thresholds must be float32 [33, 33]")
    count = ctypes.c_int64()
    err = _lib.st_error()
    _lib.check(_lib.lib.st_propose_range(
        ctypes.c_void_p(q_ptr), int(nq), ctypes.c_void_p(qlens_ptr), ctypes.c_void_p(r_ptr),
        int(nr), ctypes.c_void_p(rlens_ptr), thr.ctypes.data, ctypes.c_void_p(ranges_ptr or None),
        ctypes.c_void_p(pq_ptr or None), ctypes.c_void_p(pr_ptr or None), int(capacity),
        ctypes.byref(count), ctypes.c_void_p(stream), ctypes.byref(err)), err)
    return int(count.value)


def embed_dots_into(q_ptr: int, nq: int, r_ptr: int, nr: int, qi_ptr: int, ri_ptr: int, n: int,
                    out_ptr: int, stream: int = 0) -> None:
    """``st_embed_dots``: fp32 dot products of listed pairs of swizzled bf16 embeddings."""
    err = _lib.st_error()
    _lib.check(_lib.lib.st_embed_dots(
        ctypes.c_void_p(q_ptr), int(nq), ctypes.c_void_p(r_ptr), int(nr), ctypes.c_void_p(qi_ptr),
        ctypes.c_void_p(ri_ptr), int(n), ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream),
        ctypes.byref(err)), err)


def propose_range(q_emb, q_lens, r_emb, r_lens, thresholds, capacity: int | None = None,
                  ranges=None):
    """Every (query, ref) pair of swizzled bf16 embeddings (torch CUDA [n][64]) whose dot product
    is >= ``thresholds[len q, len r]``; lengths are uint8 CUDA tensors.  Returns (query idx,
    ref idx) int32 tensors in no particular order (the call is repeated at the exact size when
    the first ``capacity`` did not hold every pair)."""
    import torch
    nq, nr = q_emb.shape[0], r_emb.shape[0]
    cap = max(1, nq * 16) if capacity is None else max(1, int(capacity))
    stream = torch.cuda.current_stream(q_emb.device).cuda_stream
    while True:
        pq = torch.empty(cap, dtype=torch.int32, device=q_emb.device)
        pr = torch.empty(cap, dtype=torch.int32, device=q_emb.device)
        n = propose_range_into(q_emb.data_ptr(), nq, q_lens.data_ptr(), r_emb.data_ptr(), nr,
                               r_lens.data_ptr(), thresholds, pq.data_ptr(), pr.data_ptr(), cap,
                               stream, 0 if ranges is None else ranges.data_ptr())
        if n <= cap:
            return pq[:n], pr[:n]
        cap = n


def range_tile_ranges(q_lens_sorted: np.ndarray, r_lens_sorted: np.ndarray,
                      thresholds: np.ndarray) -> np.ndarray:
    """Per 256-query tile of length-sorted queries, the [first, last) 128-ref tiles of
    length-sorted refs spanning every ref length that has a finite threshold for some query length
    of the tile (int32 [tiles, 2]); tiles without one get an empty range."""
    q = np.asarray(q_lens_sorted, np.int64)
    r = np.asarray(r_lens_sorted, np.int64)
    finite = np.isfinite(np.asarray(thresholds, np.float32))
    nt = -(-q.size // QUERY_TILE)
    out = np.zeros((nt, 2), np.int32)
    for t in range(nt):
        blk = q[t * QUERY_TILE:(t + 1) * QUERY_TILE]
        on = finite[np.clip(blk.min(), 0, PAD):np.clip(blk.max(), 0, PAD) + 1].any(axis=0)
        ls = np.flatnonzero(on)
        if ls.size == 0:
            continue
        lo = np.searchsorted(r, ls[0], side="left")
        hi = np.searchsorted(r, ls[-1], side="right")
        out[t] = (lo // REF_TILE, -(-hi // REF_TILE)) if hi > lo else (0, 0)
    return out


# Cost weights of the threshold form's fallback choice, seconds per unit on one B200: an
# exhaustively scored pair (sparse gap-block kernel), a scanned (query, ref) pair of the threshold
# proposal kernel, and a rescored candidate pair (pair kernel and its filtering).  Calibration
# measures the exhaustive and candidate costs on its batch when the batch is large enough to
# fill the GPU and keeps these otherwise; only the ratios matter to the choice.
RANGE_COSTS = {"exhaustive": 1 / 3.0e11, "scan": 1 / 2.5e12, "candidate": 1 / 6.0e9}
# Candidate pairs one proposal block may hold (the search splits its queries into blocks).
RANGE_BLOCK_PAIRS = 1 << 27
# Recall levels a cell's threshold can take (fraction of the cell's calibration hits kept).
RANGE_LEVELS = (0.5, 0.75, 0.9, 0.95, 0.98, 0.99, 0.995, 1.0)


def band_tile_ranges(q_lens_sorted: np.ndarray, r_lens_sorted: np.ndarray, band: int) -> np.ndarray:
    """Per 256-query tile of length-sorted queries, the [first, last) 128-ref tiles of
    length-sorted refs that hold every ref whose length is within ``band`` of a query of the
    tile (int32 [tiles, 2])."""
    q = np.asarray(q_lens_sorted, np.int64)
    r = np.asarray(r_lens_sorted, np.int64)
    nt = -(-q.size // QUERY_TILE)
    out = np.zeros((nt, 2), np.int32)
    for t in range(nt):
        blk = q[t * QUERY_TILE:(t + 1) * QUERY_TILE]
        lo = np.searchsorted(r, blk.min() - band, side="left")
        hi = np.searchsorted(r, blk.max() + band, side="right")
        out[t] = (lo // REF_TILE, -(-hi // REF_TILE)) if hi > lo else (0, 0)
    return out


def propose_topk(q_emb, r_emb, k: int = 256):
    """Top-k refs per query by dot product of swizzled bf16 embeddings (torch CUDA tensors
    [n][64]); returns (ids int32 [nq][k], scores float32 [nq][k]), best first."""
    import torch
    nq, nr = q_emb.shape[0], r_emb.shape[0]
    ids = torch.empty((nq, k), dtype=torch.int32, device=q_emb.device)
    scores = torch.empty((nq, k), dtype=torch.float32, device=q_emb.device)
    stream = torch.cuda.current_stream(q_emb.device).cuda_stream
    propose_topk_into(q_emb.data_ptr(), nq, r_emb.data_ptr(), nr, k, ids.data_ptr(),
                      scores.data_ptr(), stream)
    stream_status(stream)
    return ids, scores


def train_gemm_bf16(a, b, c, *, trans_a: bool = False, trans_b: bool = False,
                    accumulate: bool = False) -> None:
    """The encoder's training GEMM (``st_train_gemm_bf16``) on fp32 CUDA matrices:
    ``c = op(a) @ op(b)`` (``+=`` when ``accumulate``), op the transpose when asked, products in
    bf16 with fp32 accumulation.  Row-major operands with unit column stride."""
    import torch
    for t in (a, b, c):
        if t.dtype != torch.float32 or t.dim() != 2 or not t.is_cuda or t.stride(1) != 1:
            raise ValueError("train_gemm_bf16: 2-d fp32 CUDA matrices with unit column stride")
    M, K = (a.shape[1], a.shape[0]) if trans_a else (a.shape[0], a.shape[1])
    K2, N = (b.shape[1], b.shape[0]) if trans_b else (b.shape[0], b.shape[1])
    if K2 != K or tuple(c.shape) != (M, N):
        raise ValueError("train_gemm_bf16: shapes do not chain")
    err = _lib.st_error()
    _lib.check(_lib.lib.st_train_gemm_bf16(
        int(trans_a), int(trans_b), M, N, K, ctypes.c_void_p(a.data_ptr()), max(a.stride(0), 1),
        ctypes.c_void_p(b.data_ptr()), max(b.stride(0), 1), ctypes.c_void_p(c.data_ptr()),
        max(c.stride(0), 1), int(accumulate),
        ctypes.c_void_p(torch.cuda.current_stream(c.device).cuda_stream), ctypes.byref(err)), err)


def stream_status(stream: int = 0) -> None:
    """Synchronise ``stream`` and raise if a bounded device-side wait gave up since the last
    check."""
    err = _lib.st_error()
    _lib.check(_lib.lib.st_stream_status(ctypes.c_void_p(stream), ctypes.byref(err)), err)


# ----------------------------------------------------------------------------- data ---------
# The CDR3-like generators (cdr3_lengths, cdr3_codes, codes_to_strings) live in
# seqtree_b200.workloads, which loads no compiled code; they are re-exported here.


def codes_to_packed(codes: np.ndarray, lens: np.ndarray) -> _lib.Packed:
    """Codes [n, 32] + lengths as one concatenated letter buffer (for ``device.SeqSet``)."""
    return _lib.Packed.from_arrays(*codes_to_letters(codes, lens))


def cdr3_like(seed: int, n: int) -> list[str]:
    """:func:`cdr3_codes` as strings."""
    return codes_to_strings(*cdr3_codes(seed, n))


def mutate_codes(codes: np.ndarray, lens: np.ndarray, rng, long_share: float = 0.0,
                 long_max: int = 16) -> tuple[np.ndarray, np.ndarray]:
    """Near neighbours: 1-3 random substitutions, then one random indel block of 1-3 residues at
    a random position (a deletion or an insertion with equal odds, whichever keeps 1..32
    residues; a deletion near the end removes what is there).  A ``long_share`` of the pairs
    takes a block of 4..``long_max`` residues instead: the gap blocks through which a short
    junction matches a longer one."""
    n = lens.size
    out = codes.copy()
    rows = np.arange(n)
    nsub = rng.integers(1, 4, size=n)
    for t in range(3):
        pos = np.minimum((rng.random(n) * lens).astype(np.int64), lens - 1)
        aa = _AA20_CODES[rng.integers(0, 20, size=n)]
        m = t < nsub
        out[rows[m], pos[m]] = aa[m]
    blk = rng.integers(1, 4, size=n)
    if long_share > 0:
        blk = np.where(rng.random(n) < long_share, rng.integers(4, long_max + 1, size=n), blk)
    pos = np.minimum((rng.random(n) * (lens + 1)).astype(np.int64), lens)
    want_del = rng.random(n) < 0.5
    dele = want_del & (lens - blk >= 1)
    ins = ~dele & (lens + blk <= PAD)
    gone = np.minimum(blk, lens - pos)
    j = np.arange(PAD)[None, :]
    p, b, g = pos[:, None], blk[:, None], gone[:, None]
    src = np.where(dele[:, None], np.where(j < p, j, j + g),
                   np.where(ins[:, None], np.where(j < p, j, j - b), j))
    res = np.take_along_axis(out, np.clip(src, 0, PAD - 1), axis=1)
    new = ins[:, None] & (j >= p) & (j < p + b)
    res[new] = _AA20_CODES[rng.integers(0, 20, size=int(new.sum()))]
    nl = np.where(dele, lens - gone, np.where(ins, lens + blk, lens)).astype(np.int32)
    res[j >= nl[:, None]] = 0
    return res, nl


def mutate(seqs, rng) -> list[str]:
    """:func:`mutate_codes` on strings."""
    codes, lens = pad_codes(list(seqs))
    return codes_to_strings(*mutate_codes(codes, lens, rng))


def training_pairs_codes(seed: int, n_pairs: int, long_share: float = 0.0,
                         long_max: int = 16) -> tuple[np.ndarray, np.ndarray]:
    """n_pairs seeded pairs as interleaved codes [2n, 32] / lengths [2n] (rows 2i and 2i+1 are
    one pair): the first half near neighbours made by :func:`mutate_codes`, the second half two
    independent CDR3-like junctions."""
    rng = np.random.default_rng(seed)
    a, la = cdr3_codes(seed * 2 + 1, n_pairs)
    near = n_pairs // 2
    b, lb = cdr3_codes(seed * 2 + 2, n_pairs)
    b[:near], lb[:near] = mutate_codes(a[:near], la[:near], rng, long_share, long_max)
    codes = np.empty((2 * n_pairs, PAD), np.uint8)
    lens = np.empty(2 * n_pairs, np.int32)
    codes[0::2], codes[1::2] = a, b
    lens[0::2], lens[1::2] = la, lb
    return codes, lens


def training_pairs(seed: int, n_pairs: int):
    """:func:`training_pairs_codes` as two lists of strings (a[i], b[i])."""
    codes, lens = training_pairs_codes(seed, n_pairs)
    s = codes_to_strings(codes, lens)
    return s[0::2], s[1::2]


# ------------------------------------------------------------------------- training ---------
def label_pairs(codes: np.ndarray, lens: np.ndarray, *, matrix, gap_open: int,
                gap_extend: int = 1) -> np.ndarray:
    """Exact gap-block scores of the interleaved pairs (rows 2i, 2i+1), by the GPU pair scorer."""
    import torch

    from .device import SeqSet
    n = lens.size // 2
    ss = SeqSet(codes_to_packed(codes, lens), "aa")
    qi = torch.arange(0, 2 * n, 2, dtype=torch.int32, device="cuda")
    ri = qi + 1
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    pair_scores(ss, ss, qi.data_ptr(), ri.data_ptr(), n, out.data_ptr(), stream, matrix=matrix,
                gap_open=gap_open, gap_extend=gap_extend)
    return out.cpu().numpy()


def mine_partners(codes: np.ndarray, lens: np.ndarray, rows: np.ndarray, *, seed: int, tries: int,
                  matrix, gap_open: int, gap_extend: int = 1) -> None:
    """Replaces the partner (odd row) of every pair in ``rows`` by the best-scoring of ``tries``
    random CDR3-like junctions (exact gap-block score, lowest wins), in place.  The pairs become
    'hard' random pairs whose scores sit near the search threshold instead of far above it."""
    import torch

    from .device import SeqSet
    n = rows.size
    if n == 0 or tries < 1:
        return
    pool_n = max(4096, min(1 << 20, n * tries // 4))
    pc, pl = cdr3_codes(seed, pool_n)
    a_codes, a_lens = codes[2 * rows], lens[2 * rows]
    aset = SeqSet(codes_to_packed(a_codes, a_lens), "aa")
    pset = SeqSet(codes_to_packed(pc, pl), "aa")
    rng = np.random.default_rng(seed + 1)
    cand = rng.integers(0, pool_n, size=(n, tries)).astype(np.int32)
    qi = torch.arange(n, dtype=torch.int32, device="cuda").repeat_interleave(tries)
    ri = torch.from_numpy(cand.ravel()).cuda()
    sc = torch.empty(n * tries, dtype=torch.int32, device="cuda")
    pair_scores(aset, pset, qi.data_ptr(), ri.data_ptr(), n * tries, sc.data_ptr(),
                torch.cuda.current_stream().cuda_stream, matrix=matrix, gap_open=gap_open,
                gap_extend=gap_extend)
    best = sc.view(n, tries).argmin(dim=1).cpu().numpy()
    pick = cand[np.arange(n), best]
    codes[2 * rows + 1] = pc[pick]
    lens[2 * rows + 1] = pl[pick]


def train(enc: Encoder, n_pairs: int, *, seed: int, matrix, gap_open: int, gap_extend: int = 1,
          batch_pairs: int = 2048, lr: float = 2e-3, lr_final: float = 1e-4,
          chunk_pairs: int = 1 << 20, mine: int = 0, long_share: float = 0.0,
          long_max: int = 16, log=None) -> list[float]:
    """Trains ``enc`` for one pass over ``n_pairs`` fresh seeded pairs labelled by the exact
    kernel (Adam, cosine learning-rate decay from ``lr`` to ``lr_final``).  Half the pairs are
    near neighbours (:func:`mutate_codes`, ``long_share`` of them with an indel block of
    4..``long_max`` residues); the other half are random pairs, each the best of ``mine``
    random partners when ``mine`` > 0 (:func:`mine_partners`).  Returns the mean loss of every
    chunk."""
    steps = max(1, -(-n_pairs // batch_pairs))
    t, losses = 0, []
    for c0 in range(0, n_pairs, chunk_pairs):
        m = min(chunk_pairs, n_pairs - c0)
        cseed = seed * 7919 + c0 // chunk_pairs
        codes, lens = training_pairs_codes(cseed, m, long_share, long_max)
        if mine:
            mine_partners(codes, lens, np.arange(m // 2, m), seed=cseed * 31 + 5, tries=mine,
                          matrix=matrix, gap_open=gap_open, gap_extend=gap_extend)
        perm = np.random.default_rng(cseed + 3).permutation(m)  # mix the two halves
        codes = codes.reshape(m, 2, PAD)[perm].reshape(2 * m, PAD)
        lens = lens.reshape(m, 2)[perm].reshape(2 * m)
        scores = label_pairs(codes, lens, matrix=matrix, gap_open=gap_open, gap_extend=gap_extend)
        acc = []
        for b0 in range(0, m, batch_pairs):
            b1 = min(m, b0 + batch_pairs)
            if b1 - b0 < 2:
                continue
            cur = lr_final + (lr - lr_final) * 0.5 * (1.0 + np.cos(np.pi * t / steps))
            acc.append(enc.train_step(codes[2 * b0:2 * b1], lens[2 * b0:2 * b1], scores[b0:b1],
                                      lr=float(cur)))
            t += 1
        losses.append(float(np.mean(acc)) if acc else float("nan"))
        if log:
            log(f"pairs {c0 + m}/{n_pairs}: loss {losses[-1]:.4f}")
    return losses


def allocate_recall(E, FL, CL, wq, wr, costs: dict, target: float):
    """The threshold form's plan: per (query length, ref length) cell a recall level (index into
    the last axis of ``FL`` / ``CL``, -1 = no proposals) and the query / ref lengths scored
    exhaustively, chosen greedily until the estimated recall reaches ``target``.

    ``E`` [S, S] holds the calibration batch's exact hits per cell, ``FL`` / ``CL`` [S, S, LV] the
    hits found and the candidates proposed at each level (non-decreasing along the level axis),
    ``wq`` / ``wr`` the query and ref counts per length; ``costs`` gives seconds per exhaustively
    scored pair ("exhaustive"), per scanned pair ("scan") and per candidate ("candidate").  A query
    length's proposals scan every ref whose length lies between the shortest and the longest
    ref length it has a cell on for (refs are sorted by length), so switching a cell on may widen
    that span.  Every step takes the move with the most recovered hits per added second:
    raising one cell by one level, or scoring one query or ref length exhaustively (its cells
    are then exact and cost their pairs).  Returns (level, query lengths, ref lengths, estimated
    recall, estimated seconds)."""
    E = np.asarray(E, np.float64)
    S, LV = E.shape[0], FL.shape[2]
    wq, wr = np.asarray(wq, np.float64), np.asarray(wr, np.float64)
    pairs = np.outer(wq, wr)
    exh = costs["exhaustive"] * pairs
    cum_r = np.concatenate([[0.0], np.cumsum(wr)])
    level = np.full((S, S), -1, np.int64)
    covered = np.zeros((S, S), bool)
    q_fb, r_fb = [], []

    def at(arr, lv):
        v = np.take_along_axis(arr, np.clip(lv, 0, LV - 1)[:, :, None], 2)[:, :, 0]
        return np.where(lv >= 0, v, 0.0)

    def row_scan(a, on_row):
        on = np.flatnonzero(on_row)
        if on.size == 0:
            return 0.0
        return costs["scan"] * wq[a] * (cum_r[on[-1] + 1] - cum_r[on[0]])

    def total(lv, cov):
        on = (lv >= 0) & ~cov
        t = exh[cov].sum() + costs["candidate"] * at(CL, lv)[on].sum()
        return t + sum(row_scan(a, on[a]) for a in range(S))

    te = E.sum()
    now = total(level, covered)
    while te:
        fnd = at(FL, level)
        if (E[covered].sum() + fnd[~covered].sum()) / te >= target:
            break
        best, move = 0.0, None
        on = (level >= 0) & ~covered
        for a, b in zip(*np.where(~covered & (E > 0) & (level < LV - 1))):
            nl = level[a, b] + 1
            gain = FL[a, b, nl] - fnd[a, b]
            dt = costs["candidate"] * (CL[a, b, nl] - (CL[a, b, nl - 1] if nl > 0 else 0.0))
            if nl == 0:
                row = on[a].copy()
                row[b] = True
                dt += row_scan(a, row) - row_scan(a, on[a])
            if gain > 0 and gain / max(dt, 1e-15) > best:
                best, move = gain / max(dt, 1e-15), ("cell", a, b)
        for side, w, taken in (("q", wq, q_fb), ("r", wr, r_fb)):
            for x in range(S):
                if w[x] == 0 or x in taken:
                    continue
                cov = covered.copy()
                if side == "q":
                    cov[x, :] = True
                else:
                    cov[:, x] = True
                gain = (E - fnd)[cov & ~covered].sum()
                dt = total(level, cov) - now
                if gain > 0 and gain / max(dt, 1e-15) > best:
                    best, move = gain / max(dt, 1e-15), (side, x)
        if move is None:
            break
        if move[0] == "cell":
            level[move[1], move[2]] += 1
        elif move[0] == "q":
            q_fb.append(move[1])
            covered[move[1], :] = True
        else:
            r_fb.append(move[1])
            covered[:, move[1]] = True
        now = total(level, covered)
    level[covered] = -1
    rec = (E[covered].sum() + at(FL, level)[~covered].sum()) / te if te else 1.0
    return level, sorted(q_fb), sorted(r_fb), float(rec), float(total(level, covered))


# -------------------------------------------------------------------------- search ----------
def _subset(codes, lens, rows):
    from .device import SeqSet
    return SeqSet(codes_to_packed(codes[rows], lens[rows]), "aa") if rows.size else None


def gather_rows(data: np.ndarray, offsets: np.ndarray, rows: np.ndarray):
    """(bytes, offsets) of the listed rows of a packed string set, in the listed order (one copy
    per row in the ``_pack`` extension when it is built)."""
    rows = np.ascontiguousarray(rows, np.int64)
    if _lib._pack is not None:
        d, o = _lib._pack.gather(np.ascontiguousarray(data, np.uint8),
                                 np.ascontiguousarray(offsets, np.int64), rows)
        return np.frombuffer(d, np.uint8), np.frombuffer(o, np.int64)
    sl = (offsets[rows + 1] - offsets[rows]).astype(np.int64)
    off = np.zeros(rows.size + 1, np.int64)
    np.cumsum(sl, out=off[1:])
    src = np.repeat(offsets[rows] - off[:-1], sl) + np.arange(off[-1], dtype=np.int64)
    return data[src], off


def _packed_subset(packed: _lib.Packed, rows: np.ndarray):
    """The listed rows of a packed string set as a device set (letters gathered on the host and
    encoded on the device, so an invalid symbol raises the alphabet's ValueError)."""
    from .device import SeqSet
    if not rows.size:
        return None
    return SeqSet(_lib.Packed.from_arrays(*gather_rows(packed.data, packed.offsets, rows)), "aa")


class QueryBatch:
    """Queries resident on the device for :meth:`LearnedIndex.search`, split by the index's
    query-length fallback: ``learn`` rows go through the proposals, ``fb`` rows through the
    exhaustive kernel."""

    def __init__(self, index: "LearnedIndex", codes: np.ndarray | None, lens: np.ndarray,
                 packed: _lib.Packed | None = None):
        """From padded codes [n, 32] and lengths, or (``codes`` None) from a packed string set
        whose lengths are ``lens``."""
        import torch
        self.lens = np.asarray(lens, np.int32)
        self.count = int(self.lens.size)
        fb = index.query_fallback[np.clip(self.lens, 0, PAD)]
        self.fb_rows = np.flatnonzero(fb).astype(np.int64)
        learn = np.flatnonzero(~fb).astype(np.int64)
        # learn rows in length order, so that a 256-query tile of the proposal kernel spans few
        # lengths (its ref band is then narrow)
        # (lengths are 1..32: as uint8 the stable sort is numpy's radix sort)
        self.learn_rows = learn[np.argsort(np.clip(self.lens[learn], 0, 255).astype(np.uint8),
                                           kind="stable")]
        if codes is None:
            self.fb_set = _packed_subset(packed, self.fb_rows)
            self.learn_set = _packed_subset(packed, self.learn_rows)
        else:
            self.fb_set = _subset(codes, self.lens, self.fb_rows)
            self.learn_set = _subset(codes, self.lens, self.learn_rows)
        self.fb_rows_t = torch.from_numpy(self.fb_rows).cuda()
        self.learn_rows_t = torch.from_numpy(self.learn_rows).cuda()
        self.learn_lens_t = torch.from_numpy(
            np.clip(self.lens[self.learn_rows], 0, PAD).astype(np.uint8)).cuda()
        self.ranges = None
        if index.band is not None and self.learn_rows.size and index.n_learn:
            r = band_tile_ranges(self.lens[self.learn_rows], index.learn_lens, index.band)
            self.ranges = torch.from_numpy(r.ravel()).cuda()
        self._range_key = None

    def range_tiles(self, index: "LearnedIndex"):
        """The threshold form's per-tile ref ranges for the index's current thresholds."""
        import torch
        key = (index._thr_version, index.n_learn)
        if self._range_key != key:
            r = range_tile_ranges(self.lens[self.learn_rows], index.learn_lens, index.thresholds)
            self.ranges_thr = torch.from_numpy(r.ravel()).cuda()
            self._range_key = key
        return self.ranges_thr


class LearnedIndex:
    """Thresholded gap-block search by learned proposal + exact rescore.

    The refs outside the ref-length fallback are embedded once (:meth:`embed_refs`).
    :meth:`search` embeds the queries outside the query-length fallback, proposes the top ``k``
    of those refs for each by embedding similarity (``st_propose_topk``), rescores every
    proposal with the exact gap-block kernel and keeps those with score <= ``max_penalty``.  The
    exhaustive sparse kernel answers the two fallback parts exactly: fallback-length queries
    against every ref, and the other queries against the fallback-length refs.  Every reported
    score is exact; rows are CSR with refs ascending, the format of ``score_sparse``.
    :meth:`calibrate` chooses the fallback lengths on a held-out batch.

    ``k = 0`` turns the proposals off: the index is then the method without the network (the
    calibrated exhaustive fallback alone), the baseline the encoder is measured against.

    ``proposal="range"`` replaces the top-k by thresholds: every (query, ref) pair whose
    embedding dot product reaches the threshold of its (query length, ref length) cell is
    proposed (``st_propose_range``), so no per-query selection is kept and a query proposes as
    many refs as its cells let through.  :meth:`calibrate` then sets each cell's threshold from
    the embeddings of the cell's exact hits on the held-out batch and chooses the fallback
    lengths by estimated cost (``k`` only switches the network on, ``k = 0`` off).
    """

    def __init__(self, encoder: Encoder | None, ref_codes: np.ndarray, ref_lens: np.ndarray, *,
                 matrix, gap_open: int, gap_extend: int = 1, max_penalty: int = 24, k: int = 256,
                 band: int | None = None, proposal: str = "topk"):
        """``band``: when set, a query's proposals come only from refs whose length differs from
        the query tile's lengths by at most ``band`` (refs and queries sorted by length, each
        256-query tile scanning its band of ref tiles); None scans every ref (top-k form only;
        the threshold form scans the ref lengths its thresholds leave on)."""
        from .device import SeqSet
        if max_penalty < 0:
            raise ValueError("max_penalty must be >= 0")
        if k < 0 or (k > 0 and encoder is None):
            raise ValueError("k must be >= 0, and k > 0 needs an encoder")
        if band is not None and band < 0:
            raise ValueError("band must be >= 0 or None")
        if proposal not in ("topk", "range"):
            raise ValueError("proposal is 'topk' or 'range'")
        self.proposal = proposal
        self.thresholds = np.full((PAD + 1, PAD + 1), np.inf, np.float32)
        self._thr_version = 0
        self._range_per_query = 16.0
        self.band = band
        self.encoder, self.matrix = encoder, matrix
        self.gap_open, self.gap_extend, self.max_penalty, self.k = gap_open, gap_extend, max_penalty, k
        self.ref_codes = np.ascontiguousarray(ref_codes, np.uint8)
        self.ref_lens = np.asarray(ref_lens, np.int32)
        self.nr = int(self.ref_lens.size)
        self.refs = SeqSet(codes_to_packed(self.ref_codes, self.ref_lens), "aa")
        self.query_fallback = np.zeros(PAD + 1, bool)
        self.ref_fallback = np.zeros(PAD + 1, bool)
        self._hits = None
        self._build()

    def save_model(self, path) -> None:
        """Writes the encoder and this index's search settings and calibrated fallback lengths to
        one model file, so another process can answer searches without training or calibrating
        (:meth:`from_model`)."""
        if self.encoder is None:
            raise ValueError("an index without an encoder has no model to save")
        self.encoder.save(path, {
            "k": self.k, "band": self.band, "max_penalty": self.max_penalty, "gap_open": self.gap_open,
            "gap_extend": self.gap_extend,
            "query_fallback": np.flatnonzero(self.query_fallback).tolist(),
            "ref_fallback": np.flatnonzero(self.ref_fallback).tolist(),
            "proposal": self.proposal,
            "thresholds": [[float(x) if np.isfinite(x) else None for x in row]
                           for row in self.thresholds]})

    @classmethod
    def from_model(cls, path, ref_codes: np.ndarray, ref_lens: np.ndarray, *, matrix,
                   precision: str = "bf16") -> "LearnedIndex":
        """An index over ``ref_codes`` with the encoder, settings and fallback lengths of a model
        file written by :meth:`save_model` (the matrix is the caller's: it is not stored)."""
        enc = Encoder.load(path, precision=precision)
        m = enc.meta
        idx = cls(enc, ref_codes, ref_lens, matrix=matrix, gap_open=int(m["gap_open"]),
                  gap_extend=int(m["gap_extend"]), max_penalty=int(m["max_penalty"]),
                  k=int(m["k"]), band=m.get("band"), proposal=m.get("proposal", "topk"))
        idx.set_fallback(m["query_fallback"], m["ref_fallback"])
        if m.get("thresholds") is not None:
            idx.set_thresholds(np.array([[np.inf if x is None else x for x in row]
                                         for row in m["thresholds"]], np.float32))
        return idx

    def set_thresholds(self, thresholds) -> None:
        """The threshold form's dot-product threshold per (query length, ref length) cell
        (float32 [33, 33]; +inf leaves a cell without proposals)."""
        t = np.array(thresholds, np.float32)
        if t.shape != (PAD + 1, PAD + 1) or np.isnan(t).any():
            raise ValueError("thresholds must be a float [33, 33] table without NaN")
        self.thresholds = t
        self._thr_version += 1

    def set_fallback(self, query_lengths=(), ref_lengths=()) -> None:
        self.query_fallback[:] = False
        self.ref_fallback[:] = False
        self.query_fallback[list(query_lengths)] = True
        self.ref_fallback[list(ref_lengths)] = True
        self._build()

    def _build(self) -> None:
        import torch
        fb = self.ref_fallback[np.clip(self.ref_lens, 0, PAD)]
        learn = np.flatnonzero(~fb).astype(np.int64)
        learn = learn[np.argsort(np.clip(self.ref_lens[learn], 0, 255).astype(np.uint8),
                                 kind="stable")]  # by length, then id
        fbr = np.flatnonzero(fb).astype(np.int64)
        self.learn_lens = self.ref_lens[learn]
        self.learn_lens_t = torch.from_numpy(
            np.clip(self.learn_lens, 0, PAD).astype(np.uint8)).cuda()
        self.learn_ids = torch.from_numpy(learn.astype(np.int32)).cuda()
        self.fb_ref_ids = torch.from_numpy(fbr.astype(np.int32)).cuda()
        self.learn_refs = _subset(self.ref_codes, self.ref_lens, learn)
        self.fb_refs = _subset(self.ref_codes, self.ref_lens, fbr)
        self.n_learn = int(learn.size)
        self.r_emb = torch.empty((self.n_learn if self.k else 0, 64), dtype=torch.bfloat16,
                                 device="cuda")
        self.embed_refs()

    def embed_refs(self) -> None:
        import torch
        if self.learn_refs is not None and self.k:
            self.encoder.embed_into(self.learn_refs, self.r_emb.data_ptr(), 1,
                                    torch.cuda.current_stream().cuda_stream)

    def queries(self, codes: np.ndarray, lens: np.ndarray) -> QueryBatch:
        return QueryBatch(self, codes, lens)

    def _sparse(self, qset, rset):
        """Exhaustive sparse hits of qset x rset as (local row int64, local ref int32, score)."""
        import torch

        from .device import Hits, gapblock_sparse_into
        if self._hits is None:
            self._hits = Hits()
        gapblock_sparse_into(qset, rset, self._hits, torch.cuda.current_stream().cuda_stream,
                             max_penalty=self.max_penalty, matrix=self.matrix,
                             gap_open=self.gap_open, gap_extend=self.gap_extend)
        ip, rr, sc = _hits_tensors(self._hits)
        return torch_rows(ip), rr, sc

    def search(self, qb: QueryBatch, phases: dict | None = None):
        """CSR (indptr int64 [nq+1], ref_ids int32, scores int32) torch tensors on the device.
        With ``phases`` (a dict), CUDA events bracketing embed / propose / rescore /
        exhaustive / merge are appended under those names."""
        import torch
        parts = []
        stream = torch.cuda.current_stream().cuda_stream

        def mark(name):
            if phases is not None:
                e = torch.cuda.Event(enable_timing=True)
                e.record()
                phases.setdefault(name, []).append(e)

        mark("start")
        if qb.learn_set is not None and self.n_learn and self.k:
            n = len(qb.learn_set)
            q_emb = torch.empty((n, 64), dtype=torch.bfloat16, device="cuda")
            self.encoder.embed_into(qb.learn_set, q_emb.data_ptr(), 1, stream)
            mark("embed")
            if self.proposal == "range":
                # proposals and their rescore run block by block (bounded memory)
                qi, ri, sc = self._range_hits(qb, q_emb)
                parts.append((qb.learn_rows_t[qi.long()], self.learn_ids[ri.long()], sc))
                mark("propose")
                mark("rescore")
            else:
                ids = torch.empty((n, self.k), dtype=torch.int32, device="cuda")
                propose_topk_into(q_emb.data_ptr(), n, self.r_emb.data_ptr(), self.n_learn,
                                  self.k, ids.data_ptr(), 0, stream,
                                  qb.ranges.data_ptr() if qb.ranges is not None else 0)
                qi = torch.arange(n, dtype=torch.int32, device="cuda").repeat_interleave(self.k)
                ri = ids.view(-1)
                keep = ri >= 0
                qi, ri = qi[keep], ri[keep]
                mark("propose")
                sc = torch.empty(qi.numel(), dtype=torch.int32, device="cuda")
                if qi.numel():
                    pair_scores(qb.learn_set, self.learn_refs, qi.data_ptr(), ri.data_ptr(),
                                qi.numel(), sc.data_ptr(), stream, matrix=self.matrix,
                                gap_open=self.gap_open, gap_extend=self.gap_extend)
                hit = sc <= self.max_penalty
                parts.append((qb.learn_rows_t[qi[hit].long()], self.learn_ids[ri[hit].long()],
                              sc[hit]))
                mark("rescore")
        if qb.learn_set is not None and self.fb_refs is not None:
            rows, rr, sc = self._sparse(qb.learn_set, self.fb_refs)
            parts.append((qb.learn_rows_t[rows], self.fb_ref_ids[rr.long()], sc))
        if qb.fb_set is not None and self.nr:
            rows, rr, sc = self._sparse(qb.fb_set, self.refs)
            parts.append((qb.fb_rows_t[rows], rr, sc))
        mark("exhaustive")
        if parts:
            qi = torch.cat([p[0] for p in parts])
            ri = torch.cat([p[1] for p in parts])
            sc = torch.cat([p[2] for p in parts])
        else:
            qi = torch.zeros(0, dtype=torch.int64, device="cuda")
            ri = torch.zeros(0, dtype=torch.int32, device="cuda")
            sc = torch.zeros(0, dtype=torch.int32, device="cuda")
        key, order = torch.sort(qi * max(self.nr, 1) + ri.long())
        counts = torch.bincount(qi, minlength=qb.count)
        indptr = torch.zeros(qb.count + 1, dtype=torch.int64, device="cuda")
        torch.cumsum(counts, 0, out=indptr[1:])
        out = indptr, ri[order], sc[order]
        mark("merge")
        return out

    def _range_hits(self, qb: QueryBatch, q_emb):
        """The threshold form's hits of the batch's learned rows: proposals, exact rescore and
        the threshold, as (local query, learned-ref index, score).  The queries go in blocks of
        whole 256-query tiles sized so that one block's candidates fit ``RANGE_BLOCK_PAIRS``
        (the candidate count per query of the previous search sizes the blocks; a block that
        overflows is split), so memory stays bounded whatever the thresholds let through."""
        import torch
        n = len(qb.learn_set)
        stream = torch.cuda.current_stream().cuda_stream
        tiles = qb.range_tiles(self)
        ntiles = -(-n // QUERY_TILE)
        per_q = max(self._range_per_query, 1.0)
        step = max(1, min(ntiles, int(RANGE_BLOCK_PAIRS / (per_q * QUERY_TILE))))
        out_q, out_r, out_s = [], [], []
        seen, t0 = 0, 0
        while t0 < ntiles:
            t1 = min(ntiles, t0 + step)
            q0, q1 = t0 * QUERY_TILE, min(n, t1 * QUERY_TILE)
            pq = torch.empty(RANGE_BLOCK_PAIRS, dtype=torch.int32, device="cuda")
            pr = torch.empty(RANGE_BLOCK_PAIRS, dtype=torch.int32, device="cuda")
            cnt = propose_range_into(q_emb[q0:q1].data_ptr(), q1 - q0,
                                     qb.learn_lens_t[q0:q1].data_ptr(), self.r_emb.data_ptr(),
                                     self.n_learn, self.learn_lens_t.data_ptr(), self.thresholds,
                                     pq.data_ptr(), pr.data_ptr(), RANGE_BLOCK_PAIRS, stream,
                                     tiles[2 * t0:2 * t1].data_ptr())
            if cnt > RANGE_BLOCK_PAIRS and t1 - t0 > 1:
                step = max(1, (t1 - t0) // 2)  # too many candidates: smaller blocks
                continue
            if cnt > RANGE_BLOCK_PAIRS:  # one tile alone: the exact size
                pq = torch.empty(cnt, dtype=torch.int32, device="cuda")
                pr = torch.empty(cnt, dtype=torch.int32, device="cuda")
                cnt = propose_range_into(q_emb[q0:q1].data_ptr(), q1 - q0,
                                         qb.learn_lens_t[q0:q1].data_ptr(), self.r_emb.data_ptr(),
                                         self.n_learn, self.learn_lens_t.data_ptr(),
                                         self.thresholds, pq.data_ptr(), pr.data_ptr(), cnt,
                                         stream, tiles[2 * t0:2 * t1].data_ptr())
            seen += cnt
            if cnt:
                pq, pr = pq[:cnt], pr[:cnt]
                pq += q0
                sc = torch.empty(cnt, dtype=torch.int32, device="cuda")
                pair_scores(qb.learn_set, self.learn_refs, pq.data_ptr(), pr.data_ptr(), cnt,
                            sc.data_ptr(), stream, matrix=self.matrix, gap_open=self.gap_open,
                            gap_extend=self.gap_extend)
                hit = sc <= self.max_penalty
                out_q.append(pq[hit])
                out_r.append(pr[hit])
                out_s.append(sc[hit])
            del pq, pr
            t0 = t1
        self._range_per_query = seen / max(n, 1)
        if not out_q:
            z = torch.zeros(0, dtype=torch.int32, device="cuda")
            return z, z, z
        return torch.cat(out_q), torch.cat(out_r), torch.cat(out_s)

    def search_strings(self, queries) -> "SparseScores":
        """The public call: thresholded hits of host query strings against the index's refs, as
        host CSR (``gapblock.SparseScores``, the format of ``score_sparse``).  The strings are
        packed once by the library and uploaded as they are (the device encodes them); the rows
        come back into pinned blocks of the library's cache."""
        import torch

        from .gapblock import SparseScores
        packed = _lib.pack(list(queries))
        lens = np.diff(packed.offsets).astype(np.int32)
        if lens.size and (lens.min() < 1 or lens.max() > PAD):
            raise ValueError("encoder inputs must have 1..32 residues")
        bad = _CODE[packed.data[:int(packed.offsets[-1])]] == 255
        if bad.any():  # the first invalid symbol over all queries, as pad_codes reports it
            raise ValueError(f"symbol '{chr(int(packed.data[np.argmax(bad)]))}' is not in the "
                             "alphabet")
        ip, ri, sc = self.search(QueryBatch(self, None, lens, packed))
        host = []
        for t in (ip, ri, sc):
            h = _lib.pinned_array(t.numel(), np.int64 if t.dtype == torch.int64 else np.int32)
            if t.numel():
                torch.from_numpy(h).copy_(t)
            host.append(h)
        return SparseScores(*host, (len(lens), self.nr), self.max_penalty)

    def exhaustive(self, qb: QueryBatch, codes: np.ndarray):
        """The exhaustive sparse kernel's CSR for the same queries (the exact answer)."""
        from .device import SeqSet
        qset = SeqSet(codes_to_packed(codes, qb.lens), "aa")
        from .device import Hits, gapblock_sparse_into
        import torch
        hits = Hits()
        gapblock_sparse_into(qset, self.refs, hits, torch.cuda.current_stream().cuda_stream,
                             max_penalty=self.max_penalty, matrix=self.matrix,
                             gap_open=self.gap_open, gap_extend=self.gap_extend)
        return _hits_tensors(hits)

    def recall(self, codes: np.ndarray, lens: np.ndarray) -> dict:
        """Found / exact hit counts against the exhaustive kernel, overall and per (query length,
        ref length) cell; also checks that every reported hit is an exact hit, score included."""
        import torch
        qb = self.queries(codes, lens)
        ip, ri, sc = self.search(qb)
        eip, eri, esc = self.exhaustive(qb, codes)
        nr = max(self.nr, 1)
        rows, erows = torch_rows(ip), torch_rows(eip)
        got, want = rows * nr + ri.long(), erows * nr + eri.long()
        if got.numel() == 0:
            ok = True
        elif want.numel() == 0:
            ok = False
        else:
            pos = torch.searchsorted(want, got).clamp(max=want.numel() - 1)
            ok = bool(torch.equal(want[pos], got)) and bool(torch.equal(esc[pos], sc))
        ql = torch.from_numpy(qb.lens.astype(np.int64)).cuda()
        rl = torch.from_numpy(self.ref_lens.astype(np.int64)).cuda()
        cells = lambda r, c: torch.bincount(ql[r] * (PAD + 1) + rl[c.long()],  # noqa: E731
                                            minlength=(PAD + 1) ** 2).view(PAD + 1, PAD + 1)
        found = cells(rows, ri).cpu().numpy()
        exact = cells(erows, eri).cpu().numpy()
        tf, te = int(found.sum()), int(exact.sum())
        return {"found": tf, "exact": te, "recall": tf / te if te else 1.0, "found_cells": found,
                "exact_cells": exact, "subset_of_exact": ok}

    def calibrate(self, codes: np.ndarray, lens: np.ndarray, bound: float = 0.99,
                  margin: float | None = None) -> dict:
        """Chooses the fallback lengths on a held-out calibration batch.

        Without fallback, the proposals' found / exact hit counts are measured per (query
        length, ref length) cell.  A cell is covered (answered exactly) once its query length or
        its ref length falls back.  Lengths are added greedily -- each time the query or ref
        length with the most recovered hits per exhaustively scored pair (pairs estimated from
        the calibration batch's query lengths and the refs' lengths) -- until the estimated
        recall reaches ``bound + margin``.  The recall with the chosen fallback is then measured
        on the same batch.  ``margin`` defaults to min(0.003, (1 - bound) / 3)."""
        if self.proposal == "range" and self.k:
            return self.calibrate_range(codes, lens, bound, margin)
        if margin is None:
            margin = min(0.003, (1.0 - bound) / 3.0)
        self.set_fallback()
        r0 = self.recall(codes, lens)
        f, e = r0["found_cells"].astype(np.float64), r0["exact_cells"].astype(np.float64)
        wq = np.bincount(np.asarray(lens, np.int64), minlength=PAD + 1)[:PAD + 1] / max(len(lens), 1)
        wr = np.bincount(self.ref_lens.astype(np.int64), minlength=PAD + 1)[:PAD + 1] / max(self.nr, 1)
        covered = np.zeros((PAD + 1, PAD + 1), bool)
        q_fb, ref_fb = [], []
        total = e.sum()
        while total:
            rec = (e[covered].sum() + f[~covered].sum()) / total
            if rec >= bound + margin:
                break
            best, pick = 0.0, None
            for a in range(PAD + 1):
                if a in q_fb or not wq[a]:
                    continue
                open_ = ~covered[a]
                gain, cost = (e[a] - f[a])[open_].sum(), wq[a] * wr[open_].sum()
                if gain > 0 and cost > 0 and gain / cost > best:
                    best, pick = gain / cost, ("q", a)
            for b in range(PAD + 1):
                if b in ref_fb or not wr[b]:
                    continue
                open_ = ~covered[:, b]
                gain, cost = (e[:, b] - f[:, b])[open_].sum(), wr[b] * wq[open_].sum()
                if gain > 0 and cost > 0 and gain / cost > best:
                    best, pick = gain / cost, ("r", b)
            if pick is None:
                break
            if pick[0] == "q":
                q_fb.append(pick[1])
                covered[pick[1], :] = True
            else:
                ref_fb.append(pick[1])
                covered[:, pick[1]] = True
        q_fb, ref_fb = sorted(q_fb), sorted(ref_fb)
        self.set_fallback(q_fb, ref_fb)
        r2 = self.recall(codes, lens)
        share = float(wq[q_fb].sum() + (1.0 - wq[q_fb].sum()) * wr[ref_fb].sum())
        return {"ref_fallback": ref_fb, "query_fallback": q_fb, "recall_no_fallback": r0["recall"],
                "recall": r2["recall"], "found": r2["found"], "exact": r2["exact"],
                "subset_of_exact": r2["subset_of_exact"], "exhaustive_share": share,
                "cells_no_fallback": (r0["found_cells"], r0["exact_cells"])}

    def calibrate_range(self, codes: np.ndarray, lens: np.ndarray, bound: float = 0.99,
                        margin: float | None = None, slack: float = 0.02,
                        costs: dict | None = None, levels=RANGE_LEVELS,
                        chunk_queries: int = 1024) -> dict:
        """The threshold form's calibration on a held-out batch: a per-cell recall budget.

        1. The batch's exact hits against every ref come from the exhaustive sparse kernel and
           their embedding dot products from ``st_embed_dots``.  For each (query length, ref
           length) cell and each recall level q of ``levels``, the candidate threshold is the dot
           product that keeps a fraction q of the cell's hits (the floor((1 - q) n)-th smallest),
           lowered by ``slack``.
        2. The proposals at every cell's most inclusive threshold are made on the batch in
           chunks of ``chunk_queries`` queries (bounded memory) and counted per cell and level.
        3. A greedy allocation then minimises the estimated time (``costs``: seconds per
           exhaustively scored pair -- measured on the batch when it is large enough -- per
           scanned pair and per candidate; defaults ``RANGE_COSTS``) until the recall estimate
           reaches ``bound + margin``: every step takes the move with the most recovered hits
           per added second, a move being either raising one cell to its next level (a cell
           may also stay off: its hits count as lost) or scoring one query or ref length
           exhaustively (the fallback).
        The recall with the chosen thresholds and fallback is then measured on the same batch."""
        import torch
        if margin is None:
            margin = min(0.003, (1.0 - bound) / 3.0)
        c = dict(RANGE_COSTS, **(costs or {}))
        target = bound + margin
        S, LV = PAD + 1, len(levels)
        self.set_fallback()
        self.set_thresholds(np.full((S, S), np.inf, np.float32))
        qb = self.queries(codes, lens)
        stream = torch.cuda.current_stream().cuda_stream
        n = len(qb.learn_set) if qb.learn_set is not None else 0
        ql_sorted = np.clip(qb.lens[qb.learn_rows], 0, PAD)
        wq = np.bincount(ql_sorted, minlength=S)[:S].astype(np.float64)
        wr = np.bincount(np.clip(self.ref_lens, 0, PAD), minlength=S)[:S].astype(np.float64)
        E = np.zeros((S, S))
        tau = np.full((S, S, LV), np.inf, np.float32)   # threshold per cell and level
        FL = np.zeros((S, S, LV))                       # hits found per cell and level
        CL = np.zeros((S, S, LV))                       # candidates per cell and level
        measured = {}
        if n and self.n_learn:
            q_emb = torch.empty((n, 64), dtype=torch.bfloat16, device="cuda")
            self.encoder.embed_into(qb.learn_set, q_emb.data_ptr(), 1, stream)
            rows, rr, _ = self._sparse(qb.learn_set, self.learn_refs)
            if n * self.n_learn >= 1e9:  # a second, warm call (the first one tunes the kernel)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                rows, rr, _ = self._sparse(qb.learn_set, self.learn_refs)
                e1.record()
                e1.synchronize()
                measured["exhaustive"] = e0.elapsed_time(e1) / 1e3 / (n * self.n_learn)
            dots = torch.empty(rows.numel(), dtype=torch.float32, device="cuda")
            rows32 = rows.to(torch.int32)
            embed_dots_into(q_emb.data_ptr(), n, self.r_emb.data_ptr(), self.n_learn,
                            rows32.data_ptr(), rr.data_ptr(), rows.numel(), dots.data_ptr(), stream)
            cell = ql_sorted[rows.cpu().numpy()].astype(np.int64) * S + \
                np.clip(self.learn_lens[rr.cpu().numpy()], 0, PAD)
            d = dots.cpu().numpy()
            E = np.bincount(cell, minlength=S * S).reshape(S, S).astype(np.float64)
            order = np.lexsort((d, cell))
            cs, ds = cell[order], d[order]
            start = np.searchsorted(cs, np.arange(S * S))
            cnt = E.ravel().astype(np.int64)
            tf, ff = tau.reshape(S * S, LV), FL.reshape(S * S, LV)
            for ce in np.flatnonzero(cnt):
                seg = ds[start[ce]:start[ce] + cnt[ce]]
                for li, q in enumerate(levels):
                    t = seg[min(int(np.floor((1.0 - q) * cnt[ce])), cnt[ce] - 1)] - slack
                    tf[ce, li] = t
                    ff[ce, li] = cnt[ce] - np.searchsorted(seg, t, side="left")
            # candidates per cell and level, from the most inclusive thresholds, in chunks
            self.set_thresholds(tau[:, :, LV - 1])
            ql_t = torch.from_numpy(ql_sorted.astype(np.int64)).cuda()
            rl_t = self.learn_lens_t.long()
            tau_t = torch.from_numpy(tau.reshape(S * S, LV)).cuda()
            cl_t = torch.zeros((LV, S * S), dtype=torch.float64, device="cuda")
            thr_last = self.thresholds
            for c0 in range(0, n, chunk_queries):
                c1 = min(n, c0 + chunk_queries)
                qe = q_emb[c0:c1]
                rg = range_tile_ranges(ql_sorted[c0:c1], self.learn_lens, thr_last)
                pq, pr = propose_range(qe, qb.learn_lens_t[c0:c1], self.r_emb, self.learn_lens_t,
                                       thr_last, None, torch.from_numpy(rg.ravel()).cuda())
                if pq.numel() == 0:
                    continue
                dd = torch.empty(pq.numel(), dtype=torch.float32, device="cuda")
                embed_dots_into(qe.data_ptr(), c1 - c0, self.r_emb.data_ptr(), self.n_learn,
                                pq.data_ptr(), pr.data_ptr(), pq.numel(), dd.data_ptr(), stream)
                ce_t = ql_t[c0 + pq.long()] * S + rl_t[pr.long()]
                for li in range(LV):
                    ge = (dd >= tau_t[:, li][ce_t]).to(torch.float64)
                    cl_t[li].index_add_(0, ce_t, ge)
                    del ge
                del pq, pr, dd, ce_t
            CL = cl_t.T.reshape(S, S, LV).cpu().numpy()
        c.update(measured)
        level, q_fb, r_fb, est_rec, est = allocate_recall(E, FL, CL, wq, wr, c, target)
        covered = np.zeros((S, S), bool)
        covered[q_fb, :] = True
        covered[:, r_fb] = True
        idx = np.clip(level, 0, LV - 1)
        thr = np.where((level >= 0) & ~covered,
                       np.take_along_axis(tau, idx[:, :, None], 2)[:, :, 0], np.inf)
        q_fb, r_fb = sorted(q_fb), sorted(r_fb)
        self.set_fallback(q_fb, r_fb)
        self.set_thresholds(thr.astype(np.float32))
        cand = np.take_along_axis(CL, idx[:, :, None], 2)[:, :, 0]
        cand_q = float(np.where((level >= 0) & ~covered, cand, 0.0).sum() / max(n, 1))
        self._range_per_query = 1.25 * cand_q * n / max(1, n - wq[q_fb].sum())
        te = E.sum()
        r2 = self.recall(codes, lens)
        wq1, wr1 = wq / max(wq.sum(), 1.0), wr / max(wr.sum(), 1.0)
        share = float(wq1[q_fb].sum() + (1.0 - wq1[q_fb].sum()) * wr1[r_fb].sum())
        return {"ref_fallback": r_fb, "query_fallback": q_fb,
                # share of the batch's exact hits that the chosen proposals find (the rest of
                # the recall comes from the exhaustively scored lengths)
                "recall_from_proposals": float(np.take_along_axis(
                    FL, idx[:, :, None], 2)[:, :, 0][(level >= 0) & ~covered].sum() / te)
                if te else 0.0,
                "recall_estimate": float(est_rec),
                "recall": r2["recall"], "found": r2["found"], "exact": r2["exact"],
                "subset_of_exact": r2["subset_of_exact"], "exhaustive_share": share,
                "cells_with_proposals": int(((level >= 0) & ~covered).sum()),
                "candidates_per_query": cand_q,
                "estimated_seconds_per_query": est / max(n, 1),
                "costs": {k: float(v) for k, v in c.items()}, "costs_measured": sorted(measured),
                "cells_no_fallback": (FL[:, :, LV - 1], E), "candidate_cells": CL[:, :, LV - 1],
                "levels": level}
