"""Learned candidate proposal for thresholded gap-block search at scales where the exhaustive
kernel's 10^12 pairs are the cost (1e6 x 1e6 CDR3-like junctions).

A small encoder (:class:`Encoder`; 2 conv + 2 attention layers, width 128, 64-d unit-length
output) is trained on pairs scored by the exact gap-block kernel so that squared embedding
distance tracks the score.  Its embeddings feed a BF16 tensor-core product that proposes the
top-k refs of every query.  Every proposal is rescored by the exact kernel, so reported scores are
always exact.  Recall against exhaustive search is measured on a held-out calibration slice, and
query lengths whose recall falls below the bound are routed to the exhaustive kernel.

Everything runs through ``libseqtree_b200.so``: the training kernels (forward, backward, Adam),
the embedding, the proposal kernel and the exact scorer.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .matrix import SubstitutionMatrix

AA24 = "ARNDCQEGHILKMFPSTWYVBZX*"
AA20 = "ACDEFGHIKLMNPQRSTVWY"
PAD = 32
_CODE = np.full(256, 255, np.uint8)
for _i, _c in enumerate(AA24):
    _CODE[ord(_c)] = _i
    _CODE[ord(_c.lower())] = _i


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

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        p = init_params(seed) if params is None else np.ascontiguousarray(params, np.float32)
        if p.size != param_count():
            raise ValueError(f"expected {param_count()} parameters, got {p.size}")
        self._h = ctypes.c_void_p()
        err = _lib.st_error()
        _lib.check(_lib.lib.st_encoder_create(p.ctypes.data, ctypes.byref(self._h),
                                              ctypes.byref(err)), err)

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
        """Embeddings of a device set: layout 0 fp32 [n][64], 1 bf16 swizzled [n][64]."""
        err = _lib.st_error()
        _lib.check(_lib.lib.st_encoder_embed(self._h, seqset.handle, ctypes.c_void_p(out_ptr),
                                             int(layout), ctypes.c_void_p(stream),
                                             ctypes.byref(err)), err)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib.st_encoder_destroy(h)
            self._h = ctypes.c_void_p()


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
                      scores_ptr: int = 0, stream: int = 0) -> None:
    """``st_propose_topk`` on device pointers (swizzled bf16 embeddings in, [nq][k] out)."""
    err = _lib.st_error()
    _lib.check(_lib.lib.st_propose_topk(ctypes.c_void_p(q_ptr), int(nq), ctypes.c_void_p(r_ptr),
                                        int(nr), int(k), ctypes.c_void_p(ids_ptr),
                                        ctypes.c_void_p(scores_ptr or None),
                                        ctypes.c_void_p(stream), ctypes.byref(err)), err)


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


def stream_status(stream: int = 0) -> None:
    """Synchronise ``stream`` and raise if a bounded device-side wait gave up since the last
    check."""
    err = _lib.st_error()
    _lib.check(_lib.lib.st_stream_status(ctypes.c_void_p(stream), ctypes.byref(err)), err)


# ----------------------------------------------------------------------------- data ---------
def cdr3_like(seed: int, n: int) -> list[str]:
    """'CASS' + uniform middle + 'F', length 8-25 with mode 14 (a Gaussian around 14 with sigma
    2.5 below and 3.5 above)."""
    rng = np.random.default_rng(seed)
    L = np.arange(8, 26)
    sig = np.where(L < 14, 2.5, 3.5)
    p = np.exp(-0.5 * ((L - 14) / sig) ** 2)
    lens = rng.choice(L, size=n, p=p / p.sum())
    mids = rng.integers(0, 20, size=int((lens - 5).sum()), dtype=np.uint8)
    letters = np.frombuffer(AA20.encode(), np.uint8)[mids].tobytes().decode()
    out, o = [], 0
    for length in lens:
        k = int(length) - 5
        out.append("CASS" + letters[o:o + k] + "F")
        o += k
    return out


def mutate(seqs, rng) -> list[str]:
    """Near neighbours: 1-3 random substitutions and one random indel block (a deletion or an
    insertion of 1-3 residues at a random position), kept within 1..32 residues."""
    out = []
    nsub = rng.integers(1, 4, size=len(seqs))
    for s, k in zip(seqs, nsub):
        b = bytearray(s.encode())
        for _ in range(int(k)):
            b[int(rng.integers(0, len(b)))] = ord(AA20[int(rng.integers(0, 20))])
        blk = int(rng.integers(1, 4))
        pos = int(rng.integers(0, len(b) + 1))
        if rng.random() < 0.5 and len(b) - blk >= 1:
            del b[pos:pos + blk]
        elif len(b) + blk <= PAD:
            b[pos:pos] = bytes(ord(AA20[int(x)]) for x in rng.integers(0, 20, size=blk))
        out.append(b.decode())
    return out


def training_pairs(seed: int, n_pairs: int, pool: list[str] | None = None):
    """n_pairs (a, b) string pairs: half near neighbours made by :func:`mutate`, half random
    pairs drawn from the pool (default: fresh CDR3-like strings)."""
    rng = np.random.default_rng(seed)
    if pool is None:
        pool = cdr3_like(seed + 7, max(2 * n_pairs, 1000))
    near = n_pairs // 2
    idx = rng.integers(0, len(pool), size=(n_pairs, 2))
    a = [pool[i] for i in idx[:, 0]]
    b = [pool[i] for i in idx[:, 1]]
    b[:near] = mutate(a[:near], rng)
    return a, b
