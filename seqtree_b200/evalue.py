"""Control-calibrated per-query score cutoffs on the GPU: ``thetas_from_scores`` of seqtree's
``python/seqtree/evalue.py:102-143``.

For a query with control hit scores ``s`` (found at ``theta_max``), the cutoff achieving a target
E-value ``e_target`` (``E = (N / M) * n_control``) is the largest ``t`` in ``[0, theta_max]``
whose control count ``#{s <= t}`` stays within ``k = floor(e_target * M / N)``; ``-1`` when none
exists, when ``k < 1``, or when ``t`` admits no control hit although ``e_target`` is below the
rule-of-three bound ``3N/M``.  The rows are CSR score lists -- host lists, a
:class:`seqtree_b200.gapblock.SparseScores`, or the device rows of a ``device.Hits`` (no copy) --
and every row is one warp of ``st_thetas_csr``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _run(indptr_ptr: int, scores_ptr: int, rows: int, n_target, m_control, e_target,
         theta_max, exclude_exact, out_ptr: int, stream: int) -> None:
    err = _lib.st_error()
    _lib.check(_lib.lib.st_thetas_csr(ctypes.c_void_p(indptr_ptr), ctypes.c_void_p(scores_ptr),
                                      int(rows), int(n_target), int(m_control), float(e_target),
                                      int(theta_max), int(bool(exclude_exact)),
                                      ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream),
                                      ctypes.byref(err)), err)


def _check(n_target, m_control, e_target, theta_max) -> None:
    # the reference's checks, in its order (evalue.py:132-137)
    if n_target <= 0 or m_control <= 0:
        raise ValueError("n_target and m_control must be > 0")
    if e_target <= 0.0:
        raise ValueError("e_target must be > 0")
    if theta_max < 0:
        raise ValueError("theta_max must be >= 0")


def _csr_thetas(indptr: np.ndarray, scores: np.ndarray, n_target, m_control, e_target, theta_max,
                exclude_exact) -> list[int]:
    import torch
    rows = len(indptr) - 1
    if rows <= 0:
        return []
    ip = torch.from_numpy(np.ascontiguousarray(indptr, np.int64)).cuda()
    sc = torch.from_numpy(np.ascontiguousarray(scores, np.int32)).cuda() if len(scores) else \
        torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.empty(rows, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _run(ip.data_ptr(), sc.data_ptr(), rows, n_target, m_control, e_target, theta_max,
         exclude_exact, out.data_ptr(), stream)
    return [int(x) for x in out.cpu().numpy()]


def thetas_from_scores(control_scores, n_target: int, m_control: int, e_target: float,
                       theta_max: int, *, exclude_exact: bool = False) -> list[int]:
    """One cutoff per query (``-1`` where none achieves ``e_target``), as the reference.

    ``control_scores`` is a sequence of per-query score lists (hits above ``theta_max`` may be
    omitted), or a :class:`seqtree_b200.gapblock.SparseScores` (its rows)."""
    _check(n_target, m_control, e_target, theta_max)
    if hasattr(control_scores, "indptr") and hasattr(control_scores, "scores"):
        return _csr_thetas(control_scores.indptr, control_scores.scores, n_target, m_control,
                           e_target, theta_max, exclude_exact)
    lists = [np.asarray(list(s), dtype=np.int64) for s in control_scores]
    if any(len(s) and (s.min() < -2**31 or s.max() >= 2**31) for s in lists):
        raise OverflowError("scores must fit int32")
    lens = np.fromiter((len(s) for s in lists), np.int64, len(lists))
    indptr = np.zeros(len(lists) + 1, np.int64)
    np.cumsum(lens, out=indptr[1:])
    flat = np.concatenate(lists).astype(np.int32) if len(lists) and indptr[-1] else np.zeros(0, np.int32)
    return _csr_thetas(indptr, flat, n_target, m_control, e_target, theta_max, exclude_exact)


def thetas_from_hits(hits, n_target: int, m_control: int, e_target: float, theta_max: int, *,
                     exclude_exact: bool = False, stream: int = 0):
    """Cutoffs for the rows of a device-resident ``device.Hits`` (as filled by
    ``device.gapblock_sparse_into``), without leaving the GPU: an int32 torch tensor [rows]."""
    import torch
    _check(n_target, m_control, e_target, theta_max)
    info = hits.info()
    out = torch.empty(info["rows"], dtype=torch.int32, device="cuda")
    if info["rows"]:
        _run(info["indptr"], info["scores"] or info["indptr"], info["rows"], n_target, m_control,
             e_target, theta_max, exclude_exact, out.data_ptr(),
             stream or torch.cuda.current_stream().cuda_stream)
    return out
