"""CPU checkers for the all-vs-all scoring path -- TEST INFRASTRUCTURE ONLY.

Two checkers live here, both loaded with ctypes:

* ``port``: ``oracle/oracle.c``, a plain-C restatement of the reference arithmetic
  (seqtree 0.6.0 ``src/gapblock.cpp:39-62``, ``src/pairwise.cpp:76-125``,
  ``src/distance.cpp:68-95``), built into ``oracle/liboracle.so``.
* ``ref``: the reference's own hot-path C++ sources compiled here by ``oracle/Makefile`` into
  ``oracle/_ref/libseqtree_ref.so`` (present wherever the build ran; the file travels with
  the repository snapshot).

Plus a pure-Python restatement of the reference's ``central_prior`` and ``_prior_cube``
(``python/seqtree/gapblock.py:79-94, 492-509``), so that a process timing the reference needs
nothing from ``seqtree_b200`` to build its prior cube.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import this
package, and only as the checker or the timed CPU baseline -- never on the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libseqtree_ref.so"

ALPHABETS = {"aa": 0, "nt": 1, "iupac": 2}
MATRIX_IDS = {"blosum62": 0, "blosum45": 1, "blosum80": 2, "pam250": 3, "pam100": 4,
              "structural": 5, "unit": 6, "custom": 7}

_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build(reference_tree: str | None = None) -> None:
    """Compile both checkers; the reference one only when its source tree is given (argument or
    the SEQTREE_REFERENCE environment variable) and present."""
    tree = reference_tree or os.environ.get("SEQTREE_REFERENCE")
    cmd = ["make", "-s", "-C", str(HERE)] + ([f"REF={tree}"] if tree else [])
    subprocess.run(cmd, check=True)


class Prepacked(list):
    """A list of strings that keeps its packed form, so a timed call does not re-pack it (a C++
    caller of the reference passes the same ``std::vector<std::string>`` to every call)."""

    def __init__(self, strings):
        super().__init__(strings)
        self.packed = pack(list(strings))


def pack(strings) -> tuple[np.ndarray, np.ndarray]:
    """list[str] -> (uint8 bytes, int64 offsets of len+1)."""
    if isinstance(strings, Prepacked):
        return strings.packed
    bs = [s.encode("latin-1") if isinstance(s, str) else bytes(s) for s in strings]
    lens = np.fromiter((len(b) for b in bs), dtype=np.int64, count=len(bs))
    off = np.zeros(len(bs) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = np.frombuffer(b"".join(bs), dtype=np.uint8) if bs else np.zeros(0, np.uint8)
    if data.size == 0:
        data = np.zeros(1, np.uint8)
    return np.ascontiguousarray(data), off


def _p(a, t):
    return a.ctypes.data_as(t)


class OracleError(Exception):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


# ----------------------------------------------------------------------------- port ---------
_port = None


def port():
    global _port
    if _port is None:
        if not PORT_SO.exists():
            build()
        lib = ctypes.CDLL(str(PORT_SO))
        lib.or_alphabet_size.restype = ctypes.c_int
        lib.or_encode.restype = ctypes.c_int64
        lib.or_encode.argtypes = [ctypes.c_int, _u8p, ctypes.c_int64, _u8p]
        lib.or_penalty_from_similarity.argtypes = [ctypes.c_int, _i32p, _i32p]
        lib.or_gapblock_matrix.argtypes = [_u8p, _i64p, ctypes.c_int64, _u8p, _i64p,
                                           ctypes.c_int64, _i32p, ctypes.c_int, ctypes.c_int32,
                                           ctypes.c_int32, _i32p, ctypes.c_uint32, _i32p,
                                           ctypes.c_int]
        lib.or_align_matrix.argtypes = [_u8p, _i64p, ctypes.c_int64, _u8p, _i64p, ctypes.c_int64,
                                        _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_int, _i32p, ctypes.c_int]
        for f in (lib.or_hamming_matrix, lib.or_levenshtein_matrix):
            f.argtypes = [_u8p, _i64p, ctypes.c_int64, _u8p, _i64p, ctypes.c_int64, _i32p,
                          ctypes.c_int]
        _port = lib
    return _port


def encode(strings, alphabet: str = "aa"):
    """Encode with the reference codec; raises ValueError naming the first bad symbol."""
    data, off = pack(strings)
    codes = np.zeros_like(data)
    n = int(off[-1])
    bad = port().or_encode(ALPHABETS[alphabet], _p(data, _u8p), n, _p(codes, _u8p))
    if bad >= 0:
        raise ValueError(f"symbol '{chr(data[bad])}' is not in the alphabet")
    return codes, off


def penalty_from_similarity(sim: np.ndarray | None, size: int) -> np.ndarray:
    pen = np.zeros(size * size, np.int32)
    s = None if sim is None else np.ascontiguousarray(sim, np.int32).ravel()
    port().or_penalty_from_similarity(size, None if s is None else _p(s, _i32p), _p(pen, _i32p))
    return pen.reshape(size, size)


def gapblock_matrix(queries, refs, pen, alphabet="aa", gap_open=1, gap_extend=1, prior=None,
                    prior_width=0, threads=os.cpu_count() or 1) -> np.ndarray:
    """Port of gapblock_matrix; `pen` is an A*A penalty grid."""
    qc, qo = encode(queries, alphabet)
    rc, ro = encode(refs, alphabet)
    N, K = len(queries), len(refs)
    out = np.zeros((N, K), np.int32)
    pen = np.ascontiguousarray(pen, np.int32).ravel()
    A = int(round(pen.size ** 0.5))
    pr = None if prior is None or len(prior) == 0 else np.ascontiguousarray(prior, np.int32)
    port().or_gapblock_matrix(_p(qc, _u8p), _p(qo, _i64p), N, _p(rc, _u8p), _p(ro, _i64p), K,
                              _p(pen, _i32p), A, gap_open, gap_extend,
                              None if pr is None else _p(pr, _i32p), prior_width,
                              _p(out, _i32p), threads)
    return out


def align_matrix(queries, refs, sim, alphabet="aa", mode="global", gap_open=11, gap_extend=1,
                 dist=False, threads=os.cpu_count() or 1) -> np.ndarray:
    """Port of align_score_matrix / align_dist_matrix; `sim` is an A*A similarity grid."""
    qc, qo = encode(queries, alphabet)
    rc, ro = encode(refs, alphabet)
    N, K = len(queries), len(refs)
    out = np.zeros((N, K), np.int32)
    sim = np.ascontiguousarray(sim, np.int32).ravel()
    A = int(round(sim.size ** 0.5))
    st = port().or_align_matrix(_p(qc, _u8p), _p(qo, _i64p), N, _p(rc, _u8p), _p(ro, _i64p), K,
                                _p(sim, _i32p), A, int(mode == "local"), gap_open, gap_extend,
                                int(dist), _p(out, _i32p), threads)
    if st == 2:
        raise OverflowError("the alignment %s does not fit in 32 bits" %
                            ("distance" if dist else "score"))
    return out


def hamming_matrix(a, b, threads=os.cpu_count() or 1) -> np.ndarray:
    ad, ao = pack(a)
    bd, bo = pack(b)
    la, lb = np.diff(ao), np.diff(bo)
    if len(a) and len(b) and (np.any(la != la[0]) or np.any(lb != la[0])):
        raise ValueError("hamming distance is only defined for equal-length sequences")
    out = np.zeros((len(a), len(b)), np.int32)
    port().or_hamming_matrix(_p(ad, _u8p), _p(ao, _i64p), len(a), _p(bd, _u8p), _p(bo, _i64p),
                             len(b), _p(out, _i32p), threads)
    return out


def levenshtein_matrix(a, b, threads=os.cpu_count() or 1) -> np.ndarray:
    ad, ao = pack(a)
    bd, bo = pack(b)
    out = np.zeros((len(a), len(b)), np.int32)
    port().or_levenshtein_matrix(_p(ad, _u8p), _p(ao, _i64p), len(a), _p(bd, _u8p),
                                 _p(bo, _i64p), len(b), _p(out, _i32p), threads)
    return out


# ----------------------------------------------------------------------------- ref ----------
_ref = None


def ref_available() -> bool:
    return REF_SO.exists()


def ref():
    """The reference's own C++ (oracle/_ref). Raises FileNotFoundError when it was not built."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(str(REF_SO))
        lib = ctypes.CDLL(str(REF_SO))
        lib.ref_matrix_tables.argtypes = [ctypes.c_int, _i32p, ctypes.c_int, _i32p, _i32p,
                                          ctypes.POINTER(ctypes.c_int), _i32p]
        lib.ref_gapblock_matrix.argtypes = [
            ctypes.c_char_p, _i64p, ctypes.c_int64, ctypes.c_char_p, _i64p, ctypes.c_int64,
            ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
            _i32p, ctypes.c_int64, ctypes.c_uint32, ctypes.c_int, _i32p, ctypes.c_char_p,
            ctypes.c_int]
        lib.ref_align_matrix.argtypes = [
            ctypes.c_char_p, _i64p, ctypes.c_int64, ctypes.c_char_p, _i64p, ctypes.c_int64,
            ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int32,
            ctypes.c_int32, ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_char_p, ctypes.c_int]
        lib.ref_align_score.argtypes = [
            ctypes.c_char_p, ctypes.c_int64, ctypes.c_char_p, ctypes.c_int64, ctypes.c_int,
            ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
            _i32p, ctypes.c_char_p, ctypes.c_int]
        lib.ref_align_pair.argtypes = [
            ctypes.c_char_p, ctypes.c_int64, ctypes.c_char_p, ctypes.c_int64, ctypes.c_int,
            ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
            _i32p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int64,
            ctypes.c_char_p, ctypes.c_int]
        lib.ref_index_align.argtypes = [
            ctypes.c_char_p, _i64p, ctypes.c_int64, ctypes.c_int, ctypes.c_int64,
            ctypes.c_char_p, ctypes.c_int64, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int32,
            ctypes.c_int32, _i32p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
            ctypes.c_int64, ctypes.c_char_p, ctypes.c_int]
        lib.ref_distance_matrix.argtypes = [
            ctypes.c_char_p, _i64p, ctypes.c_int64, ctypes.c_char_p, _i64p, ctypes.c_int64,
            ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_char_p, ctypes.c_int]
        _ref = lib
    return _ref


def _raise(code: int, err) -> None:
    msg = err.value.decode(errors="replace")
    if code == 1:
        raise ValueError(msg)
    if code == 2:
        raise OverflowError(msg)
    raise RuntimeError(msg)


def _matrix_args(matrix, size=0):
    """matrix: a name from MATRIX_IDS, ('unit', size), ('custom', sim grid) or None."""
    if matrix is None:
        return -1, None, 0, None
    if isinstance(matrix, str):
        return MATRIX_IDS[matrix.lower()], None, size, None
    kind, payload = matrix
    if kind == "unit":
        return MATRIX_IDS["unit"], None, int(payload), None
    sim = np.ascontiguousarray(payload, np.int32)
    return MATRIX_IDS["custom"], _p(sim, _i32p), sim.shape[0], sim


def ref_tables(matrix) -> tuple[np.ndarray, np.ndarray, int]:
    """(similarity, penalty, scale) of a reference matrix."""
    mid, simp, size, _keep = _matrix_args(matrix)
    sim = np.zeros(32 * 32, np.int32)
    pen = np.zeros(32 * 32, np.int32)
    A = ctypes.c_int(0)
    scale = ctypes.c_int32(0)
    st = ref().ref_matrix_tables(mid, simp, size, _p(sim, _i32p), _p(pen, _i32p),
                                 ctypes.byref(A), ctypes.byref(scale))
    if st:
        raise ValueError("bad matrix")
    a = A.value
    return sim[: a * a].reshape(a, a).copy(), pen[: a * a].reshape(a, a).copy(), scale.value


def central_prior(lam: int):
    """``python/seqtree/gapblock.py:79-94``: 0 at d == 0, else ``int(lam * |2i + d - m| // 2)``
    (block [i, i + d) in a longer sequence of length m)."""
    if lam < 0:
        raise ValueError("lam must be >= 0")

    def prior(i: int, d: int, m: int) -> int:
        return 0 if d == 0 else int(lam * abs(2 * i + d - m) // 2)

    return prior


def prior_cube(prior, width: int) -> list[int]:
    """``python/seqtree/gapblock.py:492-509``: ``prior`` flattened to ``[m][d][i]`` with stride
    width + 1; only d >= 1 and i <= m - d are filled, the rest stay zero; a negative value
    raises ``ValueError``."""
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


def ref_gapblock_matrix(queries, refs, alphabet="aa", matrix=None, gap_open=1, gap_extend=1,
                        prior=(), prior_width=0, threads=0) -> np.ndarray:
    qd, qo = pack(queries)
    rd, ro = pack(refs)
    mid, simp, size, _keep = _matrix_args(matrix)
    pr = np.ascontiguousarray(np.asarray(prior, dtype=np.int64).astype(np.int32))
    if pr.size == 0:
        pr = np.zeros(1, np.int32)
        plen = 0
    else:
        plen = int(np.asarray(prior).size)
    out = np.zeros((len(queries), len(refs)), np.int32)
    err = ctypes.create_string_buffer(512)
    st = ref().ref_gapblock_matrix(qd.tobytes(), _p(qo, _i64p), len(queries), rd.tobytes(),
                                   _p(ro, _i64p), len(refs), ALPHABETS[alphabet], mid, simp, size,
                                   gap_open, gap_extend, _p(pr, _i32p), plen, prior_width,
                                   threads, _p(out, _i32p), err, 512)
    if st:
        _raise(st, err)
    return out


def ref_align_matrix(queries, refs, matrix="blosum62", mode="global", gap_open=11,
                     gap_extend=1, alphabet="aa", dist=False, threads=0) -> np.ndarray:
    qd, qo = pack(queries)
    rd, ro = pack(refs)
    mid, simp, size, _keep = _matrix_args(matrix)
    out = np.zeros((len(queries), len(refs)), np.int32)
    err = ctypes.create_string_buffer(512)
    st = ref().ref_align_matrix(qd.tobytes(), _p(qo, _i64p), len(queries), rd.tobytes(),
                                _p(ro, _i64p), len(refs), ALPHABETS[alphabet], mid, simp, size,
                                int(mode == "local"), gap_open, gap_extend, int(dist), threads,
                                _p(out, _i32p), err, 512)
    if st:
        _raise(st, err)
    return out


def ref_align_score(q, r, matrix="blosum62", mode="global", gap_open=11, gap_extend=1,
                    alphabet="aa") -> int:
    mid, simp, size, _keep = _matrix_args(matrix)
    out = ctypes.c_int32(0)
    err = ctypes.create_string_buffer(512)
    qb, rb = q.encode("latin-1"), r.encode("latin-1")
    st = ref().ref_align_score(qb, len(qb), rb, len(rb), ALPHABETS[alphabet], mid, simp, size,
                               int(mode == "local"), gap_open, gap_extend, ctypes.byref(out),
                               err, 512)
    if st:
        _raise(st, err)
    return out.value


def ref_align_pair(q, r, matrix="blosum62", mode="global", gap_open=11, gap_extend=1,
                   alphabet="aa") -> tuple[int, str, str, str]:
    """The reference's align_pair: (score, aligned_query, aligned_ref, ops)."""
    mid, simp, size, _keep = _matrix_args(matrix)
    cap = len(q) + len(r) + 2
    out = ctypes.c_int32(0)
    bufs = [ctypes.create_string_buffer(cap) for _ in range(3)]
    err = ctypes.create_string_buffer(512)
    qb, rb = q.encode("latin-1"), r.encode("latin-1")
    st = ref().ref_align_pair(qb, len(qb), rb, len(rb), ALPHABETS[alphabet], mid, simp, size,
                              int(mode == "local"), gap_open, gap_extend, ctypes.byref(out),
                              bufs[0], bufs[1], bufs[2], cap, err, 512)
    if st:
        _raise(st, err)
    return (out.value,) + tuple(b.value.decode("latin-1") for b in bufs)


def ref_index_align(refs, ref_id, query, matrix=None, gap_open=1, gap_extend=1,
                    alphabet="aa") -> tuple[int, str, str, str]:
    """The reference's Index.build(refs).align(ref_id, query, params):
    (score, aligned_query, aligned_ref, ops).  ``matrix`` None is unit cost."""
    mid, simp, size, _keep = _matrix_args(matrix)
    rd, ro = pack(refs)
    qb = query.encode("latin-1")
    cap = len(qb) + max((len(r) for r in refs), default=0) + 2
    out = ctypes.c_int32(0)
    bufs = [ctypes.create_string_buffer(cap) for _ in range(3)]
    err = ctypes.create_string_buffer(512)
    st = ref().ref_index_align(rd.tobytes(), _p(ro, _i64p), len(refs), ALPHABETS[alphabet],
                               int(ref_id), qb, len(qb), mid, simp, size, gap_open, gap_extend,
                               ctypes.byref(out), bufs[0], bufs[1], bufs[2], cap, err, 512)
    if st:
        _raise(st, err)
    return (out.value,) + tuple(b.value.decode("latin-1") for b in bufs)


def _wrap32(x: int) -> int:
    return (x + 2 ** 31) % 2 ** 32 - 2 ** 31


def penalty_align(query, ref, pen=None, gap_open=1, gap_extend=1,
                  alphabet="aa") -> tuple[int, str, str, str]:
    """Port of seqtree src/index.cpp:105-179 (Index::align), pure Python for small cases:
    min-cost global Gotoh in wrapping int32 with kInf = INT32_MAX // 4 borders (:127-137),
    ties M, then X / Y only when strictly smaller (:140-145), the traceback of :157-178 with
    the caller's own characters.  ``pen`` is the penalty grid (codes x codes) or None for unit
    cost on codec equality.  Returns (score, aligned_query, aligned_ref, ops)."""
    def codes(s):
        c, o = encode([s], alphabet)
        return [int(x) for x in c[:int(o[1])]]

    qc, rc = codes(query), codes(ref)
    if gap_open < 0 or gap_extend < 0:
        raise ValueError("seqtree: gap_open and gap_extend must be >= 0")
    go, ge = gap_open, gap_extend
    inf = (2 ** 31 - 1) // 4
    m, n = len(qc), len(rc)
    M = [[inf] * (n + 1) for _ in range(m + 1)]
    X = [[inf] * (n + 1) for _ in range(m + 1)]
    Y = [[inf] * (n + 1) for _ in range(m + 1)]
    bM = [[0] * (n + 1) for _ in range(m + 1)]
    bX = [[0] * (n + 1) for _ in range(m + 1)]
    bY = [[0] * (n + 1) for _ in range(m + 1)]
    M[0][0] = 0
    for i in range(1, m + 1):
        X[i][0] = _wrap32(go + (i - 1) * ge)
        bX[i][0] = 1 if i > 1 else 0
    for j in range(1, n + 1):
        Y[0][j] = _wrap32(go + (j - 1) * ge)
        bY[0][j] = 2 if j > 1 else 0

    def best3(mv, xv, yv):
        v, w = mv, 0
        if xv < v:
            v, w = xv, 1
        if yv < v:
            v, w = yv, 2
        return v, w

    for i in range(1, m + 1):
        for j in range(1, n + 1):
            sp = (0 if qc[i - 1] == rc[j - 1] else 1) if pen is None else int(pen[qc[i - 1]][rc[j - 1]])
            v, bM[i][j] = best3(M[i - 1][j - 1], X[i - 1][j - 1], Y[i - 1][j - 1])
            M[i][j] = _wrap32(sp + v)
            X[i][j], bX[i][j] = best3(_wrap32(M[i - 1][j] + go), _wrap32(X[i - 1][j] + ge),
                                      _wrap32(Y[i - 1][j] + go))
            Y[i][j], bY[i][j] = best3(_wrap32(M[i][j - 1] + go), _wrap32(X[i][j - 1] + go),
                                      _wrap32(Y[i][j - 1] + ge))
    score, st = best3(M[m][n], X[m][n], Y[m][n])
    aq, ar, ops = [], [], []
    i, j = m, n
    while i > 0 or j > 0:
        if st == 0:
            aq.append(query[i - 1])
            ar.append(ref[j - 1])
            ops.append("M" if qc[i - 1] == rc[j - 1] else "S")
            st = bM[i][j]
            i, j = i - 1, j - 1
        elif st == 1:
            aq.append(query[i - 1])
            ar.append("-")
            ops.append("D")
            st = bX[i][j]
            i -= 1
        else:
            aq.append("-")
            ar.append(ref[j - 1])
            ops.append("I")
            st = bY[i][j]
            j -= 1
    return score, "".join(reversed(aq)), "".join(reversed(ar)), "".join(reversed(ops))


def ref_distance_matrix(a, b, levenshtein: bool, threads=0) -> np.ndarray:
    ad, ao = pack(a)
    bd, bo = pack(b)
    out = np.zeros((len(a), len(b)), np.int32)
    err = ctypes.create_string_buffer(512)
    st = ref().ref_distance_matrix(ad.tobytes(), _p(ao, _i64p), len(a), bd.tobytes(),
                                   _p(bo, _i64p), len(b), int(levenshtein), threads,
                                   _p(out, _i32p), err, 512)
    if st:
        _raise(st, err)
    return out


# ----------------------------------------------------------------------------- E-value cutoffs
def _theta(scores, k, c_max, theta_max):
    """Port of seqtree python/seqtree/evalue.py:86-99 (_theta)."""
    if k < 1:
        return -1
    theta = theta_max if len(scores) <= k else min(theta_max, scores[k] - 1)
    if theta < 0:
        return -1
    n_control = sum(1 for s in scores if s <= theta)
    if n_control == 0 and c_max < 3.0:
        return -1
    return theta


def thetas_from_scores(control_scores, n_target, m_control, e_target, theta_max, *,
                       exclude_exact=False):
    """Port of seqtree python/seqtree/evalue.py:102-143 (thetas_from_scores)."""
    if n_target <= 0 or m_control <= 0:
        raise ValueError("n_target and m_control must be > 0")
    if e_target <= 0.0:
        raise ValueError("e_target must be > 0")
    if theta_max < 0:
        raise ValueError("theta_max must be >= 0")
    c_max = e_target * m_control / n_target
    k = int(c_max)
    return [_theta(sorted(x for x in s if not (exclude_exact and x == 0)), k, c_max, theta_max)
            for s in control_scores]


# ----------------------------------------------------------------------------- island profiles
PROFILE_UNREACHABLE = 1 << 20  # seqtree python/seqtree/gapblock.py:54


def profile_score(penalties, width, c, seq, gap="-"):
    """Port of IslandProfile.score (seqtree python/seqtree/gapblock.py:365-374) with
    embed_in_frame (:186-205)."""
    if len(seq) > width or c > len(seq):
        return PROFILE_UNREACHABLE
    d = width - len(seq)
    emb = seq[:c] + gap * d + seq[c:]
    cap = PROFILE_UNREACHABLE // (width + 1)
    return sum(penalties[j].get(ch, cap) for j, ch in enumerate(emb))
