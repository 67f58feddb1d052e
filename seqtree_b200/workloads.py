"""Seeded synthetic inputs of the named all-vs-all scoring workloads.

These are the shapes and value distributions the benchmark times and the full-size parity tests
check, so both read them from here.  numpy only: importing this module loads no compiled code, so
a process that times the reference's CPU implementation on the same inputs stays free of this
library's shared object.  Seeds: numpy PCG64, 1 for queries and 0 for refs on the named
workloads (a rank r > 0 of a multi-GPU run draws its query block from seed 1 + 1000 r).

* gap-block dense (1,000 x 10,000): :func:`cdr3`, 'CASS' + uniform middle + 'F', length
  uniform 10-20;
* Hamming / Levenshtein (20,000 x 20,000): :func:`uniform_strings` over ACGT, length 12 or
  uniform 30-60;
* NW / SW (4,096 x 4,096): :func:`proteins`, residues i.i.d. from background frequencies,
  length log-normal (median 180, sigma 0.5), clipped to 50-500;
* sparse gap-block (100,000 x 1,000,000): :func:`cdr3_skewed`, length 8-25 with mode 14;
* learned proposal (1,000,000 x 1,000,000): :func:`cdr3_codes`, the same length law as codes.
"""
from __future__ import annotations

import numpy as np

AA20 = "ACDEFGHIKLMNPQRSTVWY"
AA24 = "ARNDCQEGHILKMFPSTWYVBZX*"  # the amino-acid codec's symbol order (code = index)
PAD = 32                           # code rows of the learned path are padded to 32 positions

CODE = np.full(256, 255, np.uint8)  # ASCII -> amino-acid code (255: not a symbol)
for _i, _c in enumerate(AA24):
    CODE[ord(_c)] = _i
    CODE[ord(_c.lower())] = _i
LETTER = np.frombuffer(AA24.encode(), np.uint8)             # code -> ASCII
AA20_CODES = CODE[np.frombuffer(AA20.encode(), np.uint8)]  # the 20 standard residues as codes
_C, _A, _S, _F = (int(CODE[ord(x)]) for x in "CASF")

# Background amino-acid frequencies (Robinson & Robinson 1991), order ACDEFGHIKLMNPQRSTVWY.
BG_FREQ = np.array([7.805, 1.925, 5.364, 6.295, 3.856, 7.377, 2.199, 5.142, 5.744, 9.019, 2.243,
                    4.487, 5.203, 4.264, 5.129, 7.120, 5.841, 6.441, 1.330, 3.216])


def _split(letters: str, lens) -> list[str]:
    out, p = [], 0
    for L in lens:
        out.append(letters[p:p + int(L)])
        p += int(L)
    return out


def cdr3(seed: int, n: int, lo: int = 10, hi: int = 20) -> list[str]:
    """'CASS' + uniform middle from the 20 standard residues + 'F', length uniform [lo, hi]."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, size=n)
    mid = rng.integers(0, 20, size=int((lens - 5).sum()))
    letters = np.array(list(AA20))[mid]
    out, p = [], 0
    for L in lens:
        k = int(L) - 5
        out.append("CASS" + "".join(letters[p:p + k]) + "F")
        p += k
    return out


def uniform_strings(seed: int, n: int, lo: int, hi: int, alphabet: str) -> list[str]:
    """Symbols i.i.d. uniform over ``alphabet``, length uniform [lo, hi]."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, size=n)
    codes = rng.integers(0, len(alphabet), size=int(lens.sum()))
    letters = np.array(list(alphabet))[codes]
    out, p = [], 0
    for L in lens:
        out.append("".join(letters[p:p + int(L)]))
        p += int(L)
    return out


def proteins(seed: int, n: int) -> list[str]:
    """Residues i.i.d. from :data:`BG_FREQ`; length log-normal, median 180, sigma 0.5, clipped to
    50-500."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.round(rng.lognormal(np.log(180), 0.5, size=n)), 50, 500).astype(int)
    p = BG_FREQ / BG_FREQ.sum()
    codes = rng.choice(20, size=int(lens.sum()), p=p)
    letters = np.array(list(AA20))[codes]
    out, o = [], 0
    for L in lens:
        out.append("".join(letters[o:o + int(L)]))
        o += int(L)
    return out


def cdr3_lengths(rng, n: int) -> np.ndarray:
    """Junction lengths 8-25 with mode 14: P(L) is a Gaussian around 14 with sigma 2.5 below and
    3.5 above (right-skewed, like TRB junctions)."""
    L = np.arange(8, 26)
    sig = np.where(L < 14, 2.5, 3.5)
    p = np.exp(-0.5 * ((L - 14) / sig) ** 2)
    return rng.choice(L, size=n, p=p / p.sum()).astype(np.int32)


def cdr3_skewed(seed: int, n: int) -> list[str]:
    """'CASS' + uniform middle + 'F' with the lengths of :func:`cdr3_lengths`."""
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


def cdr3_codes(seed: int, n: int) -> tuple[np.ndarray, np.ndarray]:
    """n CDR3-like junctions 'CASS' + uniform middle + 'F' (lengths from :func:`cdr3_lengths`)
    as amino-acid codes [n, 32] (zero past each length) and lengths [n]."""
    rng = np.random.default_rng(seed)
    lens = cdr3_lengths(rng, n)
    codes = AA20_CODES[rng.integers(0, 20, size=(n, PAD), dtype=np.uint8)]
    codes[:, :4] = (_C, _A, _S, _S)
    codes[np.arange(n), lens - 1] = _F
    codes[np.arange(PAD)[None, :] >= lens[:, None]] = 0
    return codes, lens


def codes_to_letters(codes: np.ndarray, lens: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Codes [n, 32] + lengths as one concatenated ASCII buffer and int64 offsets [n + 1]."""
    lens = np.asarray(lens, np.int64)
    data = LETTER[codes[np.arange(PAD)[None, :] < lens[:, None]]]
    off = np.zeros(lens.size + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    return data, off


def codes_to_strings(codes: np.ndarray, lens: np.ndarray) -> list[str]:
    data, off = codes_to_letters(codes, lens)
    text = data.tobytes().decode() if off[-1] else ""
    return [text[a:b] for a, b in zip(off[:-1].tolist(), off[1:].tolist())]
