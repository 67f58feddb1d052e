"""The C++ API (include/seqtree_b200.hpp), driven by a small C++ program compiled here with g++
against the header and linked to libseqtree_b200.so, the way a seqtree C++ caller would use it.
The built-in tables need no GPU; the matrix calls are checked against the oracle on the GPU."""
from __future__ import annotations

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from conftest import cdr3, rand_seqs
from seqtree_b200 import _lib
from seqtree_b200.gapblock import central_prior, prior_cube
from seqtree_b200.matrix import SubstitutionMatrix

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "api_check.cpp"


@pytest.fixture(scope="session")
def api_check(tmp_path_factory):
    gxx = shutil.which("g++")
    assert gxx, "g++ is needed to build the C++ API check"
    exe = tmp_path_factory.mktemp("cpp") / "api_check"
    libdir = _lib.LIB_PATH.parent
    subprocess.run([gxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                    f"-I{ROOT / 'include'}", str(SRC), f"-L{libdir}", "-lseqtree_b200",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    return exe


def parse(text: str) -> dict[str, object]:
    out = {}
    for line in text.splitlines():
        name, _, rest = line.partition(" ")
        out[name] = rest[1:] if rest.startswith("!") else [int(x) for x in rest.split()]
    return out


def test_builtin_tables_match_the_reference(api_check, golden_tables):
    got = parse(subprocess.run([str(api_check), "tables"], check=True, capture_output=True,
                               text=True).stdout)
    for name in ("blosum62", "blosum45", "blosum80", "pam250", "pam100", "structural"):
        v = got[name]
        size, scale = v[0], v[1]
        pen = np.array(v[2:2 + size * size]).reshape(size, size)
        sim = np.array(v[2 + size * size:]).reshape(size, size)
        g = golden_tables[name]
        assert size == 24 and scale == g["scale"], name
        np.testing.assert_array_equal(sim, np.asarray(g["sim"]).reshape(24, 24), err_msg=name)
        np.testing.assert_array_equal(pen, np.asarray(g["pen"]).reshape(24, 24), err_msg=name)
        py = getattr(SubstitutionMatrix, name)()
        np.testing.assert_array_equal(pen, py.penalty_grid)
    size, scale, p01, p22, s11, s12 = got["unit4"]
    g = golden_tables["unit4"]
    assert (size, scale) == (4, g["scale"])
    assert (p01, p22, s11, s12) == (1, 0, 1, 0)


def test_builtin_similarity_rejects_unknown_names():
    err = _lib.st_error()
    size = ctypes.c_int32(0)
    rc = _lib.lib.st_builtin_similarity(b"blosum99", None, 0, ctypes.byref(size),
                                        ctypes.byref(err))
    assert rc == _lib.ST_EINVAL and b"blosum99" in err.message
    buf = (ctypes.c_int32 * 100)()
    rc = _lib.lib.st_builtin_similarity(b"pam250", buf, 100, ctypes.byref(size),
                                        ctypes.byref(err))
    assert rc == _lib.ST_EINVAL and size.value == 24


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1])
def test_cpp_api_matches_the_oracle(api_check, cuda_ready, seed):
    rng = np.random.default_rng(seed)
    q = cdr3(rng, 23) + ["CASSF", "C"]
    r = cdr3(rng, 41) + ["CASSLGQF", "W"]
    h = rand_seqs(rng, 9, 14, 14, "ACGT")
    width = max(map(len, q + r))
    cube = np.asarray(prior_cube(central_prior(21), width), np.int32).ravel()
    stdin = "\n".join([f"Q {len(q)}", *q, f"R {len(r)}", *r, f"H {len(h)}", *h,
                       f"P {width} {cube.size}", " ".join(map(str, cube.tolist()))]) + "\n"
    out = subprocess.run([str(api_check), "run"], input=stdin, check=True, capture_output=True,
                         text=True).stdout
    got = parse("\n".join(line for line in out.splitlines()
                          if not line.startswith(("alignpair ", "penalign "))))
    b62 = SubstitutionMatrix.blosum62()
    N, K = len(q), len(r)

    def m(name):
        assert isinstance(got[name], list), got[name]
        return np.array(got[name], np.int32).reshape(N, K)

    np.testing.assert_array_equal(
        m("gapblock_b62_prior"),
        oracle.gapblock_matrix(q, r, b62.penalty_grid, gap_open=8, gap_extend=1, prior=cube,
                               prior_width=width))
    np.testing.assert_array_equal(
        m("gapblock_unit"),
        oracle.gapblock_matrix(q, r, SubstitutionMatrix.unit(24).penalty_grid))
    sim = b62.similarity_grid
    np.testing.assert_array_equal(m("align_score_global"),
                                  oracle.align_matrix(q, r, sim, mode="global"))
    np.testing.assert_array_equal(m("align_dist_local"),
                                  oracle.align_matrix(q, r, sim, mode="local", dist=True))
    assert got["align_score_one"] == [int(oracle.align_matrix(q[:1], r[:1], sim)[0, 0])]
    np.testing.assert_array_equal(m("levenshtein"), oracle.levenshtein_matrix(q, r))
    assert got["levenshtein_one"] == [int(oracle.levenshtein_matrix(q[:1], r[:1])[0, 0])]
    np.testing.assert_array_equal(np.array(got["hamming"]).reshape(9, 9),
                                  oracle.hamming_matrix(h, h))
    assert got["hamming_one"] == [int(oracle.hamming_matrix(h[:1], h[1:2])[0, 0])]
    assert got["hamming_ragged"] == ("invalid_argument: seqtree: hamming distance is only "
                                     "defined for equal-length sequences (got 3 and 4)")
    assert got["gapblock_bad_symbol"].startswith("invalid_argument: symbol 'J'")
    assert got["align_overflow"].startswith("overflow_error: seqtree: the alignment score")
    assert got["align_pair_bad_symbol"] == "invalid_argument: invalid symbol 'J' in sequence"
    assert got["penalty_align_bad_symbol"] == "invalid_argument: invalid symbol 'J' in query"
    pen = [line.split(" ") for line in out.splitlines() if line.startswith("penalign ")]
    assert len(pen) == min(N, K)
    for _, i, score, aq, ar, ops in pen:
        un = lambda x: "" if x == "~" else x  # noqa: E731
        i = int(i)
        want = oracle.penalty_align(q[i], r[i], None if i & 1 else b62.penalty_grid, 11, 1)
        assert (int(score), un(aq), un(ar), un(ops)) == want
    pairs = [line.split(" ") for line in out.splitlines() if line.startswith("alignpair ")]
    assert len(pairs) == 2 * min(N, K)
    for _, i, md, score, aq, ar, ops in pairs:
        un = lambda x: "" if x == "~" else x  # noqa: E731
        i, mode = int(i), "local" if md == "1" else "global"
        if oracle.ref_available():
            want = oracle.ref_align_pair(q[i], r[i], "blosum62", mode=mode)
            assert (int(score), un(aq), un(ar), un(ops)) == want
