"""The C-ABI library: it loads, exports every entry point the header declares, and rejects bad
arguments with the reference's messages before touching a device (no GPU needed here)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from seqtree_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "seqtree_b200.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(st_[a-z_0-9]+)\s*\(", text))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 18
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for n in sorted(names):
        assert hasattr(lib, n), f"{n} declared in the header but not exported"


def test_python_binding_covers_the_header():
    assert {s[0] for s in _lib.SIGNATURES} == declared_symbols()


def test_version_and_device_count_without_a_device():
    assert _lib.lib.st_version() == 100
    assert _lib.lib.st_device_count() >= 0


def _strings(seqs):
    return _lib.Packed(seqs)


def _gap(q, r, go=1, ge=1, alphabet=0, pen=None, size=0, out=None):
    err = _lib.st_error()
    out = np.zeros(max(1, len(q) * len(r)), np.int32) if out is None else out
    code = _lib.lib.st_gapblock_matrix(_strings(q).ref(), _strings(r).ref(), alphabet,
                                       _lib.i32_ptr(pen), size, go, ge, None, 0, 0, 0,
                                       out.ctypes.data, ctypes.byref(err))
    return code, err.message.decode()


def test_argument_checks_come_first_and_match_the_reference():
    # src/gapblock.cpp:71-77
    code, msg = _gap(["CAS"], ["CAS"], go=-1)
    assert code == _lib.ST_EINVAL and msg == "gap_open and gap_extend must be >= 0"
    code, msg = _gap(["CAS"], ["CAS"], ge=-3)
    assert code == _lib.ST_EINVAL
    pen = np.zeros((4, 4), np.int32)
    code, msg = _gap(["CAS"], ["CAS"], alphabet=0, pen=pen, size=4)
    assert code == _lib.ST_EINVAL and msg == "matrix size does not match the alphabet"
    code, msg = _gap(["CAS"], ["CAS"], alphabet=7)
    assert code == _lib.ST_EINVAL


def test_empty_shapes_return_without_a_device():
    # src/gapblock.cpp:80-81, src/pairwise.cpp:281-282, src/distance.cpp:33-34
    assert _gap([], ["ACGT"])[0] == _lib.ST_OK
    assert _gap(["AC#T"], [])[0] == _lib.ST_OK  # nothing is encoded when a side is empty
    err = _lib.st_error()
    out = np.zeros(1, np.int32)
    assert _lib.lib.st_hamming_matrix(_strings([]).ref(), _strings(["A"]).ref(), 0,
                                      out.ctypes.data, ctypes.byref(err)) == _lib.ST_OK
    sim = np.eye(24, dtype=np.int32)
    assert _lib.lib.st_align_score_matrix(_strings([]).ref(), _strings(["A"]).ref(),
                                          _lib.i32_ptr(sim), 24, 0, 0, 11, 1, 0, out.ctypes.data,
                                          ctypes.byref(err)) == _lib.ST_OK
    code = _lib.lib.st_align_score_matrix(_strings(["A"]).ref(), _strings(["A"]).ref(),
                                          _lib.i32_ptr(sim), 24, 0, 0, -1, 1, 0, out.ctypes.data,
                                          ctypes.byref(err))
    assert code == _lib.ST_EINVAL and "gap_open and gap_extend must be >= 0" in \
        err.message.decode()
    code = _lib.lib.st_align_score_matrix(_strings(["A"]).ref(), _strings(["A"]).ref(),
                                          _lib.i32_ptr(sim), 24, 0, 5, 11, 1, 0, out.ctypes.data,
                                          ctypes.byref(err))
    assert code == _lib.ST_EINVAL


def test_null_handles_are_rejected():
    err = _lib.st_error()
    code = _lib.lib.st_gapblock_matrix_sets(None, None, None, 0, 1, 1, None, 0, 0, None, None,
                                            ctypes.byref(err))
    assert code == _lib.ST_EINVAL
    assert _lib.lib.st_seqset_count(None) == -1


def test_no_cpu_fallback_when_no_device_is_usable():
    if _lib.device_count() > 0:
        pytest.skip("a device is present; this checks the device-less path")
    code, msg = _gap(["CASS"], ["CAS"])
    assert code == _lib.ST_ENODEV and "no usable CUDA device" in msg
    from seqtree_b200 import score_matrix
    with pytest.raises(RuntimeError, match="CUDA"):
        score_matrix(["CASS"], ["CAS"])
