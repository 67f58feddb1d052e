"""The learned encoder's model file (no device needed): round trip, the errors a damaged or
foreign file raises, and the atomic write that never leaves a half-written file or a temporary."""
from __future__ import annotations

import os
import struct

import numpy as np
import pytest

from seqtree_b200 import learned as L


def test_round_trip_keeps_every_bit_and_the_metadata():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(1234).astype(np.float32)
    p[:3] = [np.float32(-0.0), np.float32(1e-38), np.float32(3.4e38)]
    meta = {"k": 256, "query_fallback": [8, 9, 10], "ref_fallback": [], "max_penalty": 24}
    got, m = L.decode_model(L.encode_model(p, meta))
    assert got.dtype == np.float32 and got.tobytes() == p.tobytes() and m == meta
    empty, m0 = L.decode_model(L.encode_model(np.zeros(0, np.float32)))
    assert empty.size == 0 and m0 == {}


def test_foreign_truncated_and_corrupt_files_raise():
    data = L.encode_model(np.arange(10, dtype=np.float32), {"a": 1})
    with pytest.raises(ValueError, match="not a seqtree_b200 encoder file"):
        L.decode_model(b"XXXX" + data[4:])
    with pytest.raises(ValueError, match="not a seqtree_b200 encoder file"):
        L.decode_model(data[:10])
    newer = data[:4] + struct.pack("<I", 2) + data[8:]
    with pytest.raises(ValueError, match="version 2"):
        L.decode_model(newer)
    with pytest.raises(ValueError, match="truncated or corrupt"):
        L.decode_model(data[:-1])
    flipped = bytearray(data)
    flipped[30] ^= 0x40
    with pytest.raises(ValueError, match="checksum"):
        L.decode_model(bytes(flipped))


def test_atomic_write_replaces_whole_files_and_cleans_up(tmp_path):
    target = tmp_path / "enc.stbe"
    L.atomic_write(target, b"first")
    L.atomic_write(target, b"second version")
    assert target.read_bytes() == b"second version"
    assert sorted(os.listdir(tmp_path)) == ["enc.stbe"]

    bad_dir = tmp_path / "missing" / "enc.stbe"  # the temporary cannot be created
    with pytest.raises(OSError):
        L.atomic_write(bad_dir, b"x")
    with pytest.raises(TypeError):  # a write that fails part way: no temporary is left behind
        L.atomic_write(target, object())  # type: ignore[arg-type]
    assert sorted(os.listdir(tmp_path)) == ["enc.stbe"]
    assert target.read_bytes() == b"second version"
