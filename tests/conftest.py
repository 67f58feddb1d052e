"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and call the library through its
C ABI; everything else runs on the CPU (the oracle, host logic, library loading)."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

AA20 = "ACDEFGHIKLMNPQRSTVWY"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


def load_golden(name: str):
    return json.loads((GOLDEN / f"{name}.json").read_text())


@pytest.fixture(scope="session")
def golden_tables():
    return load_golden("tables")


@pytest.fixture(scope="session")
def golden_gapblock():
    return load_golden("gapblock")


@pytest.fixture(scope="session")
def golden_align():
    return load_golden("align")


@pytest.fixture(scope="session")
def golden_distance():
    return load_golden("distance")


def rand_seqs(rng, n, lo, hi, alphabet=AA20):
    lens = rng.integers(lo, hi + 1, size=n)
    return ["".join(rng.choice(list(alphabet), size=int(L))) for L in lens]


def cdr3(rng, n, lo=10, hi=20):
    lens = rng.integers(lo, hi + 1, size=n)
    return ["CASS" + "".join(rng.choice(list(AA20), size=int(L) - 5)) + "F" for L in lens]


def prior_by_name(name):
    from seqtree_b200.gapblock import central_prior, frame_prior, positions_prior, profile_prior
    return {
        "none": None,
        "central21": central_prior(21),
        "frame21_5": frame_prior(21, 5),
        "positions": positions_prior((3, 4, -4, -3)),
        "profile21": profile_prior(21, lambda j, m: 1.0 - abs(2 * j + 1 - m) / m),
    }[name]


@pytest.fixture(scope="session")
def cuda_ready():
    """The CUDA library with a device behind it; fails (never skips) when either is missing."""
    from seqtree_b200 import _lib
    n = _lib.device_count()
    assert n > 0, "no CUDA device visible to libseqtree_b200"
    return _lib


def as_np(sm) -> np.ndarray:
    return np.asarray(sm)
