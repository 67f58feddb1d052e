"""The reference's own hot-path test files, run against this library through
``tests/reference_suite_plugin.py`` (``seqtree`` mapped to ``seqtree_b200``).

The files are the reference project's ``tests/python/test_gapblock.py``, ``test_pairwise.py``,
``test_distance.py`` and ``test_matrix.py`` (with its ``conftest.py``).  They are not part of this
repository; ``SEQTREE_REFERENCE_TESTS`` names a directory holding them (the reference's
``tests/python`` or a copy of it).  Without it this test is skipped.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
FILES = ["test_gapblock.py", "test_pairwise.py", "test_distance.py", "test_matrix.py"]


def test_reference_hot_path_suites_pass_against_the_drop_in(cuda_ready):
    src = os.environ.get("SEQTREE_REFERENCE_TESTS")
    if not src:
        pytest.skip("SEQTREE_REFERENCE_TESTS does not name the reference's tests/python directory")
    src = Path(src).resolve()
    missing = [f for f in FILES if not (src / f).exists()]
    if missing:
        pytest.skip(f"reference test files not found under {src}: {missing}")
    here = Path(__file__).resolve().parent
    env = dict(os.environ, PYTHONPATH=os.pathsep.join([str(here.parent), str(here)]))
    res = subprocess.run(
        [sys.executable, "-m", "pytest", "-p", "reference_suite_plugin", "-p", "no:cacheprovider",
         "--rootdir", str(src), "-q", "-rs", *[str(src / f) for f in FILES]],
        env=env, cwd=str(src), capture_output=True, text=True, timeout=1800)
    tail = res.stdout[-6000:] + res.stderr[-2000:]
    print(tail)
    assert res.returncode == 0, tail
    m = re.search(r"(\d+) passed", res.stdout)
    assert m and int(m.group(1)) >= 100, tail
