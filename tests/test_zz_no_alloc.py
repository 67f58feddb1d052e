"""The allocation-free Levenshtein entry point, for callers that cannot let a library allocate
device memory: inputs and output live in the caller's device memory and the kernel's scratch is a
fixed array inside the library.  Checked through the C ABI against the allocating entry point
(st_levenshtein_matrix) and the oracle, on two calls in a row.  This file is collected last on
purpose."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from conftest import AA20, rand_seqs

pytestmark = pytest.mark.gpu


def _device_strings(torch, seqs):
    from seqtree_b200 import _lib
    p = _lib.Packed(seqs)
    data = torch.from_numpy(np.array(p.data, dtype=np.uint8)).cuda()
    off = torch.from_numpy(np.array(p.offsets, dtype=np.int64)).cuda()
    return data, off, p.count


def _call(lib, torch, a, b, out):
    err = lib.st_error()
    rc = lib.lib.st_levenshtein_matrix_noalloc(
        a[0].data_ptr(), a[1].data_ptr(), a[2], b[0].data_ptr(), b[1].data_ptr(), b[2],
        out.data_ptr(), torch.cuda.current_stream().cuda_stream, ctypes.byref(err))
    return rc, err.message.decode()


def _twice(lib, torch, a, b, expected):
    da, db = _device_strings(torch, a), _device_strings(torch, b)
    out = torch.empty((len(a), len(b)), dtype=torch.int32, device="cuda")
    for _ in range(2):  # the fixed scratch keeps the previous call's contents
        out.fill_(-7)
        rc, msg = _call(lib, torch, da, db, out)
        assert rc == lib.ST_OK, msg
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), expected)


def test_no_alloc_levenshtein_matches_the_allocating_entry_point(cuda_ready):
    import torch
    from seqtree_b200 import _lib
    from seqtree_b200.distance import levenshtein_matrix
    rng = np.random.default_rng(21)
    a = rand_seqs(rng, 123, 0, 70, "ACGT") + ["", "kitten"]
    b = rand_seqs(rng, 301, 0, 90, AA20 + "acgt") + ["sitting", ""]
    expected = np.asarray(levenshtein_matrix(a, b))
    _twice(_lib, torch, a, b, expected)
    assert expected[-1, -2] == 3  # kitten / sitting


@pytest.mark.parametrize("na,nb", [(1, 1), (10, 20)])
def test_no_alloc_small_matrices(cuda_ready, na, nb):
    """Fewer pairs than one block of threads: the grid is sized to the pairs, not rejected."""
    import torch
    from seqtree_b200 import _lib
    rng = np.random.default_rng(na * 100 + nb)
    a = rand_seqs(rng, na, 0, 40, "ACGT")
    b = rand_seqs(rng, nb, 1, 50, "ACGT")
    _twice(_lib, torch, a, b, oracle.levenshtein_matrix(a, b, threads=1))


def test_no_alloc_rejects_rows_beyond_the_fixed_scratch(cuda_ready):
    """256 pairs of 40,000-byte strings: enough pairs for a full block, so only the DP row
    (40,001 words per thread, 256 threads > 32 MiB) is what fails."""
    import torch
    from seqtree_b200 import _lib
    da = _device_strings(torch, ["A" * 40000] * 16)
    db = _device_strings(torch, ["C" * 40000] * 16)
    out = torch.full((16, 16), -7, dtype=torch.int32, device="cuda")
    rc, msg = _call(_lib, torch, da, db, out)
    assert rc == _lib.ST_EINVAL and "fixed 32 MiB scratch" in msg and "40001 words" in msg
    torch.cuda.synchronize()
    assert bool((out == -7).all())  # nothing was launched


def test_no_alloc_rejects_null_byte_pointers(cuda_ready):
    import torch
    from seqtree_b200 import _lib
    da = _device_strings(torch, ["ACGT"])
    out = torch.full((1, 1), -7, dtype=torch.int32, device="cuda")
    err = _lib.st_error()
    rc = _lib.lib.st_levenshtein_matrix_noalloc(
        None, da[1].data_ptr(), 1, da[0].data_ptr(), da[1].data_ptr(), 1, out.data_ptr(),
        torch.cuda.current_stream().cuda_stream, ctypes.byref(err))
    assert rc == _lib.ST_EINVAL and "null device pointer" in err.message.decode()
