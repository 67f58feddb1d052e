"""The allocation-free Levenshtein entry point, for callers that cannot let a library allocate
device memory: inputs and output live in the caller's device memory and the kernel's scratch is a
fixed array inside the library.  Checked through the C ABI against the allocating entry point
(st_levenshtein_matrix), on two calls in a row.  This file is collected last on purpose."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

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


def test_no_alloc_levenshtein_matches_the_allocating_entry_point(cuda_ready):
    import torch
    from seqtree_b200 import _lib
    from seqtree_b200.distance import levenshtein_matrix
    rng = np.random.default_rng(21)
    a = rand_seqs(rng, 123, 0, 70, "ACGT") + ["", "kitten"]
    b = rand_seqs(rng, 301, 0, 90, AA20 + "acgt") + ["sitting", ""]
    expected = np.asarray(levenshtein_matrix(a, b))
    da, db = _device_strings(torch, a), _device_strings(torch, b)
    out = torch.empty((len(a), len(b)), dtype=torch.int32, device="cuda")
    for _ in range(2):  # the fixed scratch keeps the previous call's contents
        out.fill_(-7)
        rc, msg = _call(_lib, torch, da, db, out)
        assert rc == _lib.ST_OK, msg
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), expected)
    assert expected[-1, -2] == 3  # kitten / sitting


def test_no_alloc_rejects_rows_beyond_the_fixed_scratch(cuda_ready):
    import torch
    from seqtree_b200 import _lib
    long = ["A" * 40000]
    da, db = _device_strings(torch, long), _device_strings(torch, ["C" * 40000])
    out = torch.full((1, 1), -7, dtype=torch.int32, device="cuda")
    rc, msg = _call(_lib, torch, da, db, out)
    assert rc == _lib.ST_EINVAL and "fixed" in msg
    torch.cuda.synchronize()
    assert int(out.item()) == -7  # nothing was launched
