"""The float64 encoder restatement (oracle/encoder.py) against finite differences: its
hand-derived backward pass is what the CUDA training kernels are checked against."""
from __future__ import annotations

import numpy as np

import oracle.encoder as enc


def _batch(rng, S=6):
    lens = rng.integers(3, 14, size=S).astype(np.int32)
    codes = rng.integers(0, 24, size=(S, 32)).astype(np.uint8)
    for s in range(S):
        codes[s, lens[s]:] = 0
    return codes, lens, rng.integers(0, 90, size=S // 2)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    codes, lens, scores = _batch(rng)
    flat = enc.init_params(1).astype(np.float64) + rng.normal(0, 0.05, enc.param_count())
    loss, g = enc.backward(flat, codes, lens, scores)
    assert np.isfinite(loss) and loss > 0
    o = 0
    for name, shape in enc.SHAPES:
        n = int(np.prod(shape))
        for i in o + np.argsort(-np.abs(g[o:o + n]))[:3]:
            e = 1e-5
            f1, f2 = flat.copy(), flat.copy()
            f1[i] += e
            f2[i] -= e
            num = (enc.loss_only(f1, codes, lens, scores) - enc.loss_only(f2, codes, lens, scores)) / (2 * e)
            assert abs(num - g[i]) <= 1e-6 * max(1.0, abs(num)), (name, num, g[i])
        o += n


def test_oracle_embeddings_are_unit_and_padding_free():
    rng = np.random.default_rng(2)
    codes, lens, _ = _batch(rng, 4)
    flat = enc.init_params(3)
    z = enc.forward(flat, codes, lens)
    np.testing.assert_allclose(np.linalg.norm(z, axis=1), 1.0, rtol=1e-12)
    codes2 = codes.copy()
    for s in range(4):
        codes2[s, lens[s]:] = 7  # garbage past the length changes nothing
    np.testing.assert_allclose(enc.forward(flat, codes2, lens), z)
