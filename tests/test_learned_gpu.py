"""The learned-proposal path on the GPU: the encoder's training kernels against the float64
oracle (loss, every gradient, the forward embedding), training progress, and the exact pair
scorer against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import oracle.encoder as oenc
from conftest import cdr3
from seqtree_b200.matrix import SubstitutionMatrix


def _batch(rng, S):
    from seqtree_b200.learned import pad_codes
    seqs = cdr3(rng, S, 8, 25)
    codes, lens = pad_codes(seqs)
    return seqs, codes, lens, rng.integers(0, 90, size=S // 2).astype(np.int32)


@pytest.mark.gpu
@pytest.mark.parametrize("S", [16, 258])
def test_encoder_gradients_match_the_oracle(cuda_ready, S):
    from seqtree_b200.learned import Encoder
    rng = np.random.default_rng(S)
    _, codes, lens, scores = _batch(rng, S)
    flat = (oenc.init_params(5) + rng.normal(0, 0.05, oenc.param_count())).astype(np.float32)
    enc = Encoder(flat, precision="fp32")
    loss, g = enc.loss_grad(codes, lens, scores)
    want_loss, want_g = oenc.backward(flat.astype(np.float64), codes, lens, scores)
    assert loss == pytest.approx(want_loss, rel=1e-4)
    # fp32 against float64: every block within 1e-3 of its largest gradient
    o = 0
    for name, shape in oenc.SHAPES:
        n = int(np.prod(shape))
        a, b = g[o:o + n], want_g[o:o + n]
        scale = max(np.abs(b).max(), 1e-12)
        assert np.abs(a - b).max() <= 2e-3 * scale, (name, np.abs(a - b).max(), scale)
        o += n


@pytest.mark.gpu
@pytest.mark.parametrize("S", [16, 1024])
def test_bf16_training_gradients_track_the_oracle(cuda_ready, S):
    """The default training precision: dense-layer products on the bf16 tensor cores with fp32
    accumulation.  Against the float64 oracle the loss stays within 1% and every gradient
    block within 5% (relative norm) of the exact gradient, cosine >= 0.998 -- bf16 rounding of
    the operands, not a wrong term (a dropped or misplaced product moves a block by O(1))."""
    from seqtree_b200.learned import Encoder
    rng = np.random.default_rng(S + 1)
    _, codes, lens, scores = _batch(rng, S)
    flat = (oenc.init_params(5) + rng.normal(0, 0.05, oenc.param_count())).astype(np.float32)
    enc = Encoder(flat)
    assert enc.precision == "bf16"
    loss, g = enc.loss_grad(codes, lens, scores)
    want_loss, want_g = oenc.backward(flat.astype(np.float64), codes, lens, scores)
    assert loss == pytest.approx(want_loss, rel=1e-2)
    o = 0
    for name, shape in oenc.SHAPES:
        n = int(np.prod(shape))
        a, b = g[o:o + n].astype(np.float64), want_g[o:o + n]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        cos = float(a @ b) / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        assert rel <= 0.05 and cos >= 0.998, (name, rel, cos)
        o += n
    with pytest.raises(ValueError, match="precision"):
        enc.set_precision("fp16")


@pytest.mark.gpu
def test_encoder_embeddings_match_the_oracle_forward(cuda_ready):
    import torch

    from seqtree_b200 import device
    from seqtree_b200.learned import Encoder, pad_codes
    rng = np.random.default_rng(9)
    seqs = cdr3(rng, 300, 8, 25) + ["C", "CASSLGQGAYEQYFCASSLGQGAYEQYFWWW"]
    flat = oenc.init_params(11)
    enc = Encoder(flat)
    ss = device.SeqSet(seqs, "aa")
    z32 = torch.empty((len(seqs), 64), dtype=torch.float32, device="cuda")
    zbf = torch.empty((len(seqs), 64), dtype=torch.bfloat16, device="cuda")
    enc.embed_into(ss, z32.data_ptr(), 0, torch.cuda.current_stream().cuda_stream)
    enc.embed_into(ss, zbf.data_ptr(), 1, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    codes, lens = pad_codes(seqs)
    want = oenc.forward(flat.astype(np.float64), codes, lens)
    np.testing.assert_allclose(z32.cpu().numpy(), want, atol=2e-5)
    # layout 1: row r's 16-byte chunk c sits at chunk c ^ (r & 7)
    raw = zbf.float().cpu().numpy().reshape(len(seqs), 8, 8)
    rows = np.arange(len(seqs))[:, None]
    unswz = raw[rows, np.arange(8)[None, :] ^ (rows & 7)].reshape(len(seqs), 64)
    np.testing.assert_allclose(unswz, want, atol=8e-3)
    with pytest.raises(ValueError, match="1..32 residues"):
        enc.embed_into(device.SeqSet(["C" * 33], "aa"), z32.data_ptr(), 0)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [300, 40000])
def test_bf16_inference_tracks_the_fp32_forward(cuda_ready, n):
    """The bf16 tensor-core embedding (layout 1) against the float64 forward: bf16 activations
    with fp32 accumulation, so a tolerance -- every row within 0.03 per component and cosine
    >= 0.998 to the exact unit vector.  40,000 sequences span two 32,768-sequence passes."""
    import torch

    from seqtree_b200 import device
    from seqtree_b200.learned import Encoder, pad_codes
    rng = np.random.default_rng(n)
    seqs = cdr3(rng, n - 3, 8, 25) + ["C", "CASSLGQGAYEQYFCASSLGQGAYEQYFWWW", "WY"]
    flat = (oenc.init_params(3) + rng.normal(0, 0.02, oenc.param_count())).astype(np.float32)
    enc = Encoder(flat)
    ss = device.SeqSet(seqs, "aa")
    zbf = torch.empty((len(seqs), 64), dtype=torch.bfloat16, device="cuda")
    enc.embed_into(ss, zbf.data_ptr(), 1, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    raw = zbf.float().cpu().numpy().reshape(len(seqs), 8, 8)
    rows = np.arange(len(seqs))[:, None]
    got = raw[rows, np.arange(8)[None, :] ^ (rows & 7)].reshape(len(seqs), 64)
    check = np.arange(len(seqs)) if n <= 1000 else np.r_[np.arange(500), np.arange(n - 500, n),
                                                           rng.integers(0, n, 500)]
    codes, lens = pad_codes([seqs[i] for i in check])
    want = oenc.forward(flat.astype(np.float64), codes, lens)
    err = np.abs(got[check] - want).max(axis=1)
    cos = (got[check] * want).sum(1) / np.linalg.norm(got[check], axis=1)
    print(f"bf16 vs float64: max abs {err.max():.4f}, min cos {cos.min():.5f}")
    assert err.max() <= 0.03 and cos.min() >= 0.998


@pytest.mark.gpu
def test_training_lowers_the_loss(cuda_ready):
    from seqtree_b200.learned import Encoder, pad_codes, training_pairs
    rng = np.random.default_rng(1)
    a, b = training_pairs(3, 4096)
    m = SubstitutionMatrix.blosum62()
    pen = m.penalty_grid
    sc = np.array([oracle.gapblock_matrix([x], [y], pen, gap_open=8)[0, 0] for x, y in zip(a, b)],
                  np.int32)
    seqs = [s for pair in zip(a, b) for s in pair]
    codes, lens = pad_codes(seqs)
    enc = Encoder(seed=0)
    first = None
    for epoch in range(6):
        losses = []
        for i in range(0, len(seqs), 512):
            losses.append(enc.train_step(codes[i:i + 512], lens[i:i + 512], sc[i // 2:(i + 512) // 2],
                                         lr=1e-3))
        first = first if first is not None else np.mean(losses)
    assert np.mean(losses) < 0.5 * first
    assert np.all(np.isfinite(enc.params()))


@pytest.mark.gpu
def test_pair_scorer_matches_the_oracle(cuda_ready):
    import torch

    from seqtree_b200 import device
    from seqtree_b200.gapblock import central_prior, prior_cube
    from seqtree_b200.learned import pair_scores
    rng = np.random.default_rng(4)
    q, r = cdr3(rng, 70, 8, 25), cdr3(rng, 90, 8, 25) + ["C" * 70]
    qi = rng.integers(0, len(q), 5000).astype(np.int32)
    ri = rng.integers(0, len(r), 5000).astype(np.int32)
    m = SubstitutionMatrix.blosum62()
    width = 70
    cube = np.asarray(prior_cube(central_prior(21), width), np.int32).ravel()
    dense = oracle.gapblock_matrix(q, r, m.penalty_grid, gap_open=8, gap_extend=1, prior=cube,
                                   prior_width=width)
    qs, rs = device.SeqSet(q, "aa"), device.SeqSet(r, "aa")
    tq, tr = torch.from_numpy(qi).cuda(), torch.from_numpy(ri).cuda()
    out = torch.empty(5000, dtype=torch.int32, device="cuda")
    pair_scores(qs, rs, tq.data_ptr(), tr.data_ptr(), 5000, out.data_ptr(), matrix=m, gap_open=8,
                prior=cube, prior_width=width)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), dense[qi, ri])


@pytest.mark.gpu
def test_learned_search_is_exact_and_training_pays(cuda_ready):
    """End to end on 20,000 refs: every hit the learned search reports is an exhaustive hit with
    its exact score; with the calibrated fallback the recall bound holds on held-out queries;
    and on the cells the proposals answer alone (both junctions 11+ residues) the trained
    encoder recovers clearly more hits than the same network untrained."""
    import seqtree_b200 as stb
    from seqtree_b200 import learned as L
    M = stb.SubstitutionMatrix.blosum62()
    rc, rl = L.cdr3_codes(40, 20000)
    cc, cl = L.cdr3_codes(41, 3000)
    ec, el = L.cdr3_codes(42, 1500)

    def long_recall(enc):
        idx = L.LearnedIndex(enc, rc, rl, matrix=M, gap_open=8, max_penalty=24, k=64)
        idx.set_fallback()
        r = idx.recall(ec, el)
        assert r["subset_of_exact"]
        f, e = r["found_cells"][11:, 11:].sum(), r["exact_cells"][11:, 11:].sum()
        return f / e, idx

    untrained, _ = long_recall(L.Encoder(seed=0))
    enc = L.Encoder(seed=0)
    L.train(enc, 400_000, seed=3, matrix=M, gap_open=8)
    trained, idx = long_recall(enc)
    print(f"long x long recall at k=64 of 20,000 refs: untrained {untrained:.3f}, trained {trained:.3f}")
    assert trained > untrained + 0.15
    cal = idx.calibrate(cc, cl, bound=0.99)
    ev = idx.recall(ec, el)
    print("calibrated fallback", cal["query_fallback"], cal["ref_fallback"], "eval recall", ev["recall"])
    assert ev["subset_of_exact"] and ev["recall"] >= 0.99
    # The method without the network (k = 0: the calibrated exhaustive fallback alone), held to
    # the same bound on the same batch, has to score more pairs exhaustively.
    base = L.LearnedIndex(None, rc, rl, matrix=M, gap_open=8, max_penalty=24, k=0)
    bcal = base.calibrate(cc, cl, bound=0.99)
    bev = base.recall(ec, el)
    print("without the network:", bcal["query_fallback"], bcal["ref_fallback"],
          f"share {bcal['exhaustive_share']:.3f} vs {cal['exhaustive_share']:.3f}",
          "eval recall", bev["recall"])
    assert bev["subset_of_exact"] and bev["recall"] >= 0.99
    assert cal["exhaustive_share"] < bcal["exhaustive_share"]
    # The threshold form with the same trained encoder, calibrated to the same bound on the same
    # batch: exact hits, the bound met on the batch, and no more pairs scored exhaustively than
    # without the network (held-out recall is looser at this size: a cell holds few hits).
    thr = L.LearnedIndex(enc, rc, rl, matrix=M, gap_open=8, max_penalty=24, proposal="range")
    tcal = thr.calibrate(cc, cl, bound=0.99)
    tev = thr.recall(ec, el)
    print("threshold form:", tcal["query_fallback"], tcal["ref_fallback"],
          f"share {tcal['exhaustive_share']:.3f}", "cells", tcal["cells_with_proposals"],
          "eval recall", tev["recall"])
    assert tcal["subset_of_exact"] and tcal["recall"] >= 0.99
    assert tev["subset_of_exact"] and tev["recall"] >= 0.98
    assert tcal["exhaustive_share"] <= bcal["exhaustive_share"]


@pytest.mark.gpu
def test_model_file_gives_the_same_encoder_and_search(cuda_ready, tmp_path):
    """A trained encoder with its calibrated fallback, saved and loaded in a fresh index: the same
    weights bit for bit, the same settings, and the same search results."""
    import torch

    import seqtree_b200 as stb
    from seqtree_b200 import learned as L
    M = stb.SubstitutionMatrix.blosum62()
    enc = L.Encoder(seed=5)
    L.train(enc, 20000, seed=9, matrix=M, gap_open=8)
    rc, rl = L.cdr3_codes(50, 3000)
    qc, ql = L.cdr3_codes(51, 300)
    idx = L.LearnedIndex(enc, rc, rl, matrix=M, gap_open=8, max_penalty=24, k=64)
    idx.set_fallback([8, 9], [8])
    path = tmp_path / "model.stbe"
    idx.save_model(path)
    idx2 = L.LearnedIndex.from_model(path, rc, rl, matrix=M)
    assert idx2.encoder.params().tobytes() == enc.params().tobytes()
    assert (idx2.k, idx2.max_penalty, idx2.gap_open, idx2.gap_extend) == (64, 24, 8, 1)
    assert np.array_equal(idx2.query_fallback, idx.query_fallback)
    assert np.array_equal(idx2.ref_fallback, idx.ref_fallback)
    a = idx.search(idx.queries(qc, ql))
    b = idx2.search(idx2.queries(qc, ql))
    assert all(torch.equal(x, y) for x, y in zip(a, b))
    with pytest.raises(ValueError, match="not a seqtree_b200 encoder file"):
        (tmp_path / "junk").write_bytes(b"not a model")
        L.Encoder.load(tmp_path / "junk")
