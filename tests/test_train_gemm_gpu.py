"""The encoder's bf16 tensor-core training GEMM (``st_train_gemm_bf16``) against a PyTorch
float64 product of the same bf16-rounded operands.  The kernel accumulates in fp32, so the bound
is fp32 rounding of the K-term sums, |got - want| <= (1e-5 + 1e-8 K) (|A| |B|)[i, j], far below
what a misplaced tile, chunk or K slice would cost.  The shapes cover ragged edges (M, N, K not
multiples of the 128 x 128 x 64 tile), both transposes, accumulation and the split-K path
(atomic adds of K slices)."""
from __future__ import annotations

import pytest

CASES = [
    # M, N, K, trans_a, trans_b, accumulate
    (1, 1, 1, False, False, False),
    (130, 70, 200, False, False, False),
    (300, 128, 384, False, True, True),
    (131, 257, 129, True, False, False),
    (128, 384, 40_000, True, False, True),   # split-K, accumulate into C
    (64, 64, 5_000, True, True, False),      # split-K, cleared first
    (4096, 384, 128, False, False, False),
    (2, 3, 0, False, False, False),          # K = 0: C = 0
]


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K,ta,tb,acc", CASES)
def test_train_gemm_matches_a_float64_product_of_bf16_operands(cuda_ready, M, N, K, ta, tb, acc):
    import torch

    from seqtree_b200.learned import train_gemm_bf16
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    a = torch.randn((K, M) if ta else (M, K), device="cuda", generator=g)
    b = torch.randn((N, K) if tb else (K, N), device="cuda", generator=g)
    c0 = torch.randn((M, N), device="cuda", generator=g)
    c = c0.clone()
    train_gemm_bf16(a, b, c, trans_a=ta, trans_b=tb, accumulate=acc)
    torch.cuda.synchronize()
    A = a.bfloat16().double()
    B = b.bfloat16().double()
    A = A.t() if ta else A
    B = B.t() if tb else B
    want = A @ B + (c0.double() if acc else 0)
    mag = A.abs() @ B.abs() + (c0.double().abs() if acc else 0)
    err = (c.double() - want).abs()
    bound = (1e-5 + 1e-8 * K) * mag
    assert bool((err <= bound).all()), float((err - bound).max())


@pytest.mark.gpu
def test_train_gemm_rejects_bad_shapes(cuda_ready):
    import torch

    from seqtree_b200.learned import train_gemm_bf16
    a = torch.zeros((4, 5), device="cuda")
    b = torch.zeros((6, 7), device="cuda")
    with pytest.raises(ValueError, match="chain"):
        train_gemm_bf16(a, b, torch.zeros((4, 7), device="cuda"))
    with pytest.raises(ValueError, match="fp32"):
        train_gemm_bf16(a.double(), b, torch.zeros((4, 7), device="cuda"))
