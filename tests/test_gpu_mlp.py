"""The tcgen05 dense layer (bpf_dense_bf16) against a plain PyTorch FP32
matmul of the same BF16 operands: D = act(A B^T + bias) with FP32
accumulation; only the order of the K-sum differs."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dense(A, a_rs, a_cs, B, b_rs, b_cs, M, N, K, bias=None, relu=0, want_h=False):
    import torch
    from libbi_b200 import _native as N_

    Df = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    Dh = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda") if want_h else None
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = N_.lib().bpf_dense_bf16(A.data_ptr(), a_rs, a_cs, B.data_ptr(), b_rs, b_cs, M, N, K,
                                 None if bias is None else bias.data_ptr(), relu, Df.data_ptr(), N,
                                 None if Dh is None else Dh.data_ptr(), N, err.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return Df, Dh


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (128, 80, 80), (300, 128, 128), (1000, 80, 128), (256, 256, 1000),
                                   (77, 16, 40)])
def test_dense_matches_torch(cuda, M, N, K):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(M * 7 + N + K)
    A = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    W = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    b = torch.randn(N, generator=g, device="cuda")
    D, Dh = _dense(A, K, 1, W, K, 1, M, N, K, b, 1, want_h=True)
    ref = torch.relu(A.float() @ W.float().T + b)
    tol = 1e-5 * np.sqrt(K) * float(ref.abs().max())
    assert float((D - ref).abs().max()) <= tol
    np.testing.assert_array_equal(Dh.cpu().float().numpy(), D.to(torch.bfloat16).cpu().float().numpy())


def test_dense_transposed_operands(cuda):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    M, N, K = 200, 96, 700
    At = torch.randn((K, M), generator=g, device="cuda").to(torch.bfloat16)  # A stored transposed
    Bt = torch.randn((K, N), generator=g, device="cuda").to(torch.bfloat16)
    D, _ = _dense(At, 1, M, Bt, 1, N, M, N, K)
    ref = At.float().T @ Bt.float()
    assert float((D - ref).abs().max()) <= 1e-5 * np.sqrt(K) * float(ref.abs().max())
