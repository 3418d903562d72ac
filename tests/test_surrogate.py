"""Tensor-core (tcgen05) kernels of the learned surrogate against torch."""
import ctypes

import pytest
import torch

import agbnp3_b200 as A


def _lib():
    L = A.lib()
    L.agbnp3_tc_gemm.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                 ctypes.c_void_p] + [ctypes.c_int] * 4 + [ctypes.c_void_p]
    return L


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K,lda", [(128, 16, 16, 16), (300, 128, 160, 160), (257, 128, 128, 136), (64, 2, 128, 128),
                                       (1000, 256, 256, 256), (128, 160, 4096, 4096), (5, 7, 48, 48)])
def test_tc_gemm_matches_torch(M, N, K, lda):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    Abuf = torch.randn(M, lda, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(N, device="cuda", generator=g)
    C = torch.full((M, N), float("nan"), device="cuda")
    torch.cuda.synchronize()
    assert _lib().agbnp3_tc_gemm(_p(Abuf), lda, _p(B), K, _p(b), _p(C), N, M, N, K, None) == 0
    ref = Abuf[:, :K].float() @ B.float().T + b
    assert torch.allclose(C, ref, rtol=1e-4, atol=1e-3 * (K / 128) ** 0.5), (C - ref).abs().max().item()
