"""Tensor-core (tcgen05) kernels of the learned subgrid-stress closure against
torch float32 references of the same operations (bf16 operands are exact in
float32; only the accumulation order differs)."""
import importlib

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nat():
    return importlib.import_module("3dhit_b200._native")


@pytest.mark.parametrize("M,N,K", [(300, 64, 80), (128, 16, 16), (1000, 128, 64), (257, 32, 144)])
def test_tc_gemm_bf16(nat, M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.full((M, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.call("hit_tc_gemm_bf16", nat.ptr(A), K, nat.ptr(B), K, nat.ptr(C), N, M, N, K, nat.ptr(err),
             nat.stream_ptr(A.device))
    ref = A.float() @ B.float().T
    assert int(err.item()) == 0
    assert torch.allclose(C, ref, rtol=1e-5, atol=1e-4 * float(ref.abs().max()))
