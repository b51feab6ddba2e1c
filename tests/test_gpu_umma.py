"""The tcgen05 building blocks (D = A B^T, BF16 in shared memory, FP32 in
tensor memory) against an FP32 matmul of the same BF16 values."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(16, 16), (64, 64), (256, 128), (128, 256), (208, 48)])
def test_umma_gemm_matches_fp32_matmul(N, K):
    import torch
    from chemgen_b200.runtime import lib
    g = torch.Generator(device="cuda").manual_seed(N * 1000 + K)
    A = torch.randn(128, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    D = torch.full((128, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib().chemgen_probe_umma(A.data_ptr(), B.data_ptr(), D.data_ptr(), N, K, err.data_ptr()) == 0
    assert err.item() == 0
    ref = A.float() @ B.float().T
    assert torch.allclose(D, ref, rtol=1e-5, atol=1e-4), (D - ref).abs().max().item()
