"""The hand-written tcgen05 BF16 GEMM (FP32 accumulation in tensor memory) against a torch FP32
product of the same BF16 inputs.  Products of BF16 values are exact in FP32; only the summation
order differs, so the bar is 1e-5 of the sum of |terms|."""
import pytest

import patchtable_b200 as ptb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (128, 16, 16), (300, 32, 96), (256, 256, 128), (128, 128, 8192),
                                   (1000, 64, 48)])
def test_tc_gemm_matches_torch(gpu, M, N, K):
    import torch
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).to(gpu)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).to(gpu)
    C = torch.full((M, N), float("nan"), dtype=torch.float32, device=gpu)
    err = torch.zeros(1, dtype=torch.int32, device=gpu)
    st = ptb.lib().pt_tc_gemm_f32(A.data_ptr(), K, B.data_ptr(), K, C.data_ptr(), N, M, N, K, err.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    assert st == 0, ptb.lib().pt_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.float() @ B.float().T
    mag = A.float().abs() @ B.float().abs().T
    assert torch.all((C - ref).abs() <= 1e-5 * mag + 1e-30)
