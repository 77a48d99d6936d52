"""The tcgen05 BF16 GEMM against torch's FP32 matmul of the same BF16 operands.

BF16 inputs are exact in FP32, so the only differences are FP32 accumulation order: relative
1e-4 of the largest |D| entry.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K,splits", [(128, 32, 64, 1), (200, 64, 192, 1), (300, 96, 576, 1),
                                          (1000, 256, 320, 1), (257, 130, 1024, 4), (64, 200, 4096, 8)])
def test_gemm_matches_fp32_reference(M, N, K, splits):
    from meeuuw_b200 import ops
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    D = ops.gemm_bf16_tn(A, B, bias=bias, splits=splits, err=err)
    ref = A.float() @ B.float().T + bias
    assert int(err.item()) == 0
    assert (D - ref).abs().max().item() <= 1e-4 * ref.abs().max().item()


def test_gemm_bf16_relu_epilogue():
    from meeuuw_b200 import ops
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(384, 128, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(64, 128, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(64, device="cuda", generator=g)
    D = ops.gemm_bf16_tn(A, B, bias=bias, relu=True, out_bf16=True)
    ref = torch.relu(A.float() @ B.float().T + bias)
    assert D.dtype == torch.bfloat16
    assert (D.float() - ref).abs().max().item() <= 1e-2 * ref.abs().max().item()
