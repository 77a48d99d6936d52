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


@pytest.mark.parametrize("B,H,W,C,N", [(1, 16, 16, 32, 32), (2, 32, 32, 64, 64), (1, 64, 64, 96, 32),
                                       (1, 128, 128, 32, 5), (2, 16, 16, 384, 128), (1, 32, 32, 256, 256),
                                       (1, 64, 64, 192, 64), (3, 16, 16, 128, 200)])
def test_implicit_conv_equals_im2col_gemm(B, H, W, C, N):
    """mw_conv3x3_bf16 (A tiles by 4D TMA per tap, zero fill at the image borders) against
    mw_unet_im2col + mw_gemm_bf16_tn: the same K blocks and MMAs in the same order, so the FP32
    outputs are equal bit for bit; also against torch's FP32 convolution of the same operands."""
    from meeuuw_b200 import ops
    from meeuuw_b200._lib import call, ptr, stream_ptr
    from meeuuw_b200.unet import _kp
    import meeuuw_b200.unet  # noqa: F401  (registers mw_unet_im2col)
    g = torch.Generator(device="cuda").manual_seed(B * 1000 + H * 10 + C + N)
    X = torch.randn(B * H * W, C, device="cuda", generator=g).to(torch.bfloat16)
    kp = _kp(C)
    Wt = torch.zeros(N, kp, device="cuda", dtype=torch.bfloat16)
    Wt[:, :9 * C] = (torch.randn(N, 9 * C, device="cuda", generator=g) / (3 * C ** 0.5)).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    D = ops.conv3x3_bf16(X, B, H, W, C, Wt, bias=bias, err=err)
    col = torch.empty(B * H * W, kp, device="cuda", dtype=torch.bfloat16)
    call("mw_unet_im2col", B, H, W, C, kp, 0, 0, ptr(X), ptr(col), stream_ptr())
    R = ops.gemm_bf16_tn(col, Wt, bias=bias)
    assert int(err.item()) == 0
    assert torch.equal(D, R)
    # torch: weights [N, 9C] with K = (3 dy + dx) C + c -> [N, C, 3, 3]
    w4 = Wt[:, :9 * C].float().view(N, 3, 3, C).permute(0, 3, 1, 2)
    x4 = X.float().view(B, H, W, C).permute(0, 3, 1, 2)
    ref = torch.nn.functional.conv2d(x4, w4, bias=bias, padding=1).permute(0, 2, 3, 1).reshape(B * H * W, N)
    assert (D - ref).abs().max().item() <= 1e-4 * ref.abs().max().item()


def test_implicit_conv_bf16_relu_and_refusals():
    from meeuuw_b200 import ops
    g = torch.Generator(device="cuda").manual_seed(11)
    X = torch.randn(32 * 32, 64, device="cuda", generator=g).to(torch.bfloat16)
    Wt = (torch.randn(64, 576, device="cuda", generator=g) / 24).to(torch.bfloat16)
    D = ops.conv3x3_bf16(X, 1, 32, 32, 64, Wt, relu=True, out_bf16=True)
    assert D.dtype == torch.bfloat16 and float(D.float().min()) >= 0.0
    assert not ops.conv3x3_ok(2, 128, 128) and not ops.conv3x3_ok(32, 8, 8) and ops.conv3x3_ok(32, 16, 16)
    with pytest.raises(RuntimeError):
        ops.conv3x3_bf16(X[:, :48].contiguous(), 1, 32, 32, 48, Wt[:, :432].contiguous())


def test_unet_implicit_equals_im2col():
    """The whole U-Net forward and backward with implicit convolutions and with im2col everywhere:
    equal outputs and weight gradients."""
    import meeuuw_b200.unet as U
    net = U.UNet(seed=3)
    g = torch.Generator(device="cuda").manual_seed(2)
    X = torch.randn(2, 64, 64, 2, device="cuda", generator=g).to(torch.bfloat16)
    T = torch.randn(2 * 64 * 64, U.NOUT, device="cuda", generator=g)
    res = {}
    for imp in (True, False):
        U.IMPLICIT = imp
        try:
            y = net.forward(X, 2, 64, 64).clone()
            dy, _ = net.mse(y, T)
            for l in net.layers():
                l.gw.zero_()
                l.gb.zero_()
            net.backward(dy)
            res[imp] = (y, [l.gw.clone() for l in net.layers()])
        finally:
            U.IMPLICIT = True
    assert torch.equal(res[True][0], res[False][0])
    for a, b in zip(res[True][1], res[False][1]):
        assert torch.equal(a, b)
