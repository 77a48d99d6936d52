"""Warm-start network on the device against the FP32 CPU reference: forward values, MSE loss and
every parameter gradient; the field <-> network-grid maps; a few Adam steps lower the loss."""
import numpy as np
import pytest
import torch

from oracle import unet as ounet

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("base,levels,B,H,W", [(8, 3, 2, 32, 32), (32, 4, 1, 64, 48)])
def test_forward_loss_gradients_match_fp32_reference(base, levels, B, H, W):
    from meeuuw_b200.unet import UNet
    net = UNet(base=base, levels=levels, seed=1)
    for l in net.layers():         # non-zero biases exercise the bias gradient path
        l.b.copy_(torch.randn(l.cout, generator=torch.Generator().manual_seed(l.cout)) * 0.05)
    g = torch.Generator().manual_seed(3)
    x = torch.rand(B, H, W, 2, generator=g).to(torch.bfloat16)
    t = torch.randn(B * H * W, 5, generator=g)
    y = net.forward(x.cuda(), B, H, W)
    dy, part = net.mse(y, t.cuda())
    net.backward(dy)
    torch.cuda.synchronize()
    loss = float(part.sum().item()) / t.numel()
    ref_layers = [dict(w=l.w16.float().cpu(), b=l.b.cpu(), cin=l.cin, cout=l.cout, relu=l.relu) for l in net.layers()]
    y_ref, loss_ref, grads = ounet.loss_and_grads(ref_layers, x.float(), t, levels)
    # forward: identical bf16 roundings, differences from accumulation order only
    assert _rel(y.cpu(), y_ref) < 5e-3
    assert abs(loss - loss_ref) <= 5e-3 * loss_ref
    # gradients: the device path feeds bf16 gradients to the tensor-core GEMMs
    for i, (l, (gw, gb)) in enumerate(zip(net.layers(), grads)):
        k = 9 * l.cin
        ew = _rel(l.gw.cpu()[:, :k], gw[:, :k])
        eb = _rel(l.gb.cpu(), gb)
        assert ew < 3e-2 and eb < 3e-2, (i, ew, eb)
        assert float(l.gw[:, k:].abs().max().item() if l.kp > k else 0.0) == 0.0


def test_adam_steps_lower_the_loss():
    from meeuuw_b200.unet import UNet
    net = UNet(base=8, levels=3, seed=2)
    B, H, W = 4, 32, 32
    g = torch.Generator().manual_seed(5)
    xx = torch.linspace(0, 1, W)
    zz = torch.linspace(0, 1, H)
    x = torch.stack(torch.broadcast_tensors(xx[None, :], zz[:, None]), -1)[None].repeat(B, 1, 1, 1)
    x = (x + 0.1 * torch.rand(B, H, W, 2, generator=g)).to(torch.bfloat16).cuda()
    t = torch.sin(3 * x.float()).sum(-1, keepdim=True).repeat(1, 1, 1, 5).reshape(-1, 5).contiguous()
    losses = []
    for _ in range(40):
        y = net.forward(x, B, H, W)
        dy, part = net.mse(y, t)
        losses.append(float(part.sum().item()) / t.numel())
        net.backward(dy)
        net.step(lr=3e-3)
    assert losses[-1] < 0.25 * losses[0], losses


def test_targets_to_fields_reproduce_centre_values():
    """to_fields(targets(solution)) at f = 1 is exact at the element centres (bilinear between
    centres); the RMS scales travel through the two log-scale channels; the hydrostatic part is
    carried analytically."""
    from meeuuw_b200 import _lib as L
    from meeuuw_b200.unet import features_targets, pressure_scales
    n = 16
    box = L.box_of(n, n, 1.0, 1.0)
    nnx = 2 * n + 1
    rng = np.random.default_rng(0)
    x = np.tile(np.arange(nnx) / (nnx - 1), nnx)
    z = np.repeat(np.arange(nnx) / (nnx - 1), nnx)
    solV = np.empty(2 * nnx * nnx)
    solV[0::2] = 3e4 * np.sin(np.pi * x) * np.cos(np.pi * z)
    solV[1::2] = -3e4 * np.cos(np.pi * x) * np.sin(np.pi * z)
    px = np.tile(np.arange(n + 1) / n, n + 1)
    pz = np.repeat(np.arange(n + 1) / n, n + 1)
    Ra, alphaT = 1e5, 1e-2
    pscale, ghyd = pressure_scales(Ra, alphaT)
    solP = ghyd * (0.5 - pz) + Ra * 0.3 * px * pz
    T = rng.uniform(0, 1, nnx * nnx)
    eta = np.exp(rng.normal(0, 1, n * n))
    d = lambda a: torch.as_tensor(a).cuda()
    scales = torch.empty(2, dtype=torch.float64, device="cuda")
    X, Y, stats = features_targets(box, d(T), d(eta), Ra, alphaT, 1, d(solV), d(solP), scales=scales)
    Yh = Y.cpu().numpy().reshape(n * n, 5)
    assert np.allclose(np.sqrt(np.mean(0.5 * (Yh[:, 0] ** 2 + Yh[:, 1] ** 2))), 1.0, rtol=1e-6)
    assert np.allclose(np.sqrt(np.mean(Yh[:, 2] ** 2)), 1.0, rtol=1e-6)
    sc = scales.cpu().numpy()
    assert np.allclose(Yh[:, 3], np.log10(sc[0]), rtol=1e-6) and np.allclose(Yh[:, 4], np.log10(sc[1]), rtol=1e-6)
    fix = torch.zeros(2 * nnx * nnx, dtype=torch.uint8, device="cuda")
    V2 = torch.empty(2 * nnx * nnx, dtype=torch.float64, device="cuda")
    P2 = torch.empty((n + 1) ** 2, dtype=torch.float64, device="cuda")
    yflat = Y.reshape(-1, 5).contiguous()
    pred = torch.empty(2, dtype=torch.float64, device="cuda")
    L.call("mw_unet_to_fields", box, 1, L.ptr(yflat), L.ptr(stats), pscale, ghyd, L.ptr(pred), L.ptr(fix),
           L.ptr(V2), L.ptr(P2), L.stream_ptr())
    assert np.allclose(pred.cpu().numpy(), sc, rtol=1e-5)
    V2 = V2.cpu().numpy()
    ix, iz = np.meshgrid(np.arange(1, nnx, 2), np.arange(1, nnx, 2))
    centre = (iz * nnx + ix).ravel()
    vmax = np.abs(solV).max()
    np.testing.assert_allclose(V2[2 * centre], solV[2 * centre], rtol=1e-5, atol=1e-5 * vmax)
    np.testing.assert_allclose(V2[2 * centre + 1], solV[2 * centre + 1], rtol=1e-5, atol=1e-5 * vmax)
    # features: T at the centres and the scaled log-viscosity
    Xc = X.float().cpu().numpy().reshape(n, n, 2)
    np.testing.assert_allclose(Xc[..., 0].ravel(), T[centre], atol=4e-3)
    le = np.log10(eta)
    np.testing.assert_allclose(Xc[..., 1].ravel(), (le - le.mean()) / 2.5, atol=1e-2)
    st = stats.cpu().numpy()
    assert abs(st[0] - le.mean()) < 1e-12 and abs(st[1] / (Ra / 10 ** le.mean()) - 1) < 1e-12
    # interior pressure nodes: bilinear of a bilinear field is exact away from the clamped border
    P2 = P2.cpu().numpy().reshape(n + 1, n + 1)
    Pr = solP.reshape(n + 1, n + 1)
    np.testing.assert_allclose(P2[2:-2, 2:-2], Pr[2:-2, 2:-2], rtol=1e-6, atol=1e-6 * ghyd)
