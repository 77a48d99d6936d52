"""The CPU reference of the warm-start network: its weight layout against an explicit im2col
product, and its autograd gradients against central finite differences (float64)."""
import numpy as np
import torch

from oracle import unet as ounet


def _layers(base, levels, cin=2, cout=3, seed=0, dtype=torch.float64):
    g = torch.Generator().manual_seed(seed)
    chans = [base * 2 ** i for i in range(levels)]
    spec = []
    c = cin
    for k in chans:
        spec += [(c, k, True), (k, k, True)]
        c = k
    for k in reversed(chans[:-1]):
        spec += [(c + k, k, True), (k, k, True)]
        c = k
    spec.append((c, cout, False))
    out = []
    for ci, co, relu in spec:
        kp = int(np.ceil(9 * ci / 64) * 64)
        w = torch.zeros(co, kp, dtype=dtype)
        w[:, :9 * ci] = torch.randn(co, 9 * ci, generator=g, dtype=dtype) * np.sqrt(2.0 / (9 * ci))
        b = torch.randn(co, generator=g, dtype=dtype) * 0.1
        out.append(dict(w=w, b=b, cin=ci, cout=co, relu=relu))
    return out


def test_weight_layout_matches_explicit_im2col():
    g = torch.Generator().manual_seed(1)
    B, H, W, C, Co = 2, 5, 7, 3, 4
    x = torch.randn(B, H, W, C, generator=g, dtype=torch.float64)
    kp = 64
    w = torch.zeros(Co, kp, dtype=torch.float64)
    w[:, :9 * C] = torch.randn(Co, 9 * C, generator=g, dtype=torch.float64)
    col = np.zeros((B * H * W, kp))
    xn = x.numpy()
    for b in range(B):
        for y in range(H):
            for xx in range(W):
                p = (b * H + y) * W + xx
                for tap in range(9):
                    yy, xs = y + tap // 3 - 1, xx + tap % 3 - 1
                    if 0 <= yy < H and 0 <= xs < W:
                        col[p, tap * C:(tap + 1) * C] = xn[b, yy, xs]
    ref = col @ w.numpy().T
    got = torch.nn.functional.conv2d(x.permute(0, 3, 1, 2), ounet.conv_weight(w, C, Co), padding=1)
    np.testing.assert_allclose(got.permute(0, 2, 3, 1).reshape(-1, Co).numpy(), ref, rtol=1e-12, atol=1e-12)


def test_gradients_match_finite_differences():
    levels, base = 2, 2
    layers = _layers(base, levels)
    g = torch.Generator().manual_seed(2)
    x = torch.rand(1, 4, 4, 2, generator=g, dtype=torch.float64)
    t = torch.randn(16, 3, generator=g, dtype=torch.float64)
    _, loss, grads = ounet.loss_and_grads(layers, x, t, levels, round_bf16=False)
    rng = np.random.default_rng(3)
    h = 1e-6
    for li in (0, 3, len(layers) - 1):
        for which in (0, 1):
            key = "w" if which == 0 else "b"
            p = layers[li][key].detach()
            if which == 0:
                idx = (int(rng.integers(p.shape[0])), int(rng.integers(9 * layers[li]["cin"])))
            else:
                idx = (int(rng.integers(p.shape[0])),)
            vals = []
            for s in (1, -1):
                pert = [dict(l) for l in layers]
                q = p.clone()
                q[idx] += s * h
                pert[li][key] = q
                y = ounet.forward(pert, x, levels, round_bf16=False)
                vals.append(float(((y - t) ** 2).mean()))
            fd = (vals[0] - vals[1]) / (2 * h)
            an = float(grads[li][which][idx])
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (li, key, idx, fd, an)
