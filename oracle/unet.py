"""FP32 CPU reference of the warm-start U-Net (test infrastructure only: never imported by the
library).  It restates the network the device path builds from im2col + tensor-core GEMMs with
torch's CPU conv2d and autograd, so the device forward pass, the loss and every parameter gradient
can be checked against an independent computation.

The reference code has no learned component; this network is an addition of the device path, so
the checks here are numerical (same weights, same inputs) rather than pinned to reference fixtures.

Layout conventions shared with the device path:
  * activations NHWC; the network input has 2 channels (T, scaled log10 viscosity);
  * conv weights [Cout, Kp] with column k = tap * Cin + c, tap = (dy + 1) * 3 + (dx + 1), columns
    >= 9 * Cin zero padding;
  * conv outputs (bias + ReLU applied in FP32) and pooled activations are stored as BF16; the
    head's output stays FP32.  ``round_bf16`` mirrors those roundings with a straight-through
    gradient, so the forward values agree to accumulation order.
"""
import torch
import torch.nn.functional as F


def conv_weight(w, cin, cout):
    """[Cout, Kp] (k = tap * Cin + c) -> conv2d weight [Cout, Cin, 3, 3]."""
    return w[:, :9 * cin].reshape(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous()


def _rb(t, on):
    if not on:
        return t
    return t + (t.to(torch.bfloat16).to(torch.float32) - t).detach()


def forward(layers, x, levels, round_bf16=True):
    """layers: list of dicts {w [Cout, Kp] fp32 (leaf), b [Cout] fp32 (leaf), cin, cout, relu} in the
    device order (encoder pairs, decoder pairs, head).  x: [B, H, W, 2] fp32.  Returns
    y [B*H*W, 3] fp32 (NHWC rows)."""
    def conv(l, a):
        z = F.conv2d(a, conv_weight(l["w"], l["cin"], l["cout"]), l["b"], padding=1)
        return F.relu(z) if l["relu"] else z

    a = x.permute(0, 3, 1, 2)
    it = iter(layers)
    skips = []
    for lvl in range(levels):
        c1, c2 = next(it), next(it)
        a = _rb(conv(c1, a), round_bf16)
        a = _rb(conv(c2, a), round_bf16)
        skips.append(a)
        if lvl < levels - 1:
            a = _rb(F.avg_pool2d(a, 2), round_bf16)
    for i in range(levels - 1):
        c1, c2 = next(it), next(it)
        up = F.interpolate(a, scale_factor=2, mode="nearest")
        a = torch.cat([up, skips[levels - 2 - i]], dim=1)
        a = _rb(conv(c1, a), round_bf16)
        a = _rb(conv(c2, a), round_bf16)
    head = next(it)
    y = conv(head, a)
    return y.permute(0, 2, 3, 1).reshape(-1, head["cout"])


def loss_and_grads(layers, x, target, levels, round_bf16=True):
    """MSE = mean((y - target)^2) and d MSE / d (w, b) of every layer (weights as [Cout, Kp])."""
    for l in layers:
        l["w"] = l["w"].detach().clone().requires_grad_(True)
        l["b"] = l["b"].detach().clone().requires_grad_(True)
    y = forward(layers, x, levels, round_bf16)
    loss = ((y - target) ** 2).mean()
    loss.backward()
    return y.detach(), float(loss.detach()), [(l["w"].grad.clone(), l["b"].grad.clone()) for l in layers]
