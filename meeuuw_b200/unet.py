"""Learned warm start: a 4-level U-Net mapping (T, log10 eta) to a Stokes initial guess (u, w, p).

Every convolution is a GEMM on this library's tcgen05 BF16 kernels (FP32 accumulation):
forward  A = conv(X):   out[M, Cout]  = im2col(X)[M, Kp]    . W[Cout, Kp]^T
data grad dX:           dX[M, Cin]    = im2col(dZ)[M, Kp']  . Wflip[Cin, Kp']^T
weight grad dW:         dW[Cout, Kp]  = dZ^T[Cout, M]       . im2col(X)^T[Kp, M]^T   (split-K)
The first two are implicit GEMMs (mw_conv3x3_bf16: each K block's tile loaded from the NHWC
activations by TMA at the tap's offset) wherever the input has a multiple of 32 channels; the
2-channel input layer, the 5-channel head's data gradient and the weight gradients use an
im2col matrix.
Activations are NHWC BF16, gradients FP32, master weights FP32 with Adam.  The network's
arithmetic is the library's kernels; torch allocates buffers and gathers training batches.

The network is trained on snapshots of the device time stepper (Frank-Kamenetskii convection, Ra
and contrast log-uniform, random smooth initial temperatures), in the units of
``mw_unet_features`` / ``mw_unet_targets``: velocity / (Ra / geometric-mean viscosity) and the
dynamic pressure / Ra, each normalised by its RMS over the grid, plus the two log10 RMS scales as
extra output channels.  At run time ``LearnedGuess`` proposes guesses and the solver starts from
whichever has the smallest Uzawa residual, the previous step's solution included.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib as L
from .ops import conv3x3_bf16, conv3x3_ok, gemm_bf16_tn, workspace
from ._lib import c_double, c_int32, c_int64, c_void_p, call, ptr, stream_ptr

bf16, f32 = torch.bfloat16, torch.float32
# output channels: u / sv, w / sv, dynamic p / sp, log10 sv, log10 sp (sv, sp: RMS scales of the
# velocity and of the dynamic pressure, so every channel is O(1) for any Ra and viscosity contrast)
NOUT = 5

L.extra_protos({
    "mw_unet_im2col": (c_int32, [c_int32] * 6 + [c_int64] + [c_void_p] * 3),
    "mw_unet_cast_bf16": (c_int32, [c_int64, c_void_p, c_void_p, c_void_p]),
    "mw_unet_weights_bwd": (c_int32, [c_int32] * 4 + [c_void_p] * 3),
    "mw_unet_relu_grad": (c_int32, [c_int64, c_int32, c_int32, c_int64] + [c_void_p] * 6),
    "mw_unet_colsum": (c_int32, [c_int64, c_int32, c_void_p, c_void_p, c_void_p]),
    "mw_unet_avgpool2": (c_int32, [c_int32] * 4 + [c_void_p] * 3),
    "mw_unet_avgpool2_bwd": (c_int32, [c_int32] * 4 + [c_void_p, c_void_p, c_int32, c_void_p]),
    "mw_unet_upsample2_into": (c_int32, [c_int32] * 6 + [c_void_p] * 3),
    "mw_unet_copy_channels": (c_int32, [c_int64, c_int32, c_int32, c_int32] + [c_void_p] * 3),
    "mw_unet_upsample2_bwd": (c_int32, [c_int32] * 6 + [c_void_p] * 3),
    "mw_unet_slice_grad": (c_int32, [c_int64, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_int32, c_void_p]),
    "mw_unet_mse": (c_int32, [c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p]),
    "mw_unet_adam": (c_int32, [c_int64, c_void_p, c_void_p, c_void_p, c_void_p] + [ctypes.c_float] * 6 +
                     [c_void_p, c_void_p]),
    "mw_unet_features": (c_int32, [L.MwBox, c_int32, c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p]),
    "mw_unet_features_padded": (c_int32, [L.MwBox, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_double, c_void_p,
                                          c_void_p, c_void_p]),
    "mw_unet_to_fields_padded": (c_int32, [L.MwBox, c_int32, c_int32, c_void_p, c_void_p, c_double, c_double,
                                           c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_unet_to_fields": (c_int32, [L.MwBox, c_int32, c_void_p, c_void_p, c_double, c_double, c_void_p, c_void_p,
                                    c_void_p, c_void_p, c_void_p]),
    "mw_unet_targets": (c_int32, [L.MwBox, c_void_p, c_void_p, c_void_p, c_double, c_double, c_void_p, c_void_p,
                                  c_void_p]),
})


# 3x3 convolutions whose input channels are a multiple of 32 (and images 128-pixel bands) run as
# implicit GEMMs (ops.conv3x3_bf16, no im2col matrix); False forces im2col + GEMM everywhere
IMPLICIT = True


def _kp(c):
    return int(math.ceil(9 * c / 64.0) * 64)


class Conv:
    """3x3 'same' convolution (+ bias, optional ReLU) with FP32 master weights [Cout, Kp]."""

    def __init__(self, cin, cout, relu=True, gen=None):
        self.cin, self.cout, self.relu = cin, cout, relu
        self.kp, self.kpo = _kp(cin), _kp(cout)
        std = math.sqrt((2.0 if relu else 1.0) / (9 * cin))
        w = torch.zeros(cout, self.kp, dtype=f32)
        w[:, :9 * cin] = torch.randn(cout, 9 * cin, generator=gen) * std
        self.w = w.cuda()
        self.b = torch.zeros(cout, dtype=f32, device="cuda")
        self.gw, self.gb = torch.zeros_like(self.w), torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.w16 = torch.empty(cout, self.kp, dtype=bf16, device="cuda")
        self.wt16 = torch.empty(cin, self.kpo, dtype=bf16, device="cuda")
        self.refresh()

    def refresh(self):
        call("mw_unet_cast_bf16", self.w.numel(), ptr(self.w), ptr(self.w16), stream_ptr())

    def params(self):
        return [(self.w, self.gw, self.mw, self.vw, self.w16), (self.b, self.gb, self.mb, self.vb, None)]

    def forward(self, X, B, H, W, out_f32=False):
        if IMPLICIT and conv3x3_ok(self.cin, H, W):
            return conv3x3_bf16(X, B, H, W, self.cin, self.w16, bias=self.b, relu=self.relu, out_bf16=not out_f32)
        M = B * H * W
        col = _buf(("col", M, self.kp), (M, self.kp), bf16)
        call("mw_unet_im2col", B, H, W, self.cin, self.kp, 0, 0, ptr(X), ptr(col), stream_ptr())
        return gemm_bf16_tn(col, self.w16, bias=self.b, relu=self.relu, out_bf16=not out_f32)

    def backward(self, X, A, dA, B, H, W, need_dx=True):
        """X: input [M, cin] bf16, A: output [M, cout] (bf16, post-ReLU), dA: d loss / d A (fp32)."""
        M = B * H * W
        Mp = (M + 63) // 64 * 64      # pixel (contraction) dimension of the weight-gradient GEMM, zero padded
        dZ = _buf(("dZ", M, self.cout), (M, self.cout), bf16)
        dZT = _buf(("dZT", M, self.cout), (self.cout, Mp), bf16, zero=True)
        dZ32 = _buf(("dZ32", M, self.cout), (M, self.cout), f32)
        call("mw_unet_relu_grad", M, self.cout, int(self.relu), Mp, ptr(dA), ptr(A), ptr(dZ), ptr(dZT), ptr(dZ32),
             stream_ptr())
        call("mw_unet_colsum", M, self.cout, ptr(dZ32), ptr(self.gb), stream_ptr())
        colT = _buf(("colT", M, self.kp), (self.kp, Mp), bf16)
        call("mw_unet_im2col", B, H, W, self.cin, self.kp, 1, Mp, ptr(X), ptr(colT), stream_ptr())
        splits = max(1, min(64, Mp // 4096))
        gemm_bf16_tn(dZT, colT, out=self.gw, splits=splits)
        if not need_dx:
            return None
        call("mw_unet_weights_bwd", self.cout, self.cin, self.kp, self.kpo, ptr(self.w), ptr(self.wt16), stream_ptr())
        if IMPLICIT and conv3x3_ok(self.cout, H, W):
            return conv3x3_bf16(dZ, B, H, W, self.cout, self.wt16)
        colZ = _buf(("colZ", M, self.kpo), (M, self.kpo), bf16)
        call("mw_unet_im2col", B, H, W, self.cout, self.kpo, 0, 0, ptr(dZ), ptr(colZ), stream_ptr())
        return gemm_bf16_tn(colZ, self.wt16)


_bufs = {}


def _buf(key, shape, dtype, zero=False):
    """Scratch tensor reused across calls with the same key on the same stream (consumed in stream
    order; models advanced concurrently on different streams never share one)."""
    k = (key, dtype, torch.cuda.current_stream().cuda_stream)
    b = _bufs.get(k)
    if b is None or tuple(b.shape) != tuple(shape):
        b = (torch.zeros if zero else torch.empty)(shape, dtype=dtype, device="cuda")
        _bufs[k] = b
    return b


class UNet:
    """Encoder 2-32-64-128-256 (two convs per level, 2x2 average pooling), decoder with nearest
    upsampling and skip concatenation, 3x3 head to the NOUT output channels."""

    def __init__(self, base=32, levels=4, cin=2, cout=NOUT, seed=0):
        gen = torch.Generator().manual_seed(seed)
        ch = [base * 2 ** i for i in range(levels)]
        self.ch = ch
        self.enc = []
        c = cin
        for k in ch:
            self.enc.append((Conv(c, k, gen=gen), Conv(k, k, gen=gen)))
            c = k
        self.dec = []
        for k in reversed(ch[:-1]):
            self.dec.append((Conv(c + k, k, gen=gen), Conv(k, k, gen=gen)))
            c = k
        self.head = Conv(c, cout, relu=False, gen=gen)
        self.t = 0

    def layers(self):
        out = [l for pair in self.enc for l in pair] + [l for pair in self.dec for l in pair] + [self.head]
        return out

    # ---------------------------------------------------------------- forward
    def forward(self, X, B, H, W):
        """X: [B, H, W, 2] bf16 -> [B*H*W, NOUT] fp32.  Keeps the activations for backward."""
        st = {"B": B, "H": H, "W": W, "x": X, "enc": [], "dec": []}
        h, w, x = H, W, X
        for lvl, (c1, c2) in enumerate(self.enc):
            a1 = c1.forward(x, B, h, w)
            a2 = c2.forward(a1, B, h, w)
            st["enc"].append((x, a1, a2, h, w))
            if lvl < len(self.enc) - 1:
                p = _buf(("pool", lvl), (B * (h // 2) * (w // 2), c2.cout), bf16)
                call("mw_unet_avgpool2", B, h, w, c2.cout, ptr(a2), ptr(p), stream_ptr())
                x, h, w = p, h // 2, w // 2
            else:
                x = a2
        for i, (c1, c2) in enumerate(self.dec):
            skip_x, _, skip_a2, sh, sw = st["enc"][len(self.enc) - 2 - i]
            cup = self.enc[-1][1].cout if i == 0 else self.dec[i - 1][1].cout
            cskip = skip_a2.shape[1]
            cat = _buf(("cat", i), (B * sh * sw, cup + cskip), bf16)
            call("mw_unet_upsample2_into", B, h, w, cup, cup + cskip, 0, ptr(x), ptr(cat), stream_ptr())
            call("mw_unet_copy_channels", B * sh * sw, cskip, cup + cskip, cup, ptr(skip_a2), ptr(cat), stream_ptr())
            h, w = sh, sw
            a1 = c1.forward(cat, B, h, w)
            a2 = c2.forward(a1, B, h, w)
            st["dec"].append((cat, a1, a2, h, w, cup, cskip))
            x = a2
        y = self.head.forward(x, B, h, w, out_f32=True)
        st["head_in"] = x
        st["y"] = y
        self.st = st
        return y

    # ---------------------------------------------------------------- backward
    def backward(self, dy):
        st = self.st
        B = st["B"]
        h, w = st["H"], st["W"]
        g = self.head.backward(st["head_in"], st["y"], dy, B, h, w)
        nlev = len(self.enc)
        skip_grads = [None] * (nlev - 1)
        for i in range(len(self.dec) - 1, -1, -1):
            c1, c2 = self.dec[i]
            cat, a1, a2, h, w, cup, cskip = st["dec"][i]
            g = c2.backward(a1, a2, g, B, h, w)
            gcat = c1.backward(cat, a1, g, B, h, w)
            lvl = nlev - 2 - i
            gs = _buf(("gskip", lvl), (B * h * w, cskip), f32)
            call("mw_unet_slice_grad", B * h * w, cskip, cup + cskip, cup, ptr(gcat), ptr(gs), 0, stream_ptr())
            skip_grads[lvl] = gs
            gu = _buf(("gup", i), (B * (h // 2) * (w // 2), cup), f32)
            call("mw_unet_upsample2_bwd", B, h // 2, w // 2, cup, cup + cskip, 0, ptr(gcat), ptr(gu), stream_ptr())
            g = gu
        for lvl in range(nlev - 1, -1, -1):
            c1, c2 = self.enc[lvl]
            x, a1, a2, h, w = st["enc"][lvl]
            if lvl < nlev - 1:
                # gradient into a2: skip path + pooled path
                ga2 = _buf(("ga2", lvl), (B * h * w, c2.cout), f32)
                call("mw_unet_avgpool2_bwd", B, h, w, c2.cout, ptr(g), ptr(ga2), 0, stream_ptr())
                call("mw_unet_slice_grad", B * h * w, c2.cout, c2.cout, 0, ptr(skip_grads[lvl]), ptr(ga2), 1,
                     stream_ptr())
                g = ga2
            g = c2.backward(a1, a2, g, B, h, w)
            g = c1.backward(x, a1, g, B, h, w, need_dx=lvl > 0)

    def step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        bc1, bc2 = 1 - b1 ** self.t, 1 - b2 ** self.t
        for layer in self.layers():
            for p, gp, m, v, p16 in layer.params():
                call("mw_unet_adam", p.numel(), ptr(p), ptr(m), ptr(v), ptr(gp), lr, b1, b2, eps, bc1, bc2, ptr(p16),
                     stream_ptr())

    def mse(self, y, target):
        n = y.numel()
        dy = _buf(("dy", n), y.shape, f32)
        part = _buf(("loss", 64), (64,), torch.float64)
        call("mw_unet_mse", n, ptr(y), ptr(target), ptr(dy), ptr(part), 64, stream_ptr())
        return dy, part

    def save(self, path, **meta):
        """Weights as BF16 bit patterns (the precision the forward pass uses), biases FP32."""
        arrs = {"base": np.int32(self.ch[0]), "levels": np.int32(len(self.ch))}
        for k, v in meta.items():
            arrs["meta_" + k] = np.asarray(v)
        for i, l in enumerate(self.layers()):
            arrs[f"w{i}"] = l.w16[:, :9 * l.cin].contiguous().view(torch.int16).cpu().numpy()
            arrs[f"b{i}"] = l.b.cpu().numpy()
        np.savez_compressed(path, **arrs)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        net = cls(base=int(z["base"]), levels=int(z["levels"]))
        for i, l in enumerate(net.layers()):
            w = torch.from_numpy(z[f"w{i}"].astype(np.int16)).view(bf16).float()
            l.w.zero_()
            l.w[:, :9 * l.cin].copy_(w)
            l.b.copy_(torch.from_numpy(z[f"b{i}"]))
            l.refresh()
        net.meta = {k[5:]: z[k] for k in z.files if k.startswith("meta_")}
        return net


# ------------------------------------------------------------------------------------------ data
def random_temperature(x, z, rng):
    """Smooth random field in [0, 1] around the conductive profile (boundary values 1 bottom, 0 top)."""
    T = 1.0 - z
    for _ in range(6):
        k, l = rng.integers(1, 5), rng.integers(1, 5)
        T = T + rng.normal(0, 0.08) / (k + l) * 4 * np.cos(k * np.pi * x + rng.uniform(0, np.pi)) * np.sin(l * np.pi * z)
    return np.clip(T, 0.0, 1.0)


def pressure_scales(Ra, alphaT, rho0=1.0, s=1.0):
    """(pscale, ghyd) in the solver's pressure units (p / s, s = eta_ref / L_ref): the dynamic
    pressure is O(Ra), the hydrostatic gradient of the reference density rho0 Ra / alphaT."""
    return float(Ra) / s, float(rho0 * Ra / alphaT) / s


def features_targets(box, T, eta_e, Ra, alphaT, f=1, solV=None, solP=None, stats=None, X=None, Y=None, rho0=1.0,
                     s=1.0, scales=None):
    """Network input (and, with a solution, its target) for one model state (all on the device)."""
    gx, gz = box.nelx // f, box.nelz // f
    stats = torch.empty(2, dtype=torch.float64, device="cuda") if stats is None else stats
    X = torch.empty(gz, gx, 2, dtype=bf16, device="cuda") if X is None else X
    call("mw_unet_features", box, f, ptr(T), ptr(eta_e), float(Ra), ptr(stats), ptr(X), stream_ptr())
    if solV is not None:
        Y = torch.empty(box.nelz, box.nelx, NOUT, dtype=f32, device="cuda") if Y is None else Y
        scales = torch.empty(2, dtype=torch.float64, device="cuda") if scales is None else scales
        pscale, ghyd = pressure_scales(Ra, alphaT, rho0, s)
        call("mw_unet_targets", box, ptr(solV), ptr(solP), ptr(stats), pscale, ghyd, ptr(scales), ptr(Y),
             stream_ptr())
    return X, Y, stats


def generate_dataset(n=128, nruns=20, nsteps=110, skip=10, seed=0, Ra_range=(1e4, 1e6), contrast_range=(1.0, 1e5),
                     tol=1e-8, log=None):
    """Snapshots of the time-stepping method itself: `nruns` Frank-Kamenetskii convection models
    (Ra and viscosity contrast log-uniform, random smooth initial temperature) advanced `nsteps`
    steps each on the device; every step after `skip` contributes (features of the state the Stokes
    solve saw, targets of its solution).  Returns (X [S, n, n, 2] bf16, Y [S, n, n, NOUT] fp32, meta)."""
    from dataclasses import replace
    from . import configs
    from .timestep import GPUModel
    rng = np.random.default_rng(seed)
    S = nruns * (nsteps - skip)
    Xs = torch.empty(S, n, n, 2, dtype=bf16, device="cuda")
    Ys = torch.empty(S, n, n, NOUT, dtype=f32, device="cuda")
    meta = []
    s = 0
    for run in range(nruns):
        Ra = math.exp(rng.uniform(math.log(Ra_range[0]), math.log(Ra_range[1])))
        c = math.exp(rng.uniform(math.log(contrast_range[0]), math.log(contrast_range[1])))
        cfg = replace(configs.fk_convection(n), Ra=Ra, fk_gamma=math.log(c), seed=int(seed * 1000 + run))
        host = configs.build_host_model(cfg)
        host.arrays["T"] = random_temperature(host.x_V, host.z_V, rng)
        m = GPUModel(cfg, host, stokes="mixed", tol=tol)
        rec = _Recorder(m)
        m.guess = rec
        for k in range(nsteps):
            m.step()
            err = int(m.err.item())
            if m.last_solve.get("status") != "MW_OK" or err:    # keep only converged, valid states
                if log:
                    log(f"dataset run {run}: step {k} stopped (device flags {err}, solve {m.last_solve})")
                break
            if k >= skip:
                features_targets(m.box, rec.T, rec.eta, cfg.Ra, cfg.alphaT, 1, m.solV, m.solP, X=Xs[s], Y=Ys[s],
                                 rho0=cfg.rho0, s=cfg.eta_ref / m.L_ref)
                meta.append((run, k, Ra, c, m.last_solve.get("outer_iters", -1)))
                s += 1
        if log:
            log(f"dataset run {run}/{nruns}: Ra={Ra:.3g} contrast={c:.3g} last uzawa={m.last_solve}")
        del m
    Xs, Ys = Xs[:s], Ys[:s]
    bad = ~torch.isfinite(Ys.view(s, -1)).all(1)
    if bool(bad.any()):
        keep = (~bad).nonzero().view(-1)
        Xs, Ys = Xs[keep], Ys[keep]
        meta = [meta[i] for i in keep.tolist()]
    return Xs, Ys, meta


class _Recorder:
    """Guess hook that keeps the previous solution as the guess and copies the state the solve sees."""

    def __init__(self, m):
        self.T = torch.empty_like(m.T)
        self.eta = torch.empty_like(m.eta_e)

    def __call__(self, m):
        self.T.copy_(m.T)
        self.eta.copy_(m.eta_e)


def train(net, Xs, Ys, epochs=20, batch=16, lr=1e-3, seed=0, log=None):
    """Mini-batch Adam on the device; returns the per-epoch mean losses."""
    n = Xs.shape[0]
    H, W = Xs.shape[1], Xs.shape[2]
    rng = np.random.default_rng(seed)
    losses = []
    Xb = torch.empty(batch, H, W, 2, dtype=bf16, device="cuda")
    Yb = torch.empty(batch * H * W, NOUT, dtype=f32, device="cuda")
    for ep in range(epochs):
        perm = rng.permutation(n)
        tot = torch.zeros(1, dtype=torch.float64, device="cuda")
        nb = 0
        for i in range(0, n - batch + 1, batch):
            idx = torch.as_tensor(perm[i:i + batch], device="cuda")
            torch.index_select(Xs, 0, idx, out=Xb)
            torch.index_select(Ys, 0, idx, out=Yb.view(batch, H, W, NOUT))
            y = net.forward(Xb, batch, H, W)
            dy, part = net.mse(y, Yb)
            net.backward(dy)
            lr_t = lr * 0.5 * (1 + math.cos(math.pi * (ep * n + i) / (epochs * n)))
            net.step(lr=lr_t)
            tot += part.sum()
            nb += 1
        losses.append(float(tot.item()) / (nb * batch * H * W * NOUT))
        if log:
            log(f"epoch {ep}: mse {losses[-1]:.4e}")
    return losses


class WarmStart:
    """Stokes initial guess from the trained network at the network resolution `n_net` (the model
    grid is pooled by f = nelx / n_net and the prediction interpolated back).  The network halves
    its grid three times, so the pooled grid is padded up to multiples of 8 (the last cell row and
    column repeated) and the prediction is read on the mesh's cells only."""

    def __init__(self, net, box, Ra, alphaT, bc_fix_V, n_net=128, rho0=1.0, s=1.0):
        self.net, self.box, self.Ra = net, box, float(Ra)
        self.pscale, self.ghyd = pressure_scales(Ra, alphaT, rho0, s)
        self.f = max(1, box.nelx // n_net)
        if box.nelx % self.f or box.nelz % self.f:
            raise ValueError(f"the pooling factor {self.f} does not divide the {box.nelx}x{box.nelz} mesh")
        self.gx, self.gz = box.nelx // self.f, box.nelz // self.f
        self.gxp, self.gzp = -(-self.gx // 8) * 8, -(-self.gz // 8) * 8
        self.fix = bc_fix_V.view(torch.uint8) if bc_fix_V.dtype == torch.bool else bc_fix_V
        self.stats = torch.empty(2, dtype=torch.float64, device="cuda")
        self.scales = torch.empty(2, dtype=torch.float64, device="cuda")
        self.X = torch.empty(1, self.gzp, self.gxp, 2, dtype=bf16, device="cuda")

    def guess(self, T, eta_e, solV, solP):
        call("mw_unet_features_padded", self.box, self.f, self.gxp, self.gzp, ptr(T), ptr(eta_e), self.Ra,
             ptr(self.stats), ptr(self.X), stream_ptr())
        y = self.net.forward(self.X, 1, self.gzp, self.gxp)
        call("mw_unet_to_fields_padded", self.box, self.f, self.gxp, ptr(y), ptr(self.stats), self.pscale, self.ghyd,
             ptr(self.scales), ptr(self.fix), ptr(solV), ptr(solP), stream_ptr())
        return solV, solP


class LearnedGuess:
    """Initial-guess hook for ``GPUModel.guess`` gated by the Uzawa residual.

    The Schur-complement (Uzawa) iteration recomputes the velocity from the pressure, so a
    candidate is judged by the residual it starts from: ||G^T K^-1 (f - G P) - h|| (one inner
    multigrid-PCG solve per candidate, ``StokesSolver.uzawa_residual``).  Candidates:
      * ``zero``      - the cold start (first step, or after ``reset()``);
      * ``previous``  - the previous step's solution (the method without the network);
      * ``learned``   - the network's prediction;
      * ``increment`` - previous solution + (network(now) - network(previous step)).
    The candidate with the smallest Uzawa residual is handed to the solver -- its pressure with the
    velocity the judgement computed from it (the previous solution whole) -- so the network can
    never make a solve start from a worse point than the fallback.  With ``judge="cold"`` (the
    default) the network is consulted only when there is no previous solution and the previous
    step's solution is used directly otherwise; ``judge="every"`` weighs all candidates at every
    step (one extra inner solve per candidate)."""

    def __init__(self, model, net, n_net=128, judge="cold", rtol=None):
        c = model.cfg
        self.ws = WarmStart(net, model.box, c.Ra, c.alphaT, model.bc_fix_V, n_net, c.rho0, c.eta_ref / model.L_ref)
        # inner tolerance of the judgement's velocity solves: at a cold start the candidates' residuals
        # differ by orders of magnitude and 2e-2 (the mixed solver's own inner tolerance) separates
        # them (512x512 first step: 53.9 ms with 2e-2, 79.1 with 1e-3, 57.3 from zero; 27 Schur
        # iterations either way, measured); weighing the previous solution against the network's
        # increment at every step needs 1e-3
        self.judge = judge
        self.rtol = rtol if rtol is not None else (1e-3 if judge == "every" else 2e-2)
        self.prec = "f64" if model.stokes_precision == "f64" else "f32"
        E = lambda t: torch.empty_like(t)
        self.nnV, self.nnP = E(model.solV), E(model.solP)          # network fields, this step
        self.prevV, self.prevP = E(model.solV), E(model.solP)      # network fields, previous step
        self.candP = E(model.solP)
        # the velocity K^-1 (f - G P) each candidate's judgement computes: the guess handed to the
        # solver with a learned, incremental or zero pressure (the network's own velocity is far
        # less accurate than its pressure: at the 512x512 FK model's first step 6.3x the solution's
        # norm off against 7e-4 for the pressure; with it the full residual starts at 38x that of
        # zero and the solve needs 49 Schur iterations, with the consistent velocity 27, from zero 36)
        self.uzV = {k: E(model.solV) for k in ("zero", "learned", "increment")}
        self.have_prev_nn = False
        self.cold = True
        self.picks = {k: 0 for k in ("previous", "increment", "learned", "zero")}
        self.last = {}

    def idle(self):
        """True when the next call launches nothing (the solve starts from the previous solution),
        so a recorded time step may stand in for the step with this hook."""
        return not (self.cold or self.judge == "every")

    def reset(self):
        """Forget the previous solution (the next step is a cold start)."""
        self.cold = True
        self.have_prev_nn = False

    def _res(self, m, P, V=None):
        return m.solver.uzawa_residual(m.rhs_f, m.rhs_h, P, precision=self.prec, rtol=self.rtol, V=V)

    def __call__(self, m):
        use_nn = self.cold or self.judge == "every"
        if not use_nn:
            self.picks["previous"] += 1
            self.last = dict(pick="previous")
            self.have_prev_nn = False
            return
        self.ws.guess(m.T, m.eta_e, self.nnV, self.nnP)
        res = {}
        zeroP = None
        if self.cold:
            zeroP = torch.zeros_like(m.solP)
            res["zero"] = self._res(m, zeroP, self.uzV["zero"])
        else:
            res["previous"] = self._res(m, m.solP)
            if self.have_prev_nn:
                torch.add(m.solP, self.nnP - self.prevP, out=self.candP)
                res["increment"] = self._res(m, self.candP, self.uzV["increment"])
        res["learned"] = self._res(m, self.nnP, self.uzV["learned"])
        best = min(res, key=lambda k: res[k] if math.isfinite(res[k]) else math.inf)
        # the pressure of the winner with the velocity its judgement computed (the previous step's
        # solution is kept whole: its velocity is more accurate than the judgement's solve)
        if best == "learned":
            m.solP.copy_(self.nnP)
        elif best == "increment":
            m.solP.copy_(self.candP)
        elif best == "zero":
            m.solP.zero_()
        if best != "previous":
            m.solV.copy_(self.uzV[best])
        self.picks[best] += 1
        self.last = dict(res, pick=best)
        self.nnV, self.prevV = self.prevV, self.nnV
        self.nnP, self.prevP = self.prevP, self.nnP
        self.have_prev_nn = True
        self.cold = False


def compare_guesses(net, cfg, nsteps=20, n_net=128, tol=1e-8, host=None):
    """Run the same model with the zero guess, the previous-step guess, the gated learned guess
    consulted at cold starts only, and the gated learned guess weighed at every step; return the
    Stokes iteration counts of each step."""
    from . import configs
    from .timestep import GPUModel
    host = host if host is not None else configs.build_host_model(cfg)
    out = {}
    for mode in ("zero", "previous", "learned", "learned_every"):
        m = GPUModel(cfg, host, stokes="mixed", tol=tol, warm_start="zero" if mode == "zero" else "previous")
        hook = None
        if mode.startswith("learned"):
            hook = LearnedGuess(m, net, n_net=n_net, judge="every" if mode == "learned_every" else "cold")
            m.guess = hook
        rec = []
        for _ in range(nsteps):
            m.step()
            i = m.last_solve
            rec.append(dict(outer=i["outer_iters"], inner=i["inner_iters"], r0=i["initial_rel_residual"],
                            r=i["rel_residual"], **({"pick": hook.last["pick"]} if hook else {})))
        d = m.diagnostics()
        out[mode] = dict(steps=rec, outer=sum(r["outer"] for r in rec), inner=sum(r["inner"] for r in rec),
                         vrms=d["vrms"], Nu=d["Nu"], picks=dict(hook.picks) if hook else None)
        del m
    return out


def cold_start_gain(net, cases, steps_before=0, n_net=128, tol=1e-8, log=None):
    """cases: [(cfg, seed of a random smooth initial temperature or None)].  For each model: advance
    `steps_before` steps, then solve the next step's Stokes problem twice on the same operator,
    from zero and from the network's guess for the state that solve sees.  Returns
    [(name, zero outer iterations, learned outer iterations, zero inner, learned inner)]."""
    from . import configs
    from .timestep import GPUModel
    out = []
    for cfg, tseed in cases:
        host = configs.build_host_model(cfg)
        if tseed is not None:
            host.arrays["T"] = random_temperature(host.x_V, host.z_V, np.random.default_rng(tseed))
        m = GPUModel(cfg, host, stokes="mixed", tol=tol)
        rec = _Recorder(m)
        m.guess = rec
        for _ in range(steps_before + 1):
            m.step()
        ws = WarmStart(net, m.box, cfg.Ra, cfg.alphaT, m.bc_fix_V, n_net, cfg.rho0, cfg.eta_ref / m.L_ref)
        V = torch.empty_like(m.solV)
        P = torch.empty_like(m.solP)
        ws.guess(rec.T, rec.eta, V, P)
        m.solver.uzawa_residual(m.rhs_f, m.rhs_h, P, precision="f32", rtol=1e-3, V=V)   # V = K^-1 (f - G P)
        _, _, i0 = m.solver.solve(m.rhs_f, m.rhs_h, None, None, precision="mixed", tol=tol, inner_rtol=1e-3)
        _, _, i1 = m.solver.solve(m.rhs_f, m.rhs_h, V, P, precision="mixed", tol=tol, inner_rtol=1e-3)
        out.append((cfg.name, i0["outer_iters"], i1["outer_iters"], i0["inner_iters"], i1["inner_iters"]))
        if log:
            log(f"cold start {cfg.name}: zero {i0['outer_iters']} / learned {i1['outer_iters']} outer iterations")
        del m
    return out
