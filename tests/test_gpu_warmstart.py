"""What the trained warm-start network gains over the method without it.

The network (meeuuw_b200/weights/unet_fk128.npz, trained on the GPU by
``python -m meeuuw_b200.train_warmstart`` from snapshots of the device time stepper) is applied to
held-out models -- seeds, Ra, viscosity contrasts and initial temperatures it never saw -- at a cold
start, where the method has no previous solution to start from.  The Stokes solve to 1e-8 from the
network's guess needs fewer Schur (Uzawa) iterations than the solve from zero, and the gated hook
never starts a solve from a worse Uzawa residual than its fallback."""
import math
import os
from dataclasses import replace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(__file__)), "meeuuw_b200", "weights", "unet_fk128.npz")


def _cases(k, n=128):
    from meeuuw_b200 import configs
    rng = np.random.default_rng(4242)
    out = []
    for i in range(k):
        Ra = math.exp(rng.uniform(math.log(3e4), math.log(1e6)))
        c = math.exp(rng.uniform(math.log(10.0), math.log(1e5)))
        out.append((replace(configs.fk_convection(n), name=f"t{i}", Ra=Ra, fk_gamma=math.log(c), seed=31000 + i),
                    71000 + i))
    return out


def test_learned_cold_start_needs_fewer_uzawa_iterations():
    from meeuuw_b200.unet import UNet, cold_start_gain
    net = UNet.load(WEIGHTS)
    res = cold_start_gain(net, _cases(3), steps_before=5)
    zero = sum(r[1] for r in res)
    learned = sum(r[2] for r in res)
    assert learned < zero, res


def test_gate_never_starts_worse_than_fallback():
    from meeuuw_b200 import configs
    from meeuuw_b200.timestep import GPUModel
    from meeuuw_b200.unet import LearnedGuess, UNet, random_temperature
    net = UNet.load(WEIGHTS)
    cfg, tseed = _cases(1)[0]
    host = configs.build_host_model(cfg)
    host.arrays["T"] = random_temperature(host.x_V, host.z_V, np.random.default_rng(tseed))
    m = GPUModel(cfg, host, stokes="mixed")
    hook = LearnedGuess(m, net, judge="every")
    m.guess = hook
    for _ in range(4):
        m.step()
        last = dict(hook.last)
        pick = last.pop("pick")
        fallback = last["zero"] if "zero" in last else last["previous"]
        assert last[pick] <= fallback, hook.last
        assert m.last_solve["converged"] == 1


def test_learned_cold_start_512_from_128_network():
    """The network trained at 128x128 applied to the 512x512 FK model's first step (its input pooled
    4x4, its output interpolated back): the gated guess -- the network's pressure with the velocity
    the gate computed from it -- takes the solve to 1e-8 in fewer Schur iterations than from zero."""
    from meeuuw_b200 import configs
    from meeuuw_b200.timestep import GPUModel
    from meeuuw_b200.unet import LearnedGuess, UNet
    net = UNet.load(WEIGHTS)
    cfg = configs.fk_convection(512, seed=1000)
    host = configs.build_host_model(cfg)
    outer = {}
    for arm in ("learned", "zero"):
        m = GPUModel(cfg, host, stokes="mixed", tol=1e-8, warm_start="zero" if arm == "zero" else "previous")
        if arm == "learned":
            m.guess = LearnedGuess(m, net, judge="cold")
        m.step()
        assert m.last_solve["converged"] == 1, m.last_solve
        outer[arm] = m.last_solve["outer_iters"]
        if arm == "learned":
            assert m.guess.last["pick"] == "learned", m.guess.last
        del m
    assert outer["learned"] < outer["zero"], outer


def test_warm_start_on_meshes_not_multiple_of_eight():
    """Meshes whose network grid is not a multiple of 8 (66x66, 100x60) run the network on a
    replicate-padded grid; the guess is finite, its fixed velocity dofs are zero, and the gated
    cold start converges (the ensemble's uneven members all get a learned guess)."""
    import torch
    from dataclasses import replace
    from meeuuw_b200 import configs
    from meeuuw_b200.timestep import GPUModel
    from meeuuw_b200.unet import LearnedGuess, UNet, WarmStart, _Recorder
    net = UNet.load(WEIGHTS)
    for nx, nz in ((66, 66), (100, 60)):
        cfg = replace(configs.fk_convection(nx), nelz=nz, Lz=nz / nx, name=f"pad{nx}x{nz}")
        host = configs.build_host_model(cfg)
        m = GPUModel(cfg, host, stokes="mixed")
        rec = _Recorder(m)                  # the state (T, element viscosity) a step's Stokes solve sees
        m.guess = rec
        m.step()
        ws = WarmStart(net, m.box, cfg.Ra, cfg.alphaT, m.bc_fix_V, 128, cfg.rho0, cfg.eta_ref / m.L_ref)
        assert (ws.gxp, ws.gzp) == (-(-nx // 8) * 8, -(-nz // 8) * 8)
        V, P = torch.empty_like(m.solV), torch.empty_like(m.solP)
        ws.guess(rec.T, rec.eta, V, P)
        assert bool(torch.isfinite(V).all()) and bool(torch.isfinite(P).all())
        assert float(V[m.bc_fix_V].abs().max()) == 0.0
        m = GPUModel(cfg, host, stokes="mixed")
        m.guess = LearnedGuess(m, net)
        m.step()
        assert m.last_solve["converged"] == 1, m.last_solve
        assert m.guess.last["pick"] in ("learned", "zero")


def test_padded_features_equal_unpadded_on_multiples_of_eight():
    import torch
    from meeuuw_b200 import configs
    from meeuuw_b200._lib import call, ptr, stream_ptr
    from meeuuw_b200.timestep import GPUModel
    from meeuuw_b200.unet import _Recorder
    cfg = configs.fk_convection(64)
    m = GPUModel(cfg, configs.build_host_model(cfg), stokes="mixed")
    rec = _Recorder(m)
    m.guess = rec
    m.step()
    stats = torch.empty(2, dtype=torch.float64, device="cuda")
    X0 = torch.empty(64, 64, 2, dtype=torch.bfloat16, device="cuda")
    X1 = torch.empty(72, 72, 2, dtype=torch.bfloat16, device="cuda")
    call("mw_unet_features", m.box, 1, ptr(rec.T), ptr(rec.eta), float(cfg.Ra), ptr(stats), ptr(X0), stream_ptr())
    call("mw_unet_features_padded", m.box, 1, 72, 72, ptr(rec.T), ptr(rec.eta), float(cfg.Ra), ptr(stats), ptr(X1),
         stream_ptr())
    assert bool(torch.isfinite(X0.float()).all())
    assert torch.equal(X1[:64, :64], X0)
    assert torch.equal(X1[64:, :64], X0[63:64].expand(8, 64, 2)) and torch.equal(X1[:64, 64:], X0[:, 63:64].expand(64, 8, 2))
