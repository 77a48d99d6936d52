"""The device time stepper at the benchmark configurations' sizes, against the reference.

* config 0 (Blankenbach 1a, 32x32, 4x4 regular particles, RK2, CN, 20 steps) and a 16x16
  temperature-dependent-viscosity run (geometric averaging, RK4, 3 steps): against runs of the
  reference's own driver (``tests/golden/driver_*.npz``, ``make_driver_golden.py``);
* config 2's Rayleigh-Taylor set-up as the reference ships it (``experiment1.py``: 0.9142 x 1 box,
  no slip top and bottom, two materials carried by the particles, 25 regular particles per
  element): 64x64 for 20 steps and 256x256 for 2 steps, against the reference's driver;
* config 1 (512x512 FK convection, 4.2 M seeded random particles, RK4): the first step of the
  product path (mixed precision, learned warm start) and of the plain FP64 path, against the
  FP64 oracle's step (``oracle_fk512_step1.npz``, ``make_oracle_golden.py``).

Against the reference's driver (direct solves) both arms solve Stokes to an FP64 relative residual
of 1e-10: these tests check the composition of the step, and on these buoyancy-driven problems a
relative residual of 1e-8 -- a norm dominated by the hydrostatic part of the load -- still leaves
vrms off by 3e-6 (mixed, 16x16 FK cold start) to 4e-4 (FP64, which stops at the first iterate under
the tolerance) on the small meshes (measured).  The 512x512 test runs the product path at the
benchmark's own 1e-8 and holds it to the 1e-6 bar.
Bars: vrms, Nu and dt within 1e-6 relative per step; T within 1e-7; u, w, p, q within 1e-6 of
their maximum (strain rates 1e-4: derivatives); particle element indices, active flags,
material ids and per-element counts bit-exact; positions within 1e-8.
"""
import json
import os

import numpy as np
import pytest

from conftest import golden
from test_oracle_driver import driver_config

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "meeuuw_b200", "weights",
                       "unet_fk128.npz")


def run_gpu(cfg, nsteps, stokes, guess=False, tol=1e-10):
    from meeuuw_b200 import configs
    from meeuuw_b200.timestep import GPUModel
    host = configs.build_host_model(cfg)
    gm = GPUModel(cfg, host, stokes=stokes, tol=tol)
    if guess:
        from meeuuw_b200.unet import LearnedGuess, UNet
        gm.guess = LearnedGuess(gm, UNet.load(WEIGHTS), judge="cold")
    steps = []
    for _ in range(nsteps):
        gm.step()
        d = gm.diagnostics()
        gm.check()
        assert d["stokes"]["converged"] == 1, d["stokes"]
        steps.append((d["vrms"], d["Nu"], d["dt"]))
    return gm, steps


def gpu_fields(gm):
    c = lambda t: t.cpu().numpy()
    f = dict(u=c(gm.u), w=c(gm.w), p=c(gm.p), q=c(gm.q), exx_n=c(gm.exx_n), ezz_n=c(gm.ezz_n), exz_n=c(gm.exz_n))
    if gm.cfg.solve_T:
        f["T"] = c(gm.T)
    return f


def check(d, steps, gm, nsteps_expected):
    assert len(d["vrms"]) == nsteps_expected
    for s, (vrms, nu, dt) in enumerate(steps):
        assert abs(vrms / d["vrms"][s] - 1) < 1e-6, (s, vrms, d["vrms"][s])
        assert abs(dt / d["dt"][s] - 1) < 1e-6, (s, dt, d["dt"][s])
        if len(d["Nu"]):
            assert abs(nu / d["Nu"][s] - 1) < 1e-6, (s, nu, d["Nu"][s])
    f = gpu_fields(gm)
    for k, v in f.items():
        if k not in d:
            continue
        got = v[d["pnodes"]] if k == "p" else v[d["nodes"]]
        ref = d[k]
        if k == "T":
            assert np.max(np.abs(got - ref)) < 1e-7
        else:
            tol = 1e-4 if k.startswith("e") else 1e-6
            assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref)), k
    P = d["particles"]
    act, iel = gm.active.cpu().numpy(), gm.iel.cpu().numpy()
    assert np.array_equal(act[P], d["swarm_active"])
    assert np.array_equal(iel[P], d["swarm_iel"])
    assert np.array_equal(np.bincount(iel[act], minlength=gm.nel), d["counts"])
    assert np.max(np.abs(gm.x.cpu().numpy()[P] - d["swarm_x"])) < 1e-8
    assert np.max(np.abs(gm.z.cpu().numpy()[P] - d["swarm_z"])) < 1e-8
    if "swarm_mat" in d:
        assert np.array_equal(gm.mat.cpu().numpy()[P], d["swarm_mat"])


@pytest.mark.parametrize("stokes", ["mixed", "f64"])
def test_config0_blankenbach_32_twenty_steps_vs_driver(stokes):
    cfg, d, meta = driver_config("driver_c0_32")
    gm, steps = run_gpu(cfg, meta["nstep"], stokes)
    check(d, steps, gm, 20)


def test_fk_16_vs_driver():
    cfg, d, meta = driver_config("driver_fk_16")
    gm, steps = run_gpu(cfg, meta["nstep"], "mixed")
    check(d, steps, gm, 3)


def test_config2_rt_64_twenty_steps_vs_driver():
    cfg, d, meta = driver_config("driver_rt_64")
    gm, steps = run_gpu(cfg, meta["nstep"], "mixed")
    check(d, steps, gm, 20)


def test_config2_rt_256_vs_driver():
    cfg, d, meta = driver_config("driver_rt_256")
    gm, steps = run_gpu(cfg, meta["nstep"], "mixed")
    check(d, steps, gm, 2)


@pytest.mark.parametrize("arm", ["product", "f64"])
def test_config1_fk512_first_step_vs_fp64_oracle(arm):
    from meeuuw_b200 import configs
    d = golden("oracle_fk512_step1")
    meta = json.loads(str(d["meta"]))
    cfg = configs.fk_convection(meta["n"], seed=meta["seed"])
    gm, steps = run_gpu(cfg, 1, "mixed" if arm == "product" else "f64", guess=(arm == "product"),
                        tol=1e-8 if arm == "product" else 1e-10)
    vrms, nu, dt = steps[0]
    assert abs(vrms / d["vrms"] - 1) < 1e-6, (vrms, float(d["vrms"]))
    assert abs(nu / d["Nu"] - 1) < 1e-6, (nu, float(d["Nu"]))
    assert abs(dt / d["dt"] - 1) < 1e-6
    f = gpu_fields(gm)
    assert np.max(np.abs(f["T"][d["nodes"]] - d["T"])) < 1e-7
    for k in ("u", "w", "q"):
        assert np.max(np.abs(f[k][d["nodes"]] - d[k])) <= 1e-6 * np.max(np.abs(d[k])), k
    assert np.max(np.abs(f["p"][d["pnodes"]] - d["p"])) <= 1e-6 * np.max(np.abs(d["p"]))
    assert np.max(np.abs(gm.eta_e.cpu().numpy()[::16] / d["eta_e"] - 1)) < 1e-12
    P = d["particles"]
    act, iel = gm.active.cpu().numpy(), gm.iel.cpu().numpy()
    assert np.array_equal(act[P], d["swarm_active"])
    assert np.array_equal(iel[P], d["swarm_iel"])
    assert np.array_equal(np.bincount(iel[act], minlength=gm.nel), d["counts"])
