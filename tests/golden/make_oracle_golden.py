"""Fixtures from the oracle at sizes the test suite cannot afford to recompute.

    python tests/golden/make_oracle_golden.py [case ...]

``fk512_step1``: the 512x512 FK convection model (Ra 1e6, eta = exp(-ln(1e5) T),
geometric averaging, 16 seeded random particles per element, RK4; the model the
timesteps/s figure is measured on, rank 0's seed) advanced one time step by
``oracle.model.OracleModel`` with the reference's ``cd_u_eta`` Schur-complement solver and
SuperLU inner solves (``cd_u_eta.py:13-99``, its own stopping rule), K factorised under a
symmetric minimum-degree ordering (the direct saddle-point solve and COLAMD run out of memory
at this size; on the 64x64 model the two give vrms within 5e-11 and residuals of 3e-12 and
4e-13).  The oracle is pinned to the reference's own functions and driver by
``tests/test_oracle_golden.py`` and ``tests/test_oracle_driver.py``; one step at 512x512
takes about seven minutes and 16 GB on one core, so it is stored.
Kept: the step's scalars, the fields on every eighth node of every eighth node row, the
per-element particle counts after advection and every 256th particle.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def fk512_step1():
    from meeuuw_b200 import configs
    from oracle.model import OracleModel
    n, seed = 512, 1000
    cfg = configs.fk_convection(n, seed=seed)
    host = configs.build_host_model(cfg)
    om = OracleModel(cfg, host)
    om.stokes_kw = dict(permc_spec="MMD_AT_PLUS_A")
    om.energy_kw = dict(permc_spec="MMD_AT_PLUS_A")
    t0 = time.perf_counter()
    o = om.step(solver="cd_u_eta")
    secs = time.perf_counter() - t0
    nnx = 2 * n + 1
    nodes = np.arange(nnx * nnx)
    nodes = nodes[((nodes % nnx) % 8 == 0) & ((nodes // nnx) % 8 == 0)]
    pn = np.arange((n + 1) ** 2)
    pnodes = pn[((pn % (n + 1)) % 4 == 0) & ((pn // (n + 1)) % 4 == 0)]
    parts = np.arange(0, cfg.nparticle, 256)
    out = dict(vrms=np.float64(o["vrms"]), Nu=np.float64(o["Nu"]), dt=np.float64(o["dt"]),
               stokes_residual=np.float64(o["stokes_residual"]),
               nodes=nodes.astype(np.int32), pnodes=pnodes.astype(np.int32), particles=parts.astype(np.int32),
               T=o["T"][nodes], u=o["u"][nodes], w=o["w"][nodes], q=o["q"][nodes], p=o["p"][pnodes],
               eta_e=o["eta_e"][::16].copy(),
               counts=np.bincount(om.iel[om.active], minlength=cfg.nel).astype(np.int32),
               swarm_x=om.x[parts], swarm_z=om.z[parts], swarm_iel=om.iel[parts].astype(np.int32),
               swarm_active=om.active[parts])
    out["meta"] = np.array(json.dumps(dict(config="fk_convection", n=n, seed=seed, steps=1,
                                           solver="cd_u_eta (SuperLU, MMD_AT_PLUS_A)",
                                           stokes_iterations=int(o["stokes_iterations"]), oracle_seconds=secs,
                                           phase_seconds=om.phase_seconds)))
    np.savez_compressed(os.path.join(HERE, "oracle_fk512_step1.npz"), **out)
    print("fk512_step1", {k: v.shape for k, v in out.items()}, f"{secs:.0f} s")


CASES = {"fk512_step1": fk512_step1}

if __name__ == "__main__":
    sys.path.insert(0, ROOT)
    for c in (sys.argv[1:] or list(CASES)):
        CASES[c]()
