"""The oracle's whole time step against the reference's own driver.

``tests/golden/driver_*.npz`` hold runs of the unmodified ``meeuuw.py`` (made by
``tests/golden/make_driver_golden.py``): per-step vrms, Nu and dt, and the final fields and
swarm.  ``oracle.model.OracleModel`` chains the pinned oracle functions in the driver's order;
these tests pin that order (strain rate of the previous step, T_mem, the dt rule, where the
pressure is normalised, advection then locate) to the driver itself.

Both sides solve Stokes with a sparse direct solve (SuperLU), so the differences left are
round-off amplified by the saddle-point system's conditioning: vrms 1e-8, Nu 1e-10 relative;
fields 1e-7 of their maximum (strain rates 1e-5: derivatives of that round-off); particle
element indices, active flags and per-element counts bit-exact.
"""
import json

import numpy as np
import pytest

from conftest import golden


def driver_config(name):
    from meeuuw_b200 import configs
    d = golden(name)
    meta = json.loads(str(d["meta"]))
    n = meta["nel"]
    if meta["experiment"] == 0:
        kw = dict(RKorder=meta["RKorder"], averaging=meta["averaging"], nstep=meta["nstep"])
        if "2a" in meta["overrides"]:                        # experiment0.py:74-75: eta = exp(-6.907755279 T)
            kw["fk_gamma"] = 6.907755279
        cfg = configs.blankenbach(n, **kw)
    else:                                                    # experiment1.py as shipped, regular particles
        cfg = configs.rayleigh_taylor(n, mat_rho=(1000.0, 1010.0), mat_eta=(100.0, 100.0), particle_distribution=1,
                                      nparticle_per_dim=5, nstep=meta["nstep"])
    return cfg, d, meta


def check_against_driver(d, per_step, fields, swarm, nel, vrms_tol, nu_tol, field_tol):
    """per_step: list of (vrms, Nu, dt); fields: {name: full array}; swarm: x, z, iel, active (full)."""
    for s, (vrms, nu, dt) in enumerate(per_step):
        assert abs(vrms / d["vrms"][s] - 1) < vrms_tol, (s, vrms, d["vrms"][s])
        assert abs(dt / d["dt"][s] - 1) < vrms_tol, (s, dt, d["dt"][s])
        if len(d["Nu"]):
            assert abs(nu / d["Nu"][s] - 1) < nu_tol, (s, nu, d["Nu"][s])
    nodes = d["nodes"]
    for k, v in fields.items():
        if k not in d:
            continue
        ref = d[k]
        got = v[d["pnodes"]] if k == "p" else v[nodes]
        # strain rates differentiate u, w: the solve's round-off (~1e-9 of max |u|) grows by ~1/h
        tol = 1e-5 if k.startswith("e") else field_tol
        assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref)), k
    P = d["particles"]
    x, z, iel, act = swarm
    assert np.array_equal(act[P], d["swarm_active"])
    assert np.array_equal(iel[P], d["swarm_iel"])
    assert np.array_equal(np.bincount(iel[act], minlength=nel), d["counts"])
    assert np.max(np.abs(x[P] - d["swarm_x"])) < 1e-9
    assert np.max(np.abs(z[P] - d["swarm_z"])) < 1e-9


@pytest.mark.parametrize("name", ["driver_fk_16", "driver_c0_32", "driver_rt_64"])
def test_oracle_model_matches_driver(name):
    from oracle.model import OracleModel
    from meeuuw_b200 import configs
    cfg, d, meta = driver_config(name)
    host = configs.build_host_model(cfg)
    om = OracleModel(cfg, host)
    if "swarm_mat" in d:                                     # experiment1.py:25-36 layout, bit-exact
        assert np.array_equal(om.mat[d["particles"]], d["swarm_mat"])
    steps = []
    for _ in range(meta["nstep"]):
        o = om.step(solver="direct")
        steps.append((o["vrms"], o["Nu"], o["dt"]))
    fields = dict(u=o["u"], w=o["w"], p=o["p"], q=om.q, exx_n=om.exx_n, ezz_n=om.ezz_n, exz_n=om.exz_n)
    if cfg.solve_T:
        fields["T"] = om.T
    check_against_driver(d, steps, fields, (om.x, om.z, om.iel, om.active), cfg.nel, 1e-8, 1e-10, 1e-7)
