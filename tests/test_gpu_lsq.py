"""Least-squares particle projections, their limiter, and population control on the GPU against the
reference's own outputs (``tests/golden/lsq.npz``, ``population.npz``; ``make_golden.py lsq``).

Tolerances: fit coefficients and their qpoint values 1e-12 relative (the reference solves the
normal equations with LAPACK, the kernel by Gaussian elimination; the sums themselves follow the
reference's order); element extrema exact; population control: active flags, element indices,
material ids and the drawn reduced coordinates exact, positions and means 1e-14 relative.
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu


def D(a, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(a))
    return (t.to(dtype) if dtype is not None else t).cuda()


@pytest.fixture(scope="module")
def M():
    from meeuuw_b200 import _lib
    _lib.require_cuda()
    g = golden("mesh_6x4")
    g["box"] = _lib.box_of(6, 4, 1.5, 1.0)
    return g


@pytest.mark.parametrize("ncoef,limit", [(3, False), (3, True), (4, False)])
def test_ls_fit_and_qpoints(M, ncoef, limit):
    from meeuuw_b200 import ops
    g = golden("lsq")
    nel = 24
    every = torch.ones(len(g["swarm_x"]), dtype=torch.bool, device="cuda")   # the reference's mask: iel only
    counts, offsets, order = ops.bin_particles(nel, every, D(g["swarm_iel"]))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = ops.ls_fit(M["box"], ncoef, offsets, order, D(g["swarm_x"]), D(g["swarm_z"]),
                     [D(g["swarm_rho"]), D(g["swarm_eta"])], limit_h=float(M["hx"]) if limit else 0.0, err=err)
    assert int(err.item()) == 0
    tag = "P1" if ncoef == 3 else "Q1"
    for (coef, fmin, fmax), name in zip(out, ("rho", "eta")):
        c = coef.cpu().numpy()
        ref = {k: g[f"out_{tag}_{name}_{k}"] for k in "abcd"[:ncoef]}
        if limit:
            ref["b"], ref["c"] = g[f"out_P1lim_{name}_b"], g[f"out_P1lim_{name}_c"]
        for j, k in enumerate("abcd"[:ncoef]):
            assert rel_err(c[:, j], ref[k]) < 1e-12, (name, k)
        assert np.array_equal(fmin.cpu().numpy(), g[f"out_{tag}_{name}_min"])
        assert np.array_equal(fmax.cpu().numpy(), g[f"out_{tag}_{name}_max"])
        if limit or ncoef == 4:
            q = ops.ls_to_qpoints(M["box"], coef, D(M["xq"]), D(M["zq"])).cpu().numpy()
            assert rel_err(q, g[f"out_{tag}_{name}q"]) < 1e-12


def _pop_inputs(g):
    keys = ("swarm_active", "swarm_iel", "swarm_r", "swarm_t", "swarm_x", "swarm_z", "swarm_u", "swarm_w",
            "swarm_eta", "swarm_mat")
    return {k: D(g[k]) for k in keys}


def test_population_control(M):
    from meeuuw_b200 import ops
    g = golden("population")
    nel = 24
    a = _pop_inputs(g)
    # the step-start binning: the particles active before advection, by their step-start element
    counts, offsets, order = ops.bin_particles(nel, D(g["step_active"]), a["swarm_iel"])
    assert np.array_equal(counts.cpu().numpy(), g["nparticle_e"])
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    src = torch.full((len(g["swarm_x"]),), -1, dtype=torch.int32, device="cuda")
    added = ops.population_control(M["box"], int(g["nparticle_min"]), counts, offsets, order, a["swarm_active"],
                                   a["swarm_iel"], a["swarm_r"], a["swarm_t"], a["swarm_x"], a["swarm_z"],
                                   mat=a["swarm_mat"], avg=(a["swarm_eta"], a["swarm_u"], a["swarm_w"]), source=src,
                                   draws=D(g["draws"]), err=err)
    assert int(err.item()) == 0
    assert int(added.item()) == int(g["needed"])
    for k in ("swarm_active", "swarm_iel", "swarm_mat", "swarm_r", "swarm_t"):
        assert np.array_equal(a[k].cpu().numpy(), g["out_" + k]), k
    for k in ("swarm_x", "swarm_z", "swarm_u", "swarm_w", "swarm_eta"):
        assert rel_err(a[k].cpu().numpy(), g["out_" + k]) < 1e-14, k
    s = src.cpu().numpy()
    new = s >= 0
    assert new.sum() == int(g["needed"])
    assert np.array_equal(g["out_swarm_mat"][new], g["swarm_mat"][s[new]])


def test_population_control_device_draws(M):
    """Without supplied numbers the device draws them: same elements refilled, reduced coordinates
    inside [-0.95, 0.95), positions inside their elements."""
    from meeuuw_b200 import ops
    g = golden("population")
    a = _pop_inputs(g)
    counts, offsets, order = ops.bin_particles(24, D(g["step_active"]), a["swarm_iel"])
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    added = ops.population_control(M["box"], int(g["nparticle_min"]), counts, offsets, order, a["swarm_active"],
                                   a["swarm_iel"], a["swarm_r"], a["swarm_t"], a["swarm_x"], a["swarm_z"],
                                   mat=a["swarm_mat"], seed=1234, err=err)
    assert int(err.item()) == 0 and int(added.item()) == int(g["needed"])
    assert np.array_equal(a["swarm_active"].cpu().numpy(), g["out_swarm_active"])
    assert np.array_equal(a["swarm_iel"].cpu().numpy(), g["out_swarm_iel"])
    new = g["out_swarm_active"] & ~g["swarm_active"]
    r, t = a["swarm_r"].cpu().numpy()[new], a["swarm_t"].cpu().numpy()[new]
    assert np.all(np.abs(r) <= 0.95) and np.all(np.abs(t) <= 0.95)
    e = g["out_swarm_iel"][new]
    hx, hz = float(M["hx"]), float(M["hz"])
    x, z = a["swarm_x"].cpu().numpy()[new], a["swarm_z"].cpu().numpy()[new]
    assert np.array_equal((x / hx).astype(int), e % 6) and np.array_equal((z / hz).astype(int), e // 6)


def test_population_control_errors(M):
    from meeuuw_b200 import _lib, ops
    g = golden("population")
    nel = 24
    a = _pop_inputs(g)
    counts, offsets, order = ops.bin_particles(nel, a["swarm_active"], a["swarm_iel"])
    # more particles needed than inactive ones: nothing changes, the flag is set
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    before = {k: v.clone() for k, v in a.items()}
    none = torch.zeros_like(counts)
    added = ops.population_control(M["box"], 50, none, offsets, order, a["swarm_active"], a["swarm_iel"],
                                   a["swarm_r"], a["swarm_t"], a["swarm_x"], a["swarm_z"], mat=a["swarm_mat"], err=err)
    assert int(err.item()) & _lib.FLAG_POP_UNAVAILABLE
    assert int(added.item()) == 0
    for k in a:
        assert torch.equal(a[k], before[k]), k
    # a flagged element without active particles
    err.zero_()
    act = a["swarm_active"].clone()
    act[a["swarm_iel"] == 3] = False
    ops.population_control(M["box"], int(g["nparticle_min"]), D(g["nparticle_e"]), offsets, order, act,
                           a["swarm_iel"], a["swarm_r"], a["swarm_t"], a["swarm_x"], a["swarm_z"], err=err,
                           draws=D(np.tile(g["draws"], 8)))
    assert int(err.item()) & _lib.FLAG_POP_MASK_EMPTY


def test_dropin_ls_coefficients_match_reference(M):
    """The drop-ins under the reference's names, with host (numpy) arrays in and out."""
    from meeuuw_b200.dropin import pic_functions as pf
    g = golden("lsq")
    P1 = pf.compute_ls_coefficients_P1(24, g["x_e"], g["z_e"], g["swarm_x"], g["swarm_z"], g["swarm_iel"],
                                       g["swarm_rho"], g["swarm_eta"])
    names = ("rho_a", "rho_b", "rho_c", "eta_a", "eta_b", "eta_c", "rho_min", "rho_max", "eta_min", "eta_max")
    for v, k in zip(P1, names):
        assert isinstance(v, np.ndarray) and rel_err(v, g["out_P1_" + k]) < 1e-12, k
    Q1 = pf.compute_ls_coefficients_Q1(24, g["x_e"], g["z_e"], g["swarm_x"], g["swarm_z"], g["swarm_iel"],
                                       g["swarm_rho"], g["swarm_eta"])
    names = ("rho_a", "rho_b", "rho_c", "rho_d", "eta_a", "eta_b", "eta_c", "eta_d", "rho_min", "rho_max",
             "eta_min", "eta_max")
    for v, k in zip(Q1, names):
        assert rel_err(v, g["out_Q1_" + k]) < 1e-12, k


def test_dropin_population_control_matches_reference(M):
    """Same arguments, same random draws (random.seed), same in-place results as the reference."""
    import io
    import random
    from meeuuw_b200.dropin import pic_functions as pf
    g = golden("population")
    n = len(g["swarm_x"])
    a = {k: g[k].copy() for k in ("swarm_active", "swarm_iel", "swarm_r", "swarm_t", "swarm_x", "swarm_z",
                                  "swarm_u", "swarm_w", "swarm_eta")}
    wf = np.zeros((2, n))
    wf[g["swarm_mat"], np.arange(n)] = 1.0
    paint = np.zeros(n, dtype=np.int32)
    log = io.StringIO()
    random.seed(77)
    pf.population_control(1, M["x_V"], M["z_V"], M["icon_V"], 24, 7, n, g["nparticle_e"], a["swarm_active"],
                          np.arange(n), a["swarm_iel"], a["swarm_r"], a["swarm_t"], a["swarm_x"], a["swarm_z"],
                          a["swarm_u"], a["swarm_w"], np.zeros(n), a["swarm_eta"], wf, np.zeros(n), paint, False, 2,
                          log, "")
    for k in ("swarm_active", "swarm_iel", "swarm_r", "swarm_t"):
        assert np.array_equal(a[k], g["out_" + k]), k
    for k in ("swarm_x", "swarm_z", "swarm_u", "swarm_w", "swarm_eta"):
        assert rel_err(a[k], g["out_" + k]) < 1e-14, k
    assert np.array_equal(np.argmax(wf, axis=0), g["out_swarm_mat"])
    assert (paint == -1).sum() == int(g["needed"])
    assert log.getvalue().split()[2] == str(int(g["needed"]))
