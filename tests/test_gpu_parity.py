"""GPU parity of the CUDA kernels against the reference's golden vectors and the oracle.

Every call goes through the C ABI (``libmeeuuw_b200.so``).  Tolerances:
* element indices, counts, active flags: bit-exact;
* reduced coordinates r, t and arithmetic element means: bit-exact (same operation order);
* other FP64 results: relative 1e-12 (reduction order / BLAS dot order / libm differences);
* FP32 assembly: relative 2e-5 of the largest entry.
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def M():
    from meeuuw_b200 import _lib
    _lib.require_cuda()
    g = golden("mesh_6x4")
    g["box"] = _lib.box_of(6, 4, 1.5, 1.0)
    return g


def D(a, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def H(t):
    return t.detach().cpu().numpy()


def test_locate_interp_bit_exact(M):
    from meeuuw_b200 import ops
    g = golden("pic")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    act = D(g["swarm_active"])
    r, t, iel = ops.locate(M["box"], act, D(g["swarm_x"]), D(g["swarm_z"]), err=err)
    assert np.array_equal(H(iel), g["out_iel"])
    assert np.array_equal(H(r), g["out_r"]) and np.array_equal(H(t), g["out_t"])
    assert int(err.item()) == 0
    (f,) = ops.interp(M["box"], act, r, t, iel, [D(g["phi"])])
    assert rel_err(H(f), g["out_interp"]) < 1e-14


@pytest.mark.parametrize("avg", ["arithmetic", "geometric", "harmonic"])
def test_projections(M, avg):
    from meeuuw_b200 import ops
    g = golden("pic")
    nel = 24
    act = D(g["swarm_active"])
    iel = D(g["out_iel"])
    counts, offsets, order = ops.bin_particles(nel, act, iel)
    assert np.array_equal(H(counts), g[f"out_elem_{avg}_cnt"])
    rho_e, eta_e = ops.project_elements(nel, offsets, order, D(g["swarm_rho"]), D(g["swarm_eta"]), avg)
    assert np.array_equal(H(rho_e), g[f"out_elem_{avg}_rho"])
    assert rel_err(H(eta_e), g[f"out_elem_{avg}_eta"]) < 1e-14
    for fl in (1, 2, 3, 4):
        for exact in (False, True):   # per-element partials / per-node particle-order merge
            (v,) = ops.project_nodes(M["box"], fl, [(D(g["swarm_eta"]), avg)], offsets, order, D(g["out_r"]),
                                     D(g["out_t"]), exact_order=exact)
            ref = g[f"out_nodes{fl}_{avg}"]
            v = H(v)
            ok = ~np.isnan(ref)
            assert np.array_equal(np.isnan(v), np.isnan(ref)), fl
            assert rel_err(v[ok], ref[ok]) < 1e-14, (fl, avg, exact)


@pytest.mark.parametrize("rk", [1, 2, 4])
def test_advect(M, rk):
    from meeuuw_b200 import ops
    g = golden("pic")
    x, z, a = D(g["swarm_x"]), D(g["swarm_z"]), D(g["swarm_active"])
    up = torch.empty_like(x)
    wp = torch.empty_like(x)
    ops.advect(M["box"], rk, float(g["dt"]), x, z, a, D(g["u"]), D(g["w"]), up, wp)
    assert np.array_equal(H(a), g[f"out_adv{rk}_active"])
    for k, v in (("x", x), ("z", z), ("u", up), ("w", wp)):
        assert rel_err(H(v), g[f"out_adv{rk}_{k}"]) < 1e-14, k


def test_nodal_to_qpoints(M):
    from meeuuw_b200 import ops
    from meeuuw_b200._lib import SPACE_Q1, SPACE_Q1_ON_V, SPACE_Q2
    g = golden("post")
    b = M["box"]
    assert rel_err(H(ops.nodal_to_qpoints(b, SPACE_Q2, D(M["N_V"]), D(g["u"]))), g["out_qV"]) < 1e-14
    assert rel_err(H(ops.nodal_to_qpoints(b, SPACE_Q1, D(M["N_P"]), D(g["p"]))), g["out_qP"]) < 1e-14
    assert rel_err(H(ops.nodal_to_qpoints(b, SPACE_Q1_ON_V, D(M["N_P"]), D(g["hcond_n"]))), g["out_qPV"]) < 1e-14


def _stokes_inputs(M, g):
    q = {k: D(g[k]) for k in ("rhoq", "etaq", "gxq", "gzq", "eta_e")}
    for k in ("JxWq", "jcbi00q", "jcbi01q", "jcbi10q", "jcbi11q"):
        q[k] = D(M[k])
    tables = {k: D(M[k]) for k in ("N_V", "N_P", "dNdr_V", "dNdt_V", "dNdr_P", "dNdt_P")}
    return q, tables


@pytest.mark.parametrize("case,blocks", [("stokes_full_bc", False), ("stokes_blocks", True)])
@pytest.mark.parametrize("precision", [0, 1])
def test_assemble_stokes(M, case, blocks, precision):
    from meeuuw_b200 import ops
    g = golden(case)
    q, tables = _stokes_inputs(M, g)
    out = ops.assemble_stokes(M["box"], blocks, precision, q, tables, D(g["bc_fix_V"]), D(g["bc_val_V"]),
                              float(g["eta_ref"]), float(g["L_ref"]))
    tol = TOL if precision == 0 else 2e-5
    names = ["VV_Stokes", "rhs_f", "rhs_h", "VV_K", "VV_G", "VV_GT", "VV_M", "VV_M_eta", "VV_H"]
    for k in names:
        ref = g["out_" + k]
        if ref.size == 0:
            continue
        assert rel_err(H(out[k]).astype(np.float64), ref) < tol, k


@pytest.mark.parametrize("case", ["energy_BA", "energy_EBA"])
@pytest.mark.parametrize("precision", [0, 1])
def test_assemble_energy(M, case, precision):
    from meeuuw_b200 import ops
    g = golden(case)
    q = {k: D(g[k]) for k in ("rhoq", "etaq", "Tq", "uq", "wq", "hcondq", "hcapaq", "alphaq", "hprodq", "exxq", "ezzq",
                              "exzq")}
    for k in ("JxWq", "jcbi00q", "jcbi01q", "jcbi10q", "jcbi11q"):
        q[k] = D(M[k])
    tables = {k: D(M[k]) for k in ("N_V", "dNdr_V", "dNdt_V")}
    VV, rhs = ops.assemble_energy(M["box"], precision, D(g["T"]), q, tables, D(g["bc_fix_T"]), D(g["bc_val_T"]),
                                  float(g["dt"]), float(g["rho0"]), str(g["formulation"]))
    tol = TOL if precision == 0 else 2e-5
    assert rel_err(H(VV).astype(np.float64), g["out_VV_T"]) < tol
    assert rel_err(H(rhs), g["out_rhs"]) < (TOL if precision == 0 else 1e-4)


def test_post(M):
    from meeuuw_b200 import ops
    g = golden("post")
    b = M["box"]
    tables = {k: D(M[k]) for k in ("dNdr_V_n", "dNdt_V_n")}
    for norm in ("surface", "volume"):
        off = ops.pressure_offset(b, norm, D(g["p"]), D(M["N_P"]), D(M["JxWq"]), 1.5)
        ref = float(g["out_poff_" + norm])
        assert abs(off.item() - ref) <= 1e-13 * max(1.0, abs(ref)), norm
    p = D(g["p"])
    q = ops.nodal_pressure(b, p, None, D(M["N_P_n"]), subtract=False)
    assert rel_err(H(q), g["out_q"]) < 1e-14
    e = ops.nodal_strain_rate(b, D(g["u"]), D(g["w"]), tables,
                              jcbi=[D(M[k]) for k in ("jcbi00n", "jcbi01n", "jcbi10n", "jcbi11n")])
    for v, k in zip(e, ("exx_n", "ezz_n", "exz_n")):
        assert rel_err(H(v), g["out_" + k]) < TOL, k
    e0 = ops.nodal_strain_rate(b, D(g["u"]), D(g["w"]), tables)          # uniform-box Jacobian
    assert rel_err(H(e0[0]), g["out_exx_n"]) < TOL
    hf = ops.nodal_heat_flux(b, D(g["T"]), D(g["hcond_n"]), tables)
    for v, k in zip(hf, ("dTdx", "dTdz", "qx", "qz")):
        assert rel_err(H(v), g["out_" + k]) < TOL, k
    nu = ops.compute_nu(b, D(g["T"]), D(g["out_dTdx"]), D(g["out_dTdz"]), D(g["hcond_n"]))
    assert rel_err(H(nu), g["out_Nu_tuple"]) < TOL
    gq = ops.global_quantities(D(g["gq_uq"]), D(g["gq_wq"]), D(g["gq_Tq"]), D(g["gq_rhoq"]), D(M["JxWq"]), 1.5)
    assert abs(gq[0].item() - float(g["out_vrms"])) < 1e-13 * float(g["out_vrms"])
    assert abs(gq[1].item() - float(g["out_Tavrg"])) < 1e-12 * max(1.0, abs(float(g["out_Tavrg"])))


def test_locate_flags_out_of_bounds(M):
    """locate_particles.py:61-64: r outside [-1,1] is reported through the device flag."""
    from meeuuw_b200 import _lib, ops
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    x = torch.tensor([0.3, 1.5], dtype=torch.float64, device="cuda")    # 1.5 == Lx: wraps to next row
    z = torch.tensor([0.3, 0.1], dtype=torch.float64, device="cuda")
    act = torch.ones(2, dtype=torch.bool, device="cuda")
    ops.locate(M["box"], act, x, z, err=err)
    assert int(err.item()) & _lib.FLAG_R_OUT
