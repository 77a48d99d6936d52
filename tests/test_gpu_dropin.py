"""The drop-in functions, called with the reference's positional arguments (numpy in, numpy out, as
the reference's driver calls them), against outputs of the reference's own functions (golden
fixtures), and once more with CUDA tensors (device in, device out, no host copies).

Tolerances as in the kernel parity tests: indices, counts, flags and reduced coordinates
bit-exact; FP64 sums 1e-12 relative (summation order); the matrix-free solver against the
reference's direct solution at the solver's 1e-8 relative residual.
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def m():
    from meeuuw_b200 import _lib
    _lib.require_cuda()
    return golden("mesh_6x4")


def _stokes_args(m, g, blocks):
    nel = 24
    nfv, nfp = len(g["bc_fix_V"]), len(g["out_rhs_h"])
    return (0, 0, 0, 0, nel, 9, 9, 4, 2, nfv, nfp, 18, m["icon_V"], m["icon_P"], g["rhoq"], g["etaq"], m["JxWq"],
            m["local_to_globalV"], g["gxq"], g["gzq"], m["N_V"], m["N_P"], m["dNdr_V"], m["dNdt_V"], m["dNdr_P"],
            m["dNdt_P"], m["jcbi00q"], m["jcbi01q"], m["jcbi10q"], m["jcbi11q"], g["eta_e"], float(g["eta_ref"]),
            float(g["L_ref"]), g["bc_fix_V"], g["bc_val_V"], m["bot_element"], m["top_element"], False, False, "box",
            None, False, m["xq"], blocks)


@pytest.mark.parametrize("case,blocks", [("stokes_full_bc", False), ("stokes_blocks", True)])
def test_build_matrix_stokes(m, case, blocks):
    from meeuuw_b200.dropin.build_matrix_stokes import build_matrix_stokes
    g = golden(case)
    out = build_matrix_stokes(*_stokes_args(m, g, blocks))
    names = ("VV_Stokes", "rhs_f", "rhs_h", "VV_K", "VV_G", "VV_GT", "VV_M", "VV_M_eta", "VV_H")
    assert len(out) == 9
    for k, v in zip(names, out):
        assert isinstance(v, np.ndarray) and v.dtype == np.float64
        ref = g["out_" + k]
        assert v.shape == ref.shape, k
        if ref.size:
            assert rel_err(v, ref) < TOL, k


@pytest.mark.parametrize("form", ["BA", "EBA"])
def test_build_matrix_energy(m, form):
    from meeuuw_b200.dropin.build_matrix_energy import build_matrix_energy
    g = golden(f"energy_{form}")
    args = (24 * 81, 24, 9, 9, 117, g["T"], m["icon_V"], g["rhoq"], g["etaq"], g["Tq"], g["uq"], g["wq"], g["hcondq"],
            g["hcapaq"], g["alphaq"], g["hprodq"], g["exxq"], g["ezzq"], g["exzq"], g["dpdxq"], g["dpdzq"], m["JxWq"],
            m["N_V"], m["dNdr_V"], m["dNdt_V"], m["jcbi00q"], m["jcbi01q"], m["jcbi10q"], m["jcbi11q"], g["bc_fix_T"],
            g["bc_val_T"], float(g["dt"]), str(g["formulation"]), float(g["rho0"]))
    VV, rhs = build_matrix_energy(*args)
    assert rel_err(VV, g["out_VV_T"]) < TOL and rel_err(rhs, g["out_rhs"]) < TOL


def test_pic_functions(m):
    from meeuuw_b200.dropin import locate_particles as lp
    from meeuuw_b200.dropin import pic_functions as pf
    g = golden("pic")
    n = len(g["swarm_x"])
    hx, hz = float(m["hx"]), float(m["hz"])
    r, t, iel = pf.locate_particles___box(n, g["swarm_active"], g["swarm_x"], g["swarm_z"], hx, hz, m["x_V"],
                                          m["z_V"], m["icon_V"], 6)
    assert np.array_equal(iel, g["out_iel"]) and np.array_equal(r, g["out_r"]) and np.array_equal(t, g["out_t"])
    r2, t2, iel2 = lp.locate_particles("box", n, g["swarm_active"], g["swarm_x"], g["swarm_z"], None, None, hx, hz, 0,
                                       0, m["x_V"], m["z_V"], None, None, m["icon_V"], 6, 0)
    assert np.array_equal(iel2, g["out_iel"]) and np.array_equal(r2, g["out_r"])
    phi = pf.interpolate_field_on_particles(n, g["swarm_active"], r, t, iel, g["phi"], m["icon_V"])
    assert rel_err(phi, g["out_interp"]) < 1e-14
    for avg in ("arithmetic", "geometric", "harmonic"):
        rho_e, eta_e, cnt = pf.project_particles_on_elements(24, n, g["swarm_active"], g["swarm_rho"], g["swarm_eta"],
                                                             iel, avg)
        assert np.array_equal(cnt, g[f"out_elem_{avg}_cnt"]) and cnt.dtype == np.int32
        assert np.array_equal(rho_e, g[f"out_elem_{avg}_rho"])
        assert rel_err(eta_e, g[f"out_elem_{avg}_eta"]) < 1e-14
        for fl in (1, 2, 3, 4):
            fn = getattr(pf, f"project_particle_field_on_nodes_{fl}")
            v = fn(24, 117, n, g["swarm_active"], g["swarm_eta"], m["icon_V"], iel, r, t, avg)
            ref = g[f"out_nodes{fl}_{avg}"]
            ok = ~np.isnan(ref)
            assert np.array_equal(np.isnan(v), np.isnan(ref))
            assert rel_err(v[ok], ref[ok]) < 1e-14, (fl, avg)


@pytest.mark.parametrize("rk", [1, 2, 4])
def test_advect_in_place(m, rk):
    from meeuuw_b200.dropin import pic_functions as pf
    g = golden("pic")
    n = len(g["swarm_x"])
    x, z, a = g["swarm_x"].copy(), g["swarm_z"].copy(), g["swarm_active"].copy()
    out = pf.advect_particles___box(rk, float(g["dt"]), n, x, z, a, g["u"], g["w"], float(m["Lx"]), float(m["Lz"]),
                                    float(m["hx"]), float(m["hz"]), 6, m["icon_V"], m["x_V"], m["z_V"])
    assert out[0] is x and out[1] is z and out[4] is a          # the reference mutates and returns them
    assert np.array_equal(a, g[f"out_adv{rk}_active"])
    assert rel_err(x, g[f"out_adv{rk}_x"]) < 1e-14 and rel_err(z, g[f"out_adv{rk}_z"]) < 1e-14
    assert rel_err(out[2], g[f"out_adv{rk}_u"]) < 1e-13 and rel_err(out[3], g[f"out_adv{rk}_w"]) < 1e-13


def test_post_functions(m):
    from meeuuw_b200.dropin import (compute_nodal_heat_flux, compute_nodal_pressure, compute_pressure_offset,
                                    compute_strain_rate, postprocessors, project_nodal_field_onto_qpoints as pq)
    g = golden("post")
    assert rel_err(pq.project_nodal_Vfield_onto_qpoints(g["u"], 9, 24, 9, m["N_V"], m["icon_V"]), g["out_qV"]) < TOL
    assert rel_err(pq.project_nodal_Pfield_onto_qpoints(g["p"], 9, 24, 4, m["N_P"], m["icon_P"]), g["out_qP"]) < TOL
    assert rel_err(pq.project_nodal_Pfield_onto_qpoints(g["hcond_n"], 9, 24, 4, m["N_P"], m["icon_V"]),
                   g["out_qPV"]) < TOL
    for norm in ("surface", "volume"):
        off = compute_pressure_offset.compute_pressure_offset("box", norm, False, m["top_element"], 24, 6, 9, m["N_P"],
                                                              m["JxWq"], g["p"], m["icon_P"], None, m["xq"],
                                                              float(m["Lx"] * m["Lz"]))
        ref = float(g[f"out_poff_{norm}"])
        assert abs(off - ref) <= TOL * max(1.0, abs(ref))
    assert compute_pressure_offset.compute_pressure_offset("box", "none", False, None, 24, 6, 9, None, None, None,
                                                           None, None, None, 1.0) == 0.
    with pytest.raises(ValueError):
        compute_pressure_offset.compute_pressure_offset("box", "bogus", False, None, 24, 6, 9, None, None, None, None,
                                                        None, None, 1.0)
    q = compute_nodal_pressure.compute_nodal_pressure(9, 117, m["icon_V"], m["icon_P"], g["p"], m["N_P_n"])
    assert rel_err(q, g["out_q"]) < TOL
    e = compute_strain_rate.compute_nodal_strain_rate(m["icon_V"], g["u"], g["w"], 117, 9, 24, m["dNdr_V_n"],
                                                      m["dNdt_V_n"], m["jcbi00n"], m["jcbi01n"], m["jcbi10n"],
                                                      m["jcbi11n"])
    for v, k in zip(e, ("exx_n", "ezz_n", "exz_n")):
        assert rel_err(v, g["out_" + k]) < TOL, k
    hf = compute_nodal_heat_flux.compute_nodal_heat_flux(m["icon_V"], g["T"], g["hcond_n"], 117, 9, 24, m["dNdr_V_n"],
                                                         m["dNdt_V_n"], m["jcbi00n"], m["jcbi01n"], m["jcbi10n"],
                                                         m["jcbi11n"])
    for v, k in zip(hf, ("dTdx", "dTdz", "qx", "qz")):
        assert rel_err(v, g["out_" + k]) < TOL, k
    nu = postprocessors.compute_Nu(float(m["Lx"]), float(m["Lz"]), m["x_V"], m["z_V"], 24, m["left_element"],
                                   m["right_element"], m["top_element"], m["bot_element"], m["icon_V"], g["T"],
                                   g["out_dTdx"], g["out_dTdz"], 3, list(m["qcoords"]), list(m["qweights"]),
                                   g["hcond_n"])
    assert len(nu) == 13 and rel_err(np.array(nu), g["out_Nu_tuple"]) < TOL
    z9 = np.zeros((24, 9))
    gq = postprocessors.compute_global_quantities(24, 9, m["xq"], m["zq"], g["gq_uq"], g["gq_wq"], g["gq_Tq"],
                                                  g["gq_rhoq"], g["gq_hcapaq"], z9, g["gq_etaq"], g["gq_exxq"],
                                                  g["gq_ezzq"], g["gq_exzq"], z9, z9, z9, float(m["Lx"] * m["Lz"]),
                                                  m["JxWq"], g["gq_gxq"], g["gq_gzq"])
    for i, (a, b) in enumerate(zip(gq, g["out_gq_tuple"])):
        assert abs(a - b) <= TOL * max(1.0, abs(b)), i


def test_device_tensors_stay_on_device(m):
    """CUDA tensors in -> CUDA tensors out, and the in-place contract holds on device memory."""
    from meeuuw_b200.dropin import pic_functions as pf
    g = golden("pic")
    n = len(g["swarm_x"])
    d = lambda a: torch.as_tensor(a).cuda()
    x, z, a = d(g["swarm_x"]), d(g["swarm_z"]), d(g["swarm_active"])
    xp = x.data_ptr()
    r, t, iel = pf.locate_particles___box(n, a, x, z, float(m["hx"]), float(m["hz"]), d(m["x_V"]), d(m["z_V"]),
                                          d(m["icon_V"]), 6)
    assert r.is_cuda and iel.is_cuda and np.array_equal(iel.cpu().numpy(), g["out_iel"])
    out = pf.advect_particles___box(4, float(g["dt"]), n, x, z, a, d(g["u"]), d(g["w"]), float(m["Lx"]),
                                    float(m["Lz"]), float(m["hx"]), float(m["hz"]), 6, d(m["icon_V"]), d(m["x_V"]),
                                    d(m["z_V"]))
    assert out[0] is x and x.data_ptr() == xp
    assert rel_err(x.cpu().numpy(), g["out_adv4_x"]) < 1e-14
    assert np.array_equal(a.cpu().numpy(), g["out_adv4_active"])


def test_schur_solvers_against_direct():
    """build_matrix_stokes (blocks) -> SciPy matrices as the driver builds them -> cd_u_eta drop-in."""
    from oracle import solvers
    from oracle.fe import BoxMesh
    from meeuuw_b200.dropin.build_matrix_stokes import build_matrix_stokes
    from meeuuw_b200.dropin.cd_u_eta import cd_u_eta
    g = golden("solvers_8")
    mm = BoxMesh(8, 8)
    fix = g["bc_fix_V"]
    gx, gz = np.zeros((mm.nel, 9)), np.full((mm.nel, 9), -1e6)
    args = (0, 0, 0, 0, mm.nel, 9, 9, 4, 2, mm.Nfem_V, mm.Nfem_P, 18, mm.icon_V, mm.icon_P, g["rhoq"], g["etaq"],
            mm.JxWq, mm.local_to_globalV, gx, gz, mm.N_V, mm.N_P, mm.dNdr_V, mm.dNdt_V, mm.dNdr_P, mm.dNdt_P,
            mm.jcbi00q, mm.jcbi01q, mm.jcbi10q, mm.jcbi11q, g["eta_e"], 1.0, 1.0, fix, np.zeros(mm.Nfem_V),
            mm.bot_element, mm.top_element, False, False, "box", None, False, mm.xq, True)
    blk = build_matrix_stokes(*args)
    K, G, GT, M, Me, H = solvers.stokes_blocks(mm, *blk[3:])
    V, P, it, xiV, xiP, alpha, beta = cd_u_eta(K, G, GT, M, Me, H, blk[1], blk[2], mm.Nfem_P)
    d = g["out_direct"]
    # the forward error a 1e-8 relative residual allows at this viscosity contrast
    assert rel_err(V, d[:mm.Nfem_V]) < 2e-5
    assert len(xiV) == 100 and 0 < it <= 100 and np.all(xiV[:it] > 0) and np.all(xiV[it:] == 0)
    # warm start from the solution: converges at once
    V2, P2, it2, *_ = cd_u_eta(K, G, GT, M, Me, H, blk[1], blk[2], mm.Nfem_P, V0=V, P0=P)
    assert it2 < it and rel_err(V2, V) < 1e-6
    # matrices that were not assembled by the drop-in are refused
    with pytest.raises(RuntimeError):
        cd_u_eta(K * 2.0, G, GT, M, Me, H, blk[1], blk[2], mm.Nfem_P)
