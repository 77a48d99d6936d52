"""Pin the oracle against golden vectors produced by the reference's own functions.

Tolerances: element indices and counts exact; FP64 values to a few ulp-scale
relative error (1e-13), since the reference's BLAS dot products may sum in a
different order (and with FMA) than numpy.
"""
import numpy as np
import pytest

from conftest import golden, rel_err
from oracle import assembly, pic, post, solvers
from oracle.fe import BoxMesh

TOL = 1e-13


@pytest.fixture(scope="module")
def mesh():
    return BoxMesh(6, 4, 1.5, 1.0)


def test_mesh_matches_reference(mesh, mesh64):
    g = mesh64
    assert np.array_equal(mesh.icon_V, g["icon_V"])
    assert np.array_equal(mesh.icon_P, g["icon_P"])
    assert np.array_equal(mesh.local_to_globalV, g["local_to_globalV"])
    assert np.array_equal(mesh.x_V, g["x_V"]) and np.array_equal(mesh.z_V, g["z_V"])
    for k in ("top_element", "bot_element", "left_element", "right_element"):
        assert np.array_equal(getattr(mesh, k), g[k])
    for k in ("N_V", "N_P", "dNdr_V", "dNdt_V", "dNdr_P", "dNdt_P", "N_P_n", "dNdr_V_n", "dNdt_V_n"):
        assert rel_err(getattr(mesh, k), g[k]) < TOL, k
    for k in ("JxWq", "jcbi00q", "jcbi01q", "jcbi10q", "jcbi11q", "jcbi00n", "jcbi11n", "xq", "zq"):
        assert rel_err(getattr(mesh, k), g[k]) < TOL, k
    assert (mesh.cornerBL, mesh.cornerBR, mesh.cornerTL, mesh.cornerTR) == tuple(
        int(g[k]) for k in ("cornerBL", "cornerBR", "cornerTL", "cornerTR"))


def test_coo_patterns_match_driver_loops(mesh):
    """II/JJ of meeuuw.py:884-1017, rebuilt with explicit loops."""
    l2g, iP = mesh.local_to_globalV, mesh.icon_P
    II, JJ = [], []
    for iel in range(mesh.nel):
        for ikk in range(18):
            for jkk in range(18):
                II.append(l2g[ikk, iel])
                JJ.append(l2g[jkk, iel])
            for jkk in range(4):
                m2 = iP[jkk, iel] + mesh.Nfem_V
                II += [l2g[ikk, iel], m2]
                JJ += [m2, l2g[ikk, iel]]
    I2, J2 = mesh.coo_stokes()
    assert np.array_equal(I2, II) and np.array_equal(J2, JJ)


def _stokes(mesh, g, blocks):
    m = mesh
    return assembly.build_matrix_stokes(
        0, 0, 0, 0, m.nel, 9, 9, 4, 2, m.Nfem_V, m.Nfem_P, 18, m.icon_V, m.icon_P, g["rhoq"], g["etaq"],
        m.JxWq, m.local_to_globalV, g["gxq"], g["gzq"], m.N_V, m.N_P, m.dNdr_V, m.dNdt_V, m.dNdr_P,
        m.dNdt_P, m.jcbi00q, m.jcbi01q, m.jcbi10q, m.jcbi11q, g["eta_e"], float(g["eta_ref"]),
        float(g["L_ref"]), g["bc_fix_V"], g["bc_val_V"], m.bot_element, m.top_element, False, False,
        "box", None, False, m.xq, blocks)


@pytest.mark.parametrize("case,blocks", [("stokes_full_bc", False), ("stokes_blocks", True)])
def test_build_matrix_stokes(mesh, case, blocks):
    g = golden(case)
    out = _stokes(mesh, g, blocks)
    names = ["VV_Stokes", "rhs_f", "rhs_h", "VV_K", "VV_G", "VV_GT", "VV_M", "VV_M_eta", "VV_H"]
    for k, v in zip(names, out):
        ref = g["out_" + k]
        assert v.shape == ref.shape, k
        assert rel_err(v, ref) < TOL, k


@pytest.mark.parametrize("case", ["energy_BA", "energy_EBA"])
def test_build_matrix_energy(mesh, case):
    g = golden(case)
    m = mesh
    VV, rhs = assembly.build_matrix_energy(
        0, m.nel, 9, 9, m.nn_V, g["T"], m.icon_V, g["rhoq"], g["etaq"], g["Tq"], g["uq"], g["wq"],
        g["hcondq"], g["hcapaq"], g["alphaq"], g["hprodq"], g["exxq"], g["ezzq"], g["exzq"], g["dpdxq"],
        g["dpdzq"], m.JxWq, m.N_V, m.dNdr_V, m.dNdt_V, m.jcbi00q, m.jcbi01q, m.jcbi10q, m.jcbi11q,
        g["bc_fix_T"], g["bc_val_T"], float(g["dt"]), str(g["formulation"]), float(g["rho0"]))
    assert rel_err(VV, g["out_VV_T"]) < TOL
    assert rel_err(rhs, g["out_rhs"]) < TOL


def test_pic_locate_interp(mesh):
    g = golden("pic")
    m = mesh
    n = len(g["swarm_x"])
    r, t, iel = pic.locate_particles___box(n, g["swarm_active"], g["swarm_x"], g["swarm_z"], m.hx, m.hz,
                                           m.x_V, m.z_V, m.icon_V, m.nelx)
    assert np.array_equal(iel, g["out_iel"])               # bit-exact indices
    assert np.array_equal(r, g["out_r"]) and np.array_equal(t, g["out_t"])
    f = pic.interpolate_field_on_particles(n, g["swarm_active"], r, t, iel, g["phi"], m.icon_V)
    assert rel_err(f, g["out_interp"]) < TOL


@pytest.mark.parametrize("avg", ["arithmetic", "geometric", "harmonic"])
def test_pic_projections(mesh, avg):
    g = golden("pic")
    m = mesh
    n = len(g["swarm_x"])
    re, ee, cnt = pic.project_particles_on_elements(m.nel, n, g["swarm_active"], g["swarm_rho"],
                                                    g["swarm_eta"], g["out_iel"], avg)
    assert np.array_equal(cnt, g[f"out_elem_{avg}_cnt"])
    assert np.array_equal(re, g[f"out_elem_{avg}_rho"])     # same summation order -> identical
    assert rel_err(ee, g[f"out_elem_{avg}_eta"]) < TOL
    for fl in (1, 2, 3, 4):
        v = pic.project_particle_field_on_nodes(fl, m.nel, m.nn_V, n, g["swarm_active"], g["swarm_eta"],
                                                m.icon_V, g["out_iel"], g["out_r"], g["out_t"], avg)
        ref = g[f"out_nodes{fl}_{avg}"]
        assert np.array_equal(np.isnan(v), np.isnan(ref))
        ok = ~np.isnan(ref)
        assert rel_err(v[ok], ref[ok]) < TOL, (fl, avg)


@pytest.mark.parametrize("rk", [1, 2, 4])
def test_pic_advect(mesh, rk):
    g = golden("pic")
    m = mesh
    x, z, a = g["swarm_x"].copy(), g["swarm_z"].copy(), g["swarm_active"].copy()
    xo, zo, up, wp, ao = pic.advect_particles___box(rk, float(g["dt"]), len(x), x, z, a, g["u"], g["w"],
                                                     m.Lx, m.Lz, m.hx, m.hz, m.nelx, m.icon_V, m.x_V, m.z_V)
    assert np.array_equal(ao, g[f"out_adv{rk}_active"])
    assert (~ao).sum() > 0
    for k, v in (("x", xo), ("z", zo), ("u", up), ("w", wp)):
        assert rel_err(v, g[f"out_adv{rk}_{k}"]) < TOL, k


def test_post(mesh):
    g = golden("post")
    m = mesh
    assert rel_err(post.project_nodal_field_onto_qpoints(g["u"], m.N_V, m.icon_V), g["out_qV"]) < TOL
    assert rel_err(post.project_nodal_field_onto_qpoints(g["p"], m.N_P, m.icon_P), g["out_qP"]) < TOL
    assert rel_err(post.project_nodal_field_onto_qpoints(g["hcond_n"], m.N_P, m.icon_V), g["out_qPV"]) < TOL
    for norm in ("surface", "volume"):
        v = post.compute_pressure_offset(norm, m.top_element, m.nelx, m.N_P, m.JxWq, g["p"], m.icon_P, m.volume)
        assert abs(v - float(g["out_poff_" + norm])) <= 1e-13 * max(1.0, abs(v))
    assert rel_err(post.compute_nodal_pressure(m.nn_V, m.icon_V, m.icon_P, g["p"], m.N_P_n), g["out_q"]) < TOL
    e = post.compute_nodal_strain_rate(m.icon_V, g["u"], g["w"], m.nn_V, m.dNdr_V_n, m.dNdt_V_n, m.jcbi00n,
                                       m.jcbi01n, m.jcbi10n, m.jcbi11n)
    for v, k in zip(e, ("exx_n", "ezz_n", "exz_n")):
        assert rel_err(v, g["out_" + k]) < 1e-12, k
    hf = post.compute_nodal_heat_flux(m.icon_V, g["T"], g["hcond_n"], m.nn_V, m.dNdr_V_n, m.dNdt_V_n,
                                      m.jcbi00n, m.jcbi01n, m.jcbi10n, m.jcbi11n)
    for v, k in zip(hf, ("dTdx", "dTdz", "qx", "qz")):
        assert rel_err(v, g["out_" + k]) < 1e-12, k
    nu = post.compute_Nu(m.Lx, m.Lz, m.x_V, m.z_V, m.nel, m.left_element, m.right_element, m.top_element,
                         m.bot_element, m.icon_V, g["T"], g["out_dTdx"], g["out_dTdz"], 3, m.qcoords,
                         m.qweights, g["hcond_n"])
    assert rel_err(np.array(nu), g["out_Nu_tuple"]) < 1e-12
    vrms, Tavrg, TM = post.compute_global_quantities(g["gq_uq"], g["gq_wq"], g["gq_Tq"], g["gq_rhoq"],
                                                     m.JxWq, m.volume)
    assert abs(vrms - float(g["out_vrms"])) < 1e-13 * float(g["out_vrms"])
    assert abs(Tavrg - float(g["out_Tavrg"])) < 1e-12 * max(1, abs(float(g["out_Tavrg"])))
    full = post.compute_global_quantities_full(*(g["gq_" + k] for k in ("uq", "wq", "Tq", "rhoq", "hcapaq", "etaq",
                                                                         "exxq", "ezzq", "exzq", "gxq", "gzq")),
                                               m.JxWq, m.volume)
    ref = g["out_gq_tuple"]
    for i, (a, b) in enumerate(zip(full, ref)):
        assert abs(a - b) <= 1e-12 * max(1.0, abs(b)), (i, a, b)


def test_solvers_match_reference():
    g = golden("solvers_8")
    m = BoxMesh(8, 8)
    fix = g["bc_fix_V"]
    zero = np.zeros(m.Nfem_V)
    gx = np.zeros((m.nel, 9))
    gz = np.full((m.nel, 9), -1e6)
    args = (0, 0, 0, 0, m.nel, 9, 9, 4, 2, m.Nfem_V, m.Nfem_P, 18, m.icon_V, m.icon_P, g["rhoq"], g["etaq"],
            m.JxWq, m.local_to_globalV, gx, gz, m.N_V, m.N_P, m.dNdr_V, m.dNdt_V, m.dNdr_P, m.dNdt_P,
            m.jcbi00q, m.jcbi01q, m.jcbi10q, m.jcbi11q, g["eta_e"], 1.0, 1.0, fix, zero, m.bot_element,
            m.top_element, False, False, "box", None, False, m.xq)
    full = assembly.build_matrix_stokes(*args, False)
    assert rel_err(full[1], g["out_rhs_f"]) < TOL
    A = solvers.stokes_full(m, full[0])
    sol = solvers.direct_solve(A, full[1], full[2])
    assert rel_err(sol[:m.Nfem_V], g["out_direct"][:m.Nfem_V]) < 1e-9
    blk = assembly.build_matrix_stokes(*args, True)
    K, G, GT, M, Me, H = solvers.stokes_blocks(m, *blk[3:])
    cd = solvers.cd_u_eta(K, G, GT, M, Me, H, blk[1], blk[2], m.Nfem_P)
    assert cd[2] == int(g["out_cd_it"])
    assert rel_err(cd[0], g["out_cd_V"]) < 1e-9
    it = cd[2]
    assert rel_err(cd[5][:it], g["out_cd_alpha"][:it]) < 1e-6
    assert rel_err(cd[6][:it], g["out_cd_beta"][:it]) < 1e-6
    # uzawa3 does not converge at this viscosity contrast (the reference stops at its
    # 100-iteration cap, uzawa3_solver_L2.py:26); both stagnate at the same distance
    # from the direct solution.
    uz = solvers.uzawa3_solver_L2(K, G, GT, M, H, blk[1], blk[2], m.Nfem_P)
    assert uz[2] == int(g["out_uz_it"]) == 100
    d = g["out_direct"][:m.Nfem_V]
    assert rel_err(uz[0], d) < 1e-3 and rel_err(g["out_uz_V"], d) < 1e-3
