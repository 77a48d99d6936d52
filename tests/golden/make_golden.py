"""Generate golden input/output vectors by running the reference's own functions.

Run in a container that holds the reference checkout (it is read from
``/root/reference``; nothing at test time reads it):

    python tests/golden/make_golden.py          # every fixture
    python tests/golden/make_golden.py lsq      # least-squares fits and population control only

Each case stores its inputs and the reference outputs in ``tests/golden/*.npz``.
Sizes are small so the fixtures stay a few hundred KB.  Inputs are seeded.
"""
import os
import random
import sys
import types

import numpy as np

REF = "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))


def _import_reference():
    # The output writers import matplotlib, which this image does not ship; none
    # of the modules below needs it, but give the import system a stub anyway.
    sys.modules.setdefault("matplotlib", types.ModuleType("matplotlib"))
    sys.path.insert(0, REF)
    import basis_functions_setup_q as bsq
    import basis_functions_setup_Vnodes as bsv
    import build_matrix_energy as bme
    import build_matrix_stokes as bms
    import build_pressure_connectivity as bpc
    import build_pressure_mesh as bpm
    import build_velocity_connectivity as bvc
    import build_velocity_mesh as bvm
    import compute_center_coordinates as ccc
    import cd_u_eta as cde
    import compute_nodal_heat_flux as cnh
    import compute_nodal_pressure as cnp
    import compute_pressure_offset as cpo
    import compute_strain_rate as csr
    import pic_functions as pf
    import postprocessors as pp
    import project_nodal_field_onto_qpoints as pnq
    import quadrature_setup as qs
    import uzawa3_solver_L2 as uz
    return types.SimpleNamespace(**locals())


def mesh_case(R, nelx, nelz, Lx, Lz):
    nn_V = (2 * nelx + 1) * (2 * nelz + 1)
    nn_P = (nelx + 1) * (nelz + 1)
    nel = nelx * nelz
    (hx, hz, nnx, nnz, x_V, z_V, rad_V, theta_V, top_V, bot_V, left_V, right_V, midH, midV, hull,
     cBL, cBR, cTL, cTR) = R.bvm.build_velocity_mesh("box", 9, nn_V, nelx, nelz, Lx, Lz, 0.55, 1, 0, False)
    icon_V, top_e, bot_e, left_e, right_e, _, _ = R.bvc.build_velocity_connectivity(
        "box", 9, nelx, nelz, nnx, nnz, midH, midV)
    icon_P = R.bpc.build_pressure_connectivity("box", nelx, nelz, nel, 4)
    qcoords, qweights, nqe, nq = R.qs.quadrature_setup(3, nel)
    (rq, tq, wq, N_V, N_P, N_T, dNdr_V, dNdt_V, dNdr_P, dNdt_P, dNdr_T, dNdt_T, JxWq, j00, j01, j10,
     j11, area) = R.bsq.basis_functions_setup_q(3, 9, 4, 9, nel, x_V, z_V, icon_V, qcoords, qweights, Lx * Lz)
    r_V = np.array([-1, 1, 1, -1, 0, 1, 0, -1, 0], dtype=np.float64)
    t_V = np.array([-1, -1, 1, 1, -1, 0, 1, 0, 0], dtype=np.float64)
    N_P_n, dNdr_V_n, dNdt_V_n, j00n, j01n, j10n, j11n = R.bsv.basis_functions_setup_Vnodes(
        9, 4, nel, r_V, t_V, x_V, z_V, icon_V)
    l2g = np.zeros((18, nel), dtype=np.int32)
    for iel in range(nel):
        for k1 in range(9):
            for i1 in range(2):
                l2g[2 * k1 + i1, iel] = 2 * icon_V[k1, iel] + i1
    xq = R.pnq.project_nodal_Vfield_onto_qpoints(x_V, 9, nel, 9, N_V, icon_V)
    zq = R.pnq.project_nodal_Vfield_onto_qpoints(z_V, 9, nel, 9, N_V, icon_V)
    return dict(nelx=nelx, nelz=nelz, Lx=Lx, Lz=Lz, hx=hx, hz=hz, x_V=x_V, z_V=z_V, icon_V=icon_V,
                icon_P=icon_P, top_element=top_e, bot_element=bot_e, left_element=left_e,
                right_element=right_e, N_V=N_V, N_P=N_P, dNdr_V=dNdr_V, dNdt_V=dNdt_V, dNdr_P=dNdr_P,
                dNdt_P=dNdt_P, JxWq=JxWq, jcbi00q=j00, jcbi01q=j01, jcbi10q=j10, jcbi11q=j11,
                N_P_n=N_P_n, dNdr_V_n=dNdr_V_n, dNdt_V_n=dNdt_V_n, jcbi00n=j00n, jcbi01n=j01n,
                jcbi10n=j10n, jcbi11n=j11n, local_to_globalV=l2g, xq=xq, zq=zq,
                qcoords=np.array(qcoords), qweights=np.array(qweights),
                cornerBL=cBL, cornerBR=cBR, cornerTL=cTL, cornerTR=cTR)


def free_slip(M, nonzero=False, rng=None):
    nn = len(M["x_V"])
    fix = np.zeros(2 * nn, dtype=bool)
    val = np.zeros(2 * nn)
    x, z, Lx, Lz = M["x_V"], M["z_V"], M["Lx"], M["Lz"]
    fix[0::2] |= (x / Lx < 1e-8) | (x / Lx > 1 - 1e-8)
    fix[1::2] |= (z / Lz < 1e-8) | (z / Lz > 1 - 1e-8)
    if nonzero:
        val[fix] = rng.uniform(-1, 1, size=fix.sum())
    return fix, val


def case_stokes(R, rng, M, blocks, nonzero_bc):
    nel = M["nelx"] * M["nelz"]
    nn = len(M["x_V"])
    nnP = (M["nelx"] + 1) * (M["nelz"] + 1)
    rhoq = rng.uniform(0.9, 1.1, size=(nel, 9))
    etaq = np.exp(rng.uniform(-3, 3, size=(nel, 9)))
    gx = np.full((nel, 9), 0.3)
    gz = np.full((nel, 9), -10.0)
    eta_e = np.exp(rng.uniform(-3, 3, size=nel))
    fix, val = free_slip(M, nonzero_bc, rng)
    out = R.bms.build_matrix_stokes(
        nel * (18 * 18 + 2 * 18 * 4), nel * 324, nel * 16, nel * 72, nel, 9, 9, 4, 2, 2 * nn, nnP, 18,
        M["icon_V"], M["icon_P"], rhoq, etaq, M["JxWq"], M["local_to_globalV"], gx, gz, M["N_V"], M["N_P"],
        M["dNdr_V"], M["dNdt_V"], M["dNdr_P"], M["dNdt_P"], M["jcbi00q"], M["jcbi01q"], M["jcbi10q"],
        M["jcbi11q"], eta_e, 2.0, 1.25, fix, val, M["bot_element"], M["top_element"], False, False, "box",
        np.zeros(nn), False, M["xq"], blocks)
    names = ["VV_Stokes", "rhs_f", "rhs_h", "VV_K", "VV_G", "VV_GT", "VV_M", "VV_M_eta", "VV_H"]
    d = dict(rhoq=rhoq, etaq=etaq, gxq=gx, gzq=gz, eta_e=eta_e, bc_fix_V=fix, bc_val_V=val,
             eta_ref=2.0, L_ref=1.25, blocks=blocks)
    d.update({"out_" + k: v for k, v in zip(names, out)})
    return d


def case_energy(R, rng, M, formulation):
    nel = M["nelx"] * M["nelz"]
    nn = len(M["x_V"])
    f = lambda lo, hi: rng.uniform(lo, hi, size=(nel, 9))
    T = rng.uniform(0, 1, size=nn)
    fix = (M["z_V"] < 1e-8) | (M["z_V"] > M["Lz"] - 1e-8)
    val = np.where(M["z_V"] < 1e-8, 1.0, 0.0)
    args = dict(rhoq=f(0.9, 1.1), etaq=f(0.5, 2), Tq=f(0, 1), uq=f(-50, 50), wq=f(-50, 50),
                hcondq=f(0.5, 1.5), hcapaq=f(0.5, 1.5), alphaq=f(1e-3, 1e-2), hprodq=f(0, 1),
                exxq=f(-1, 1), ezzq=f(-1, 1), exzq=f(-1, 1), dpdxq=f(-1, 1), dpdzq=f(-1, 1))
    dt = 1.7e-3
    VV_T, rhs = R.bme.build_matrix_energy(
        nel * 81, nel, 9, 9, nn, T, M["icon_V"], args["rhoq"], args["etaq"], args["Tq"], args["uq"],
        args["wq"], args["hcondq"], args["hcapaq"], args["alphaq"], args["hprodq"], args["exxq"],
        args["ezzq"], args["exzq"], args["dpdxq"], args["dpdzq"], M["JxWq"], M["N_V"], M["dNdr_V"],
        M["dNdt_V"], M["jcbi00q"], M["jcbi01q"], M["jcbi10q"], M["jcbi11q"], fix, val, dt, formulation, 1.3)
    d = dict(T=T, bc_fix_T=fix, bc_val_T=val, dt=dt, rho0=1.3, formulation=formulation, out_VV_T=VV_T,
             out_rhs=rhs)
    d.update(args)
    return d


def case_pic(R, rng, M):
    nelx, nelz, hx, hz = M["nelx"], M["nelz"], M["hx"], M["hz"]
    nel = nelx * nelz
    ppe = 9
    npart = nel * ppe
    r0 = rng.uniform(-1, 1, npart)
    t0 = rng.uniform(-1, 1, npart)
    iel0 = np.repeat(np.arange(nel), ppe)
    perm = rng.permutation(npart)            # particles are not stored element by element
    r0, t0, iel0 = r0[perm], t0[perm], iel0[perm]
    ex, ez = iel0 % nelx, iel0 // nelx
    x = (ex + (r0 + 1) / 2) * hx
    z = (ez + (t0 + 1) / 2) * hz
    active = rng.uniform(size=npart) > 0.05
    icon = M["icon_V"]
    r, t, iel = R.pf.locate_particles___box(npart, active, x, z, hx, hz, M["x_V"], M["z_V"], icon, nelx)
    nn = len(M["x_V"])
    phi = rng.uniform(0.5, 2.0, nn)
    interp = R.pf.interpolate_field_on_particles(npart, active, r, t, iel, phi, icon)
    rho_p = rng.uniform(0.9, 1.1, npart)
    eta_p = np.exp(rng.uniform(-4, 4, npart))
    d = dict(swarm_x=x, swarm_z=z, swarm_active=active, phi=phi, swarm_rho=rho_p, swarm_eta=eta_p,
             out_r=r, out_t=t, out_iel=iel, out_interp=interp)
    for avg in ("arithmetic", "geometric", "harmonic"):
        re, ee, cnt = R.pf.project_particles_on_elements(nel, npart, active, rho_p, eta_p, iel, avg)
        d[f"out_elem_{avg}_rho"], d[f"out_elem_{avg}_eta"], d[f"out_elem_{avg}_cnt"] = re, ee, cnt
        for fl in (1, 2, 3, 4):
            fn = getattr(R.pf, f"project_particle_field_on_nodes_{fl}")
            d[f"out_nodes{fl}_{avg}"] = fn(nel, nn, npart, active, eta_p, icon, iel, r, t, avg)
    # advection: a smooth velocity field strong enough to push some particles out
    xV, zV = M["x_V"], M["z_V"]
    u = np.sin(np.pi * xV / M["Lx"]) * np.cos(np.pi * zV / M["Lz"]) + 0.3
    w = -np.cos(np.pi * xV / M["Lx"]) * np.sin(np.pi * zV / M["Lz"]) + 0.2
    d.update(u=u, w=w, dt=0.9 * hx)
    for rk in (1, 2, 4):
        xx, zz, aa = x.copy(), z.copy(), active.copy()
        xo, zo, up, wp, ao = R.pf.advect_particles___box(rk, 0.9 * hx, npart, xx, zz, aa, u, w, M["Lx"],
                                                         M["Lz"], hx, hz, nelx, icon, xV, zV)
        d[f"out_adv{rk}_x"], d[f"out_adv{rk}_z"] = xo, zo
        d[f"out_adv{rk}_u"], d[f"out_adv{rk}_w"], d[f"out_adv{rk}_active"] = up, wp, ao
    return d


def case_post(R, rng, M):
    nelx, nelz = M["nelx"], M["nelz"]
    nel = nelx * nelz
    nn = len(M["x_V"])
    nnP = (nelx + 1) * (nelz + 1)
    p = rng.normal(size=nnP)
    u = rng.normal(size=nn)
    w = rng.normal(size=nn)
    T = rng.uniform(0, 1, nn)
    hc = rng.uniform(0.5, 1.5, nn)
    d = dict(p=p, u=u, w=w, T=T, hcond_n=hc)
    icon_V, icon_P = M["icon_V"], M["icon_P"]
    d["out_qV"] = R.pnq.project_nodal_Vfield_onto_qpoints(u, 9, nel, 9, M["N_V"], icon_V)
    d["out_qP"] = R.pnq.project_nodal_Pfield_onto_qpoints(p, 9, nel, 4, M["N_P"], icon_P)
    d["out_qPV"] = R.pnq.project_nodal_Pfield_onto_qpoints(hc, 9, nel, 4, M["N_P"], icon_V)
    for norm in ("surface", "volume"):
        d["out_poff_" + norm] = R.cpo.compute_pressure_offset(
            "box", norm, False, M["top_element"], nel, nelx, 9, M["N_P"], M["JxWq"], p, icon_P,
            np.zeros(nnP), M["xq"], M["Lx"] * M["Lz"])
    d["out_q"] = R.cnp.compute_nodal_pressure(9, nn, icon_V, icon_P, p, M["N_P_n"])
    exx, ezz, exz = R.csr.compute_nodal_strain_rate(icon_V, u, w, nn, 9, nel, M["dNdr_V_n"], M["dNdt_V_n"],
                                                    M["jcbi00n"], M["jcbi01n"], M["jcbi10n"], M["jcbi11n"])
    d.update(out_exx_n=exx, out_ezz_n=ezz, out_exz_n=exz)
    dTdx, dTdz, qx, qz = R.cnh.compute_nodal_heat_flux(icon_V, T, hc, nn, 9, nel, M["dNdr_V_n"], M["dNdt_V_n"],
                                                       M["jcbi00n"], M["jcbi01n"], M["jcbi10n"], M["jcbi11n"])
    d.update(out_dTdx=dTdx, out_dTdz=dTdz, out_qx=qx, out_qz=qz)
    nu = R.pp.compute_Nu(M["Lx"], M["Lz"], M["x_V"], M["z_V"], nel, M["left_element"], M["right_element"],
                         M["top_element"], M["bot_element"], icon_V, T, dTdx, dTdz, 3, list(M["qcoords"]),
                         list(M["qweights"]), hc)
    d["out_Nu_tuple"] = np.array(nu, dtype=np.float64)
    f = lambda: rng.normal(size=(nel, 9))
    uq, wq, Tq, rhoq = f(), f(), f(), f()
    z9 = np.zeros((nel, 9))
    hcapaq, etaq, exxq, ezzq, exzq = f() ** 2 + 1, np.exp(f()), f(), f(), f()
    gxq, gzq = f(), f() - 1
    gq = R.pp.compute_global_quantities(nel, 9, M["xq"], M["zq"], uq, wq, Tq, rhoq, hcapaq, z9, etaq,
                                        exxq, ezzq, exzq, f(), f(), f(), M["Lx"] * M["Lz"], M["JxWq"], gxq, gzq)
    d.update(gq_uq=uq, gq_wq=wq, gq_Tq=Tq, gq_rhoq=rhoq, gq_hcapaq=hcapaq, gq_etaq=etaq, gq_exxq=exxq, gq_ezzq=ezzq,
             gq_exzq=exzq, gq_gxq=gxq, gq_gzq=gzq, out_vrms=gq[0], out_Tavrg=gq[7], out_TM=gq[6],
             out_gq_tuple=np.array(gq, dtype=np.float64))
    return d


def case_solvers(R, rng, n=8):
    """FK-viscosity Stokes system at n x n: direct, uzawa3 and cd_u_eta from the reference."""
    import scipy.sparse as sps
    import scipy.sparse.linalg as sla
    M = mesh_case(R, n, n, 1.0, 1.0)
    nel = n * n
    nn = len(M["x_V"])
    nnP = (n + 1) * (n + 1)
    T = (1 - M["zq"]) + 0.05 * np.cos(np.pi * M["xq"]) * np.sin(np.pi * M["zq"])
    etaq = np.exp(-np.log(1e3) * T)
    eta_e = etaq.mean(axis=1)
    rhoq = 1 - 1e-2 * T
    gx = np.zeros((nel, 9))
    gz = np.full((nel, 9), -1e4 / 1e-2)
    fix, val = free_slip(M)
    args = (nel * 468, nel * 324, nel * 16, nel * 72, nel, 9, 9, 4, 2, 2 * nn, nnP, 18, M["icon_V"],
            M["icon_P"], rhoq, etaq, M["JxWq"], M["local_to_globalV"], gx, gz, M["N_V"], M["N_P"],
            M["dNdr_V"], M["dNdt_V"], M["dNdr_P"], M["dNdt_P"], M["jcbi00q"], M["jcbi01q"], M["jcbi10q"],
            M["jcbi11q"], eta_e, 1.0, 1.0, fix, val, M["bot_element"], M["top_element"], False, False,
            "box", np.zeros(nn), False, M["xq"])
    full = R.bms.build_matrix_stokes(*args, False)
    blk = R.bms.build_matrix_stokes(*args, True)
    from oracle.fe import BoxMesh     # only for the COO index pattern (checked against meeuuw.py loops in tests)
    bm = BoxMesh(n, n)
    II, JJ = bm.coo_stokes()
    A = sps.coo_matrix((full[0], (II, JJ)), shape=(2 * nn + nnP,) * 2).tocsr()
    sol = sla.spsolve(A, np.concatenate([full[1], full[2]]))
    IK, JK = bm.coo_K()
    IG, JG, IGT, JGT = bm.coo_G()
    IM, JM = bm.coo_MP()
    K = sps.coo_matrix((blk[3], (IK, JK)), shape=(2 * nn, 2 * nn)).tocsc()
    G = sps.coo_matrix((blk[4], (IG, JG)), shape=(2 * nn, nnP)).tocsr()
    GT = sps.coo_matrix((blk[5], (IGT, JGT)), shape=(nnP, 2 * nn)).tocsr()
    Mp = sps.coo_matrix((blk[6], (IM, JM)), shape=(nnP, nnP)).tocsc()
    Me = sps.coo_matrix((blk[7], (IM, JM)), shape=(nnP, nnP)).tocsc()
    H = sps.coo_matrix((blk[8], (IGT, JGT)), shape=(nnP, 2 * nn)).tocsr()
    uz = R.uz.uzawa3_solver_L2(K, G, GT, Mp, H, blk[1], blk[2], nnP)
    cd = R.cde.cd_u_eta(K, G, GT, Mp, Me, H, blk[1], blk[2], nnP)
    return dict(etaq=etaq, eta_e=eta_e, rhoq=rhoq, bc_fix_V=fix, out_direct=sol, out_rhs_f=full[1],
                out_uz_V=uz[0], out_uz_P=uz[1], out_uz_it=uz[2], out_cd_V=cd[0], out_cd_P=cd[1], out_cd_it=cd[2],
                out_cd_alpha=cd[5], out_cd_beta=cd[6])


def case_lsq(R, rng, M):
    """Least-squares P1/Q1 fits (pic_functions.py:1098-1285), the driver's limiter loop
    (meeuuw.py:1241-1248, h = hx) and qpoint evaluation (meeuuw.py:1517-1532).  Some particles are
    inactive with x = z = 0 and iel = 0, as advection and locate leave them: the reference's mask
    (swarm_iel == iel) counts them in element 0."""
    nelx, nelz, hx, hz = M["nelx"], M["nelz"], M["hx"], M["hz"]
    nel = nelx * nelz
    ppe = 12
    npart = nel * ppe
    iel = np.repeat(np.arange(nel), ppe).astype(np.int32)
    perm = rng.permutation(npart)
    iel = iel[perm]
    r0, t0 = rng.uniform(-1, 1, npart), rng.uniform(-1, 1, npart)
    x = (iel % nelx + (r0 + 1) / 2) * hx
    z = (iel // nelx + (t0 + 1) / 2) * hz
    active = rng.uniform(size=npart) > 0.06
    x[~active] = 0.0
    z[~active] = 0.0
    iel[~active] = 0
    rho = rng.uniform(0.9, 1.1, npart)
    eta = np.exp(rng.uniform(-2, 2, npart))
    x_e, z_e, _, _ = R.ccc.compute_center_coordinates("box", nel, M["x_V"], M["z_V"], M["icon_V"])
    d = dict(swarm_x=x, swarm_z=z, swarm_iel=iel, swarm_active=active, swarm_rho=rho, swarm_eta=eta, x_e=x_e, z_e=z_e)
    P1 = R.pf.compute_ls_coefficients_P1(nel, x_e, z_e, x, z, iel, rho, eta)
    Q1 = R.pf.compute_ls_coefficients_Q1(nel, x_e, z_e, x, z, iel, rho, eta)
    for k, v in zip(("rho_a", "rho_b", "rho_c", "eta_a", "eta_b", "eta_c", "rho_min", "rho_max", "eta_min",
                     "eta_max"), P1):
        d["out_P1_" + k] = np.array(v)
    for k, v in zip(("rho_a", "rho_b", "rho_c", "rho_d", "eta_a", "eta_b", "eta_c", "eta_d", "rho_min", "rho_max",
                     "eta_min", "eta_max"), Q1):
        d["out_Q1_" + k] = np.array(v)
    lim = {f: (d[f"out_P1_{f}_b"].copy(), d[f"out_P1_{f}_c"].copy()) for f in ("rho", "eta")}
    for e in range(nel):                                              # meeuuw.py:1241-1248
        for f in ("rho", "eta"):
            lim[f][0][e], lim[f][1][e] = R.pf.limiter(d[f"out_P1_{f}_a"][e], lim[f][0][e], lim[f][1][e],
                                                      d[f"out_P1_{f}_min"][e], d[f"out_P1_{f}_max"][e], hx)
    xq, zq = M["xq"], M["zq"]
    for f in ("rho", "eta"):
        d[f"out_P1lim_{f}_b"], d[f"out_P1lim_{f}_c"] = lim[f]
        a_, b_, c_ = d[f"out_P1_{f}_a"], lim[f][0], lim[f][1]
        q = np.zeros((nel, 9))
        for e in range(nel):                                          # meeuuw.py:1517-1523
            for iq in range(9):
                q[e, iq] = a_[e] + b_[e] * (xq[e, iq] - x_e[e]) + c_[e] * (zq[e, iq] - z_e[e])
        d[f"out_P1_{f}q"] = q
        a_, b_, c_, dd = (d[f"out_Q1_{f}_{k}"] for k in "abcd")
        q = np.zeros((nel, 9))
        for e in range(nel):                                          # meeuuw.py:1524-1532
            for iq in range(9):
                q[e, iq] = (a_[e] + b_[e] * (xq[e, iq] - x_e[e]) + c_[e] * (zq[e, iq] - z_e[e])
                            + dd[e] * (xq[e, iq] - x_e[e]) * (zq[e, iq] - z_e[e]))
        d[f"out_Q1_{f}q"] = q
    # the limiter on its own, over slopes that trip both of its branches
    c0 = rng.uniform(0, 1, 64)
    c1, c2 = rng.uniform(-4, 4, 64), rng.uniform(-4, 4, 64)
    c1[:4] = [0.0, -0.0, 1e-3, -1e-3]
    lo, hi = c0 - rng.uniform(0, 0.5, 64), c0 + rng.uniform(0, 0.5, 64)
    L = np.array([R.pf.limiter(c0[i], c1[i], c2[i], lo[i], hi[i], 0.25) for i in range(64)])
    d.update(lim_c0=c0, lim_c1=c1, lim_c2=c2, lim_S=lo, lim_L=hi, lim_h=0.25, out_lim=L)
    return d


def case_population(R, rng, M):
    """population_control (pic_functions.py:1621-1812) after an advection step: counts and element
    indices from the start of the step, positions and active flags after advection.  The reference
    draws r, t with random.uniform(-0.95, 0.95); the uniform numbers it consumes are stored."""
    import io
    nelx, nelz, hx, hz = M["nelx"], M["nelz"], M["hx"], M["hz"]
    nel = nelx * nelz
    per = np.full(nel, 9)
    per[[3, 7, 13, 20]] = [5, 7, 3, 6]                                 # depleted elements
    iel = np.concatenate([np.repeat(np.arange(nel), per), np.zeros(40, dtype=np.int64)]).astype(np.int32)
    npart = len(iel)                                                   # + a pool of 40 inactive particles
    active = np.concatenate([np.ones(per.sum(), dtype=bool), np.zeros(40, dtype=bool)])
    perm = rng.permutation(npart)                                      # not stored element by element
    iel, active = iel[perm], active[perm]
    nparticle_e = np.bincount(iel[active], minlength=nel).astype(np.int32)   # counts at the step start
    step_active = active.copy()
    # advection moved the particles (positions from the step's end, element indices from its start)
    # and pushed two of element 7's and one of element 10's particles out of the box
    r0, t0 = rng.uniform(-0.9, 0.9, npart), rng.uniform(-0.9, 0.9, npart)
    x = (iel % nelx + (r0 + 1) / 2) * hx
    z = (iel // nelx + (t0 + 1) / 2) * hz
    for e, k in ((7, 2), (10, 1)):
        active[np.flatnonzero((iel == e) & active)[:k]] = False
    x[~active] = 0.0
    z[~active] = 0.0
    d = dict(nparticle_min=7, nparticle_e=nparticle_e, step_active=step_active, swarm_active=active.copy(),
             swarm_iel=iel.copy(), swarm_x=x.copy(), swarm_z=z.copy(), swarm_r=rng.uniform(-1, 1, npart),
             swarm_t=rng.uniform(-1, 1, npart), swarm_u=rng.uniform(-1, 1, npart), swarm_w=rng.uniform(-1, 1, npart),
             swarm_eta=np.exp(rng.uniform(-2, 2, npart)), swarm_mat=rng.integers(0, 2, npart).astype(np.int8))
    needed = int(np.maximum(0, 7 - nparticle_e).sum())
    random.seed(77)
    d["draws"] = np.array([random.random() for _ in range(2 * needed)])
    wf = np.zeros((2, npart))
    wf[d["swarm_mat"], np.arange(npart)] = 1.0
    arrs = {k: d[k].copy() for k in ("swarm_active", "swarm_iel", "swarm_r", "swarm_t", "swarm_x", "swarm_z",
                                     "swarm_u", "swarm_w", "swarm_eta")}
    random.seed(77)
    R.pf.population_control(1, M["x_V"], M["z_V"], M["icon_V"], nel, 7, npart, nparticle_e, arrs["swarm_active"],
                            np.arange(npart), arrs["swarm_iel"], arrs["swarm_r"], arrs["swarm_t"], arrs["swarm_x"],
                            arrs["swarm_z"], arrs["swarm_u"], arrs["swarm_w"], np.zeros(npart), arrs["swarm_eta"], wf,
                            np.zeros(npart), np.zeros(npart), False, 2, io.StringIO(), "")
    for k, v in arrs.items():
        d["out_" + k] = v
    d["out_swarm_mat"] = np.argmax(wf, axis=0).astype(np.int8)
    d["needed"] = needed
    return d


def main_lsq():
    """Only the least-squares and population-control fixtures (their own seeded generator)."""
    R = _import_reference()
    rng = np.random.default_rng(20261204)
    M = mesh_case(R, 6, 4, 1.5, 1.0)
    np.savez_compressed(os.path.join(HERE, "lsq.npz"), **case_lsq(R, rng, M))
    np.savez_compressed(os.path.join(HERE, "population.npz"), **case_population(R, rng, M))
    print("wrote lsq.npz, population.npz")


def main():
    R = _import_reference()
    rng = np.random.default_rng(20261203)
    random.seed(1)
    M = mesh_case(R, 6, 4, 1.5, 1.0)
    np.savez_compressed(os.path.join(HERE, "mesh_6x4.npz"), **M)
    cases = {}
    cases["stokes_full_bc"] = case_stokes(R, rng, M, False, True)
    cases["stokes_blocks"] = case_stokes(R, rng, M, True, False)
    cases["energy_BA"] = case_energy(R, rng, M, "BA")
    cases["energy_EBA"] = case_energy(R, rng, M, "EBA")
    cases["pic"] = case_pic(R, rng, M)
    cases["post"] = case_post(R, rng, M)
    for k, v in cases.items():
        np.savez_compressed(os.path.join(HERE, f"{k}.npz"), **v)
    np.savez_compressed(os.path.join(HERE, "solvers_8.npz"), **case_solvers(R, rng, 8))
    write_signatures()
    print("wrote", sorted(os.listdir(HERE)))


def write_signatures():
    """Positional parameter lists of the reference functions the drop-ins replace."""
    import importlib
    import inspect
    import json
    from meeuuw_b200.dropin import TABLE
    sig = {}
    for mod, names in TABLE.items():
        m = importlib.import_module(mod)
        for n in names:
            sig[f"{mod}.{n}"] = list(inspect.signature(getattr(m, n)).parameters)
    with open(os.path.join(HERE, "signatures.json"), "w") as f:
        json.dump(sig, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    if sys.argv[1:] == ["lsq"]:
        main_lsq()
    else:
        main()
