"""Oracle: one reference timestep of the box path, restated with the oracle functions.

Test infrastructure only.  Follows the order of the reference's time loop
(``meeuuw.py:1105-2864``) for the options the box configurations use:
particle interpolation (``:1118-1125``), material model (``:1154``, e.g.
``experiment0.py:230-264``, ``experiment1.py:91-113``), element and nodal
projections (``:1194``, ``:1344-1405``), qpoint fields (``:1503-1590``), Stokes
assembly and solve (``:1705-1851``), pressure normalisation (``:1958-1977``),
nodal pressure (``:2051``), time step (``:2112-2139``), energy assembly and solve
(``:2186-2235``), heat flux and Nu (``:2259-2308``), nodal strain rate
(``:2385``), vrms (``:2512``), advection (``:2726``) and locate (``:2862``).
"""
import time

import numpy as np

from . import assembly, lsq, pic, post, solvers
from .fe import BoxMesh


class OracleModel:
    """FP64 reference-state time stepper for a ``meeuuw_b200.configs.StepConfig``."""

    def __init__(self, cfg, host):
        self.cfg = cfg
        self.mesh = BoxMesh(cfg.nelx, cfg.nelz, cfg.Lx, cfg.Lz)
        m = self.mesh
        h = host
        self.bc_fix_V, self.bc_val_V = h.bc_fix_V.copy(), h.bc_val_V.copy()
        self.bc_fix_T, self.bc_val_T = h.bc_fix_T.copy(), h.bc_val_T.copy()
        self.T = h.T.copy()
        self.x = h.swarm_x.copy()
        self.z = h.swarm_z.copy()
        self.active = h.swarm_active.copy()
        self.mat = h.swarm_mat.copy()
        self.r, self.t, self.iel = pic.locate_particles___box(
            len(self.x), self.active, self.x, self.z, m.hx, m.hz, m.x_V, m.z_V, m.icon_V, m.nelx)
        nn = m.nn_V
        self.exx_n = np.zeros(nn)
        self.ezz_n = np.zeros(nn)
        self.exz_n = np.zeros(nn)
        self.q = np.zeros(nn)
        self.dt1_mem = 1e50
        self.dt2_mem = 1e50
        self.istep = 0
        # solver options (defaults: the reference's): keyword arguments of solvers.cd_u_eta /
        # solvers.uzawa3_solver_L2 and of solvers.energy_solve
        self.stokes_kw = {}
        self.energy_kw = {}
        gx, gz = cfg.gxz
        self.gxq = np.full((m.nel, 9), float(gx))
        self.gzq = np.full((m.nel, 9), float(gz))

    def material(self, swarm_T):
        """experiment0.py:254-264 (Boussinesq + FK) / experiment1.py:104-111 (two materials)."""
        c = self.cfg
        n = len(self.x)
        if c.material == "two_material":
            rho = np.zeros(n)
            eta = np.zeros(n)
            a = self.active
            rho[a] = np.asarray(c.mat_rho)[self.mat[a]]
            eta[a] = np.asarray(c.mat_eta)[self.mat[a]]
            z = np.zeros(n)
            return rho, eta, z, z, z, z
        rho = c.rho0 * (1 - c.alphaT * swarm_T)
        eta = np.exp(-c.fk_gamma * swarm_T) if c.fk_gamma != 0.0 else np.ones(n)
        return (rho, eta, np.full(n, c.hcond), np.full(n, c.hcapa), np.full(n, c.hprod),
                np.full(n, c.alphaT))

    def step(self, solver="direct"):
        c, m = self.cfg, self.mesh
        n = len(self.x)
        out = {}
        # wall time of each phase of the step (s), in the order they run
        self.phase_seconds = times = {}
        clock = [time.perf_counter()]

        def mark(phase):
            t = time.perf_counter()
            times[phase] = times.get(phase, 0.0) + t - clock[0]
            clock[0] = t
        ip = lambda phi: pic.interpolate_field_on_particles(n, self.active, self.r, self.t, self.iel, phi, m.icon_V)
        s_exx, s_ezz, s_exz, s_p = ip(self.exx_n), ip(self.ezz_n), ip(self.exz_n), ip(self.q)
        s_T = ip(self.T) if c.solve_T else np.zeros(n)
        out.update(swarm_exx=s_exx, swarm_ezz=s_ezz, swarm_exz=s_exz, swarm_p=s_p, swarm_T=s_T)
        rho, eta, hcond, hcapa, hprod, alpha = self.material(s_T)
        out.update(swarm_rho=rho, swarm_eta=eta)
        mark("interpolation+material")
        rho_e, eta_e, cnt = pic.project_particles_on_elements(m.nel, n, self.active, rho, eta, self.iel, c.averaging)
        if cnt.min() == 0:
            raise SystemExit("ABORT: an element contains no particle!")   # meeuuw.py:1198-1199
        out.update(rho_e=rho_e, eta_e=eta_e, nparticle_e=cnt)
        proj = lambda phi, avg: pic.project_particle_field_on_nodes(
            c.nodal_projection_type if avg is not None else 2, m.nel, m.nn_V, n, self.active, phi, m.icon_V,
            self.iel, self.r, self.t, avg if avg is not None else "arithmetic")
        out["rho_n"] = proj(rho, "arithmetic")
        out["eta_n"] = proj(eta, c.averaging)
        rhoq = np.repeat(rho_e[:, None], 9, axis=1)                      # "elemental", meeuuw.py:1512
        etaq = np.repeat(eta_e[:, None], 9, axis=1)
        if c.ls_order:                                                   # meeuuw.py:1225-1297, 1517-1562
            x_e, z_e = m.x_V[m.icon_V[8]], m.z_V[m.icon_V[8]]
            coefs, fmin, fmax = lsq.ls_coefficients(c.ls_order, m.nel, x_e, z_e, self.x, self.z, self.iel,
                                                    [rho, eta])
            if c.ls_order == 3:
                coefs = [lsq.limit_p1(cf, lo, hi, m.hx) for cf, lo, hi in zip(coefs, fmin, fmax)]
            out.update(ls_rho=coefs[0], ls_eta=coefs[1])
            if c.particle_rho_projection.startswith("least_squares"):
                rhoq = lsq.ls_to_qpoints(coefs[0], m.xq, m.zq, x_e, z_e)
            if c.particle_eta_projection.startswith("least_squares"):
                etaq = lsq.ls_to_qpoints(coefs[1], m.xq, m.zq, x_e, z_e)
        if c.solve_T:
            hcond_n = proj(hcond, None)
            hcapa_n = proj(hcapa, None)
            hprod_n = proj(hprod, None)
            alpha_n = proj(alpha, None)
            Tq = post.project_nodal_field_onto_qpoints(self.T, m.N_V, m.icon_V)
            hcapaq = post.project_nodal_field_onto_qpoints(hcapa_n, m.N_P, m.icon_V)
            hcondq = post.project_nodal_field_onto_qpoints(hcond_n, m.N_P, m.icon_V)
            hprodq = post.project_nodal_field_onto_qpoints(hprod_n, m.N_P, m.icon_V)
            alphaq = post.project_nodal_field_onto_qpoints(alpha_n, m.N_P, m.icon_V)
            out.update(hcond_n=hcond_n, hcapa_n=hcapa_n, hprod_n=hprod_n, alpha_n=alpha_n)
        else:
            z9 = np.zeros((m.nel, 9))
            Tq = hcapaq = hcondq = hprodq = alphaq = z9
            hcond_n = np.zeros(m.nn_V)
        exxq = post.project_nodal_field_onto_qpoints(self.exx_n, m.N_V, m.icon_V)
        ezzq = post.project_nodal_field_onto_qpoints(self.ezz_n, m.N_V, m.icon_V)
        exzq = post.project_nodal_field_onto_qpoints(self.exz_n, m.N_V, m.icon_V)
        out.update(rhoq=rhoq, etaq=etaq, Tq=Tq)
        mark("projections")
        # Stokes
        blocks = solver in ("cd_u_eta", "uzawa3")
        res = assembly.build_matrix_stokes(
            0, 0, 0, 0, m.nel, 9, 9, 4, 2, m.Nfem_V, m.Nfem_P, 18, m.icon_V, m.icon_P, rhoq, etaq,
            m.JxWq, m.local_to_globalV, self.gxq, self.gzq, m.N_V, m.N_P, m.dNdr_V, m.dNdt_V,
            m.dNdr_P, m.dNdt_P, m.jcbi00q, m.jcbi01q, m.jcbi10q, m.jcbi11q, eta_e, c.eta_ref, m.L_ref,
            self.bc_fix_V, self.bc_val_V, m.bot_element, m.top_element, False, False, "box", None,
            False, m.xq, blocks)
        VV_Stokes, rhs_f, rhs_h = res[0], res[1], res[2]
        out.update(rhs_f=rhs_f, rhs_h=rhs_h)
        mark("stokes assembly")
        A = solvers.stokes_full(m, VV_Stokes if not blocks else self._full_from_blocks(res))
        if solver == "direct":
            sol = solvers.direct_solve(A, rhs_f, rhs_h)
            solV, solP, nit = sol[:m.Nfem_V], sol[m.Nfem_V:], 0
        else:
            K, G, GT, M, Me, H = solvers.stokes_blocks(m, *res[3:])
            if solver == "cd_u_eta":
                solV, solP, nit = solvers.cd_u_eta(K, G, GT, M, Me, H, rhs_f, rhs_h, m.Nfem_P,
                                                   **self.stokes_kw)[:3]
            else:
                solV, solP, nit = solvers.uzawa3_solver_L2(K, G, GT, M, H, rhs_f, rhs_h, m.Nfem_P)[:3]
        mark("stokes solve")
        out["stokes_residual"] = solvers.stokes_relative_residual(A, np.concatenate([solV, solP]), rhs_f, rhs_h)
        out["stokes_iterations"] = nit
        out["solV"], out["solP"] = solV.copy(), solP.copy()
        u, w = solV[0::2].copy(), solV[1::2].copy()
        p = solP * (c.eta_ref / m.L_ref)                                  # meeuuw.py:1848
        offset = post.compute_pressure_offset(c.pressure_normalisation, m.top_element, m.nelx, m.N_P,
                                              m.JxWq, p, m.icon_P, m.volume)
        p = p - offset
        self.q = post.compute_nodal_pressure(m.nn_V, m.icon_V, m.icon_P, p, m.N_P_n)
        T_mem = self.T.copy()
        dt, dt1, dt2 = post.compute_dt(c.CFLnb, m.hx, m.hz, u, w, hcond, hcapa, rho, self.dt1_mem,
                                       self.dt2_mem, c.dt_max, c.solve_T)
        self.dt1_mem, self.dt2_mem = dt1, dt2
        uq = post.project_nodal_field_onto_qpoints(u, m.N_V, m.icon_V)
        wq = post.project_nodal_field_onto_qpoints(w, m.N_V, m.icon_V)
        out.update(u=u, w=w, p=p, q=self.q.copy(), dt=dt, pressure_offset=offset)
        mark("pressure, dt")
        Nu = np.nan
        if c.solve_T:
            z9 = np.zeros((m.nel, 9))
            VV_T, rhs_T = assembly.build_matrix_energy(
                0, m.nel, 9, 9, m.nn_V, T_mem, m.icon_V, rhoq, etaq, Tq, uq, wq, hcondq, hcapaq, alphaq,
                hprodq, exxq, ezzq, exzq, z9, z9, m.JxWq, m.N_V, m.dNdr_V, m.dNdt_V, m.jcbi00q,
                m.jcbi01q, m.jcbi10q, m.jcbi11q, self.bc_fix_T, self.bc_val_T, dt, c.formulation, c.rho0)
            mark("energy assembly")
            self.T = solvers.energy_solve(m, VV_T, rhs_T, **self.energy_kw)
            mark("energy solve")
            dTdx, dTdz, qx, qz = post.compute_nodal_heat_flux(
                m.icon_V, self.T, hcond_n, m.nn_V, m.dNdr_V_n, m.dNdt_V_n, m.jcbi00n, m.jcbi01n,
                m.jcbi10n, m.jcbi11n)
            Nu = post.compute_Nu(m.Lx, m.Lz, m.x_V, m.z_V, m.nel, m.left_element, m.right_element,
                                 m.top_element, m.bot_element, m.icon_V, self.T, dTdx, dTdz, 3,
                                 m.qcoords, m.qweights, hcond_n)[-1]
            out.update(T=self.T.copy(), rhs_T=rhs_T)
        self.exx_n, self.ezz_n, self.exz_n = post.compute_nodal_strain_rate(
            m.icon_V, u, w, m.nn_V, m.dNdr_V_n, m.dNdt_V_n, m.jcbi00n, m.jcbi01n, m.jcbi10n, m.jcbi11n)
        Tq_new = Tq
        vrms, Tavrg, _ = post.compute_global_quantities(uq, wq, Tq_new, rhoq, m.JxWq, m.volume)
        out.update(vrms=vrms, Nu=Nu, exx_n=self.exx_n.copy())
        mark("heat flux, Nu, strain rate, vrms")
        _, _, up, wp, _ = pic.advect_particles___box(c.RKorder, dt, n, self.x, self.z, self.active, u, w, m.Lx,
                                                     m.Lz, m.hx, m.hz, m.nelx, m.icon_V, m.x_V, m.z_V)
        if c.allow_population_control and c.RKorder > 0:                # meeuuw.py:2846-2850
            need = int(np.maximum(0, c.nmin - cnt).sum())
            draws = lsq.splitmix_u01(c.population_seed(self.istep), 2 * need)
            out["population_added"] = lsq.population_control(
                m.x_V, m.z_V, m.icon_V, m.nel, c.nmin, cnt, self.active, self.iel, self.r, self.t, self.x, self.z,
                up, wp, eta, self.mat, draws)
        self.r, self.t, self.iel = pic.locate_particles___box(
            n, self.active, self.x, self.z, m.hx, m.hz, m.x_V, m.z_V, m.icon_V, m.nelx)
        if not pic.locate_bounds_ok(self.r, self.t):
            raise SystemExit("r value out of bounds")
        mark("advection+locate")
        out.update(swarm_x=self.x.copy(), swarm_z=self.z.copy(), swarm_iel=self.iel.copy())
        self.istep += 1
        return out

    def _full_from_blocks(self, res):
        nel = self.mesh.nel
        K = res[3].reshape(nel, 18, 18)
        G = res[4].reshape(nel, 18, 4)
        full = np.zeros((nel, 18, 26))
        full[:, :, :18] = K
        full[:, :, 18::2] = G
        full[:, :, 19::2] = G
        return full.reshape(-1)
