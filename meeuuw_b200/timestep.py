"""One model's timestep, entirely on the GPU, in the order of the reference's time loop.

meeuuw.py:1105-2864 (box path): particle interpolation + material model (:1118-1154),
element and nodal projections (:1194, :1344-1405), qpoint fields (:1503-1590), Stokes
right-hand side and solve (:1705-1851), pressure normalisation and nodal pressure (:1958-2051),
time step (:2112-2139), energy assembly and solve (:2186-2235), heat flux and Nu (:2259-2308),
nodal strain rate (:2385), vrms (:2512), advection (:2726) and locate (:2862).

All state lives in device tensors allocated once; a step launches only this library's kernels
(plus the solver's host-driven convergence checks).  Scalars (dt, vrms, Nu, solver statistics)
stay on the device until `diagnostics()` reads them.
"""
import torch

from . import _lib as L
from . import configs, fe_tables, ops
from .stokes import StokesSolver

f64 = torch.float64


class GPUModel:
    def __init__(self, cfg, host=None, stokes="mixed", scheme="cd_u_eta", tol=1e-8, warm_start="previous",
                 inner_rtol=None, energy="matrix_free", device="cuda"):
        L.require_cuda()
        self.cfg = cfg
        host = host if host is not None else configs.build_host_model(cfg)
        self.box = box = L.box_of(cfg.nelx, cfg.nelz, cfg.Lx, cfg.Lz)
        self.nel = nel = cfg.nel
        self.nn = nn = (2 * cfg.nelx + 1) * (2 * cfg.nelz + 1)
        self.np_ = npp = (cfg.nelx + 1) * (cfg.nelz + 1)
        self.npart = npart = len(host.swarm_x)
        self.L_ref = (cfg.Lx + cfg.Lz) / 2
        self.volume = cfg.Lx * cfg.Lz
        self.stokes_precision, self.scheme, self.tol, self.warm_start = stokes, scheme, tol, warm_start
        # inner multigrid-PCG tolerance: loose under FP64 refinement (mixed; 2e-2 is the fastest
        # setting whose vrms stays within 1e-7 of the FP64 solve at 512x512); without refinement
        # (plain FP64) the loosest setting with which the Schur iteration converges on every step,
        # the cold start included: on the 512x512 FK model 1e-9 does (93 ms per warm step, 97 at
        # 1e-10), 1e-8 ... 1e-7 stall at the first step (200 Schur iterations, residual ~1e-8 to
        # 1e-7) although they would be faster on warm steps (86 ... 77 ms) (measured)
        # The inexact Schur iteration stalls near its inner solves' accuracy, so a tighter outer
        # tolerance tightens the FP64 inner one with it (10x below; at an outer 1e-10, inner 1e-9
        # stalls the 512x512 cold start at 200 iterations)
        if inner_rtol is None:
            inner_rtol = 2e-2 if stokes == "mixed" else min(1e-9, 0.1 * tol)
        self.inner_rtol = inner_rtol
        D = lambda a, dt=None: torch.as_tensor(a, dtype=dt).to(device).contiguous()
        self.tables = fe_tables.device_tables(device)
        self.geo = fe_tables.uniform_geometry(nel, box.hx, box.hz, device)
        E = lambda *s, dt=f64: torch.empty(*s, dtype=dt, device=device)
        Z = lambda *s, dt=f64: torch.zeros(*s, dtype=dt, device=device)
        # swarm
        self.x, self.z = D(host.swarm_x, f64), D(host.swarm_z, f64)
        self.active = D(host.swarm_active, torch.bool)
        self.mat = D(host.swarm_mat, torch.int8)
        self.r, self.t, self.iel = E(npart), E(npart), E(npart, dt=torch.int32)
        self.props = {k: E(npart) for k in ("exx", "ezz", "exz", "p", "T", "rho", "eta", "hcond", "hcapa", "hprod",
                                            "alpha")}
        self.up, self.wp = E(npart), E(npart)
        self.counts, self.offsets, self.order = E(nel, dt=torch.int32), E(nel + 1, dt=torch.int32), E(npart,
                                                                                                           dt=torch.int32)
        self.err = Z(1, dt=torch.int32)
        # nodal / elemental / qpoint fields
        self.T = D(host.T, f64)
        self.exx_n, self.ezz_n, self.exz_n, self.q = Z(nn), Z(nn), Z(nn), Z(nn)
        self.u, self.w, self.p = Z(nn), Z(nn), Z(npp)
        self.rho_e, self.eta_e = E(nel), E(nel)
        self.nodal = {k: E(nn) for k in ("rho", "eta", "hcond", "hcapa", "hprod", "alpha")}
        self.qf = {k: E(nel, 9) for k in ("rhoq", "etaq", "Tq", "hcapaq", "hcondq", "hprodq", "alphaq", "uq", "wq")}
        if cfg.formulation == "EBA":
            for k in ("exxq", "ezzq", "exzq"):
                self.qf[k] = E(nel, 9)
        gx, gz = cfg.gxz
        self.gxq = torch.full((nel, 9), float(gx), dtype=f64, device=device)
        self.gzq = torch.full((nel, 9), float(gz), dtype=f64, device=device)
        self.bc_fix_V, self.bc_val_V = D(host.bc_fix_V, torch.bool), D(host.bc_val_V, f64)
        self.zero_bc_values = not bool((host.bc_val_V != 0).any())
        self.bc_fix_T, self.bc_val_T = D(host.bc_fix_T, torch.bool), D(host.bc_val_T, f64)
        self.rhs_f, self.rhs_h = E(2 * nn), E(npp)
        self.solV, self.solP = Z(2 * nn), Z(npp)
        # energy operator: "matrix_free" (Gauss-point coefficients, 360 B per element, no element
        # matrices) or "matrices" (the reference's VV_T, 648 B per element, regrouped per solve)
        if energy not in ("matrix_free", "matrices"):
            raise ValueError(f"energy must be 'matrix_free' or 'matrices', not {energy!r}")
        self.energy_form = energy
        self.rhs_T = E(nn)
        if energy == "matrix_free":
            self.VV_T = None
            self.energy_op = torch.empty(L.lib().mw_energy_op_bytes(box), dtype=torch.uint8, device=device)
        else:
            self.VV_T, self.energy_op = E(nel * 81), None
        self.hf = [E(nn) for _ in range(4)]
        # device scalars
        self.dt_state = torch.tensor([1e50, 1e50], dtype=f64, device=device)
        self.dt_out = Z(3)
        self.offset = Z(1)
        self.nu_out = Z(13)
        self.gq_out = Z(3)
        self.material = ops.material_struct(cfg)
        precs = ("f64",) if stokes == "f64" else ("f32",)
        # Smoothing per arithmetic: an FP64 V-cycle is apply-bound, so one Chebyshev step per sweep
        # with more PCG iterations is faster; in FP32 two steps per sweep pay for themselves, and six
        # warm-started power iterations per viscosity update (three in FP64) give the Chebyshev
        # intervals that make the mixed solve fastest (measured on the 512x512 FK step).
        self.solver = StokesSolver(box, self.bc_fix_V, eta_ref=cfg.eta_ref, L_ref=self.L_ref, precisions=precs,
                                   cheb_degree=1 if stokes == "f64" else 2,
                                   power_iters_warm=3 if stokes == "f64" else 6)
        self.last_solve = {}
        self.istep = 0
        self.guess = None      # optional callable(model) -> (solV, solP) used as the Stokes initial guess
        # extra mw_solve_params fields: six Chebyshev steps on the M_eta preconditioner of the
        # Schur complement leave the outer iteration counts of the FK step unchanged (vs 12)
        self.solve_kw = dict(mass_iters=6)
        # the mixed arm's refinement sweeps aim at a tenth of the tolerance once they are close
        # (sweep_target): 13 instead of 15 Schur iterations on the 512x512 FK step, vrms within 6e-8
        # of a tight FP64 solve (measured)
        if stokes == "mixed":
            self.solve_kw["sweep_target"] = 0.1
        # energy BiCGSTAB tolerance (relative residual): T within 1e-9 of a direct solve
        self.energy_rtol = 1e-10
        self.graph = None      # recorded time step (capture_step)
        if cfg.ls_order:       # least-squares projections: qpoint coordinates, bins of every particle
            xV = torch.as_tensor(host.x_V, dtype=f64, device=device)
            zV = torch.as_tensor(host.z_V, dtype=f64, device=device)
            self.xq, self.zq = E(nel, 9), E(nel, 9)
            ops.nodal_to_qpoints(box, L.SPACE_Q2, self.tables["N_V"], xV, self.xq)
            ops.nodal_to_qpoints(box, L.SPACE_Q2, self.tables["N_V"], zV, self.zq)
            self.every = torch.ones(npart, dtype=torch.uint8, device=device)
            self.ls_bins = (E(nel, dt=torch.int32), E(nel + 1, dt=torch.int32), E(npart, dt=torch.int32))
        if cfg.allow_population_control:
            self.pc_added = Z(1, dt=torch.int32)
        self._replayed = False
        self._capturing = False
        ops.locate(box, self.active, self.x, self.z, self.r, self.t, self.iel, self.err)

    # ------------------------------------------------------------------------------------------
    def stokes_inputs(self):
        q = dict(rhoq=self.qf["rhoq"], etaq=self.qf["etaq"], gxq=self.gxq, gzq=self.gzq, eta_e=self.eta_e)
        q.update(self.geo)
        return q

    def enable_phase_timing(self, on=True):
        """Record CUDA events between the phases of each step (read with phase_times())."""
        self._phases = [] if on else None

    def _mark(self, name):
        if getattr(self, "_phases", None) is not None:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            self._phases.append((name, ev))

    def phase_times(self):
        """{phase: milliseconds} summed over the steps recorded since enable_phase_timing()."""
        ph = getattr(self, "_phases", None) or []
        torch.cuda.synchronize()
        out = {}
        for (n0, e0), (n1, e1) in zip(ph, ph[1:]):
            if n0 == "end":
                continue
            out[n0] = out.get(n0, 0.0) + e0.elapsed_time(e1)
        return out

    def capture_step(self):
        """Record one whole time step as a CUDA graph; later step() calls replay it (one launch per
        step, no host synchronisation).  The Stokes and energy solves record their loops as
        conditional nodes; their outcomes are read from the device by diagnostics().  Runs one
        eager step first when none has run (it sizes every workspace).  A guess hook runs device
        work between the solves' inputs and the solve, so it can only be left out of the record
        while it is idle (``hook.idle()`` true: the solve starts from the previous solution); a step
        whose hook is not idle runs eagerly, with the hook, and later idle steps replay again."""
        if self.guess is not None and not self._guess_idle():
            raise ValueError("a Stokes guess hook that is not idle runs device work and cannot be recorded")
        if self.cfg.allow_population_control:
            # the generator key of population control changes every step; a record would freeze it
            raise ValueError("steps with population control run eagerly (their random draws are keyed by the step)")
        if self.istep == 0:
            self.step()
        torch.cuda.synchronize()
        self._phases = None
        g = torch.cuda.CUDAGraph()
        self._capturing = True
        try:
            with ops.workspace_scope(self):
                with torch.cuda.graph(g, capture_error_mode="thread_local"):
                    self._step_body()
        finally:
            self._capturing = False
        self.istep -= 1                 # the capture recorded the step; nothing ran
        self.graph = g

    def _guess_idle(self):
        idle = getattr(self.guess, "idle", None)
        return bool(idle()) if idle is not None else False

    def step(self):
        if self.graph is not None and (self.guess is None or self._guess_idle()):
            if self.guess is not None:
                self.guess(self)        # an idle hook only keeps its tally; it launches nothing
            self.graph.replay()
            self.istep += 1
            self._replayed = True
            return
        self._replayed = False
        with ops.workspace_scope(self):
            self._step_body()

    def _step_body(self):
        self._step_pre()
        _, _, info = self.solver.solve(self.rhs_f, self.rhs_h, self.solV, self.solP, **self.stokes_solve_kw())
        self.last_solve = info
        self._step_post()

    def stokes_solve_kw(self):
        """The Stokes solve's settings (StokesSolver.solve keywords)."""
        return dict(scheme=self.scheme, precision=self.stokes_precision, tol=self.tol, inner_rtol=self.inner_rtol,
                    **self.solve_kw)

    def _step_pre(self):
        """The step up to the Stokes solve: particles, projections, qpoint fields, the Stokes
        right-hand side (rhs_f, rhs_h) and viscosity, the guess (solV, solP)."""
        c, b, tb = self.cfg, self.box, self.tables
        P = self.props
        self._mark("particles+projections")
        # particle fields + material (meeuuw.py:1118-1154)
        nodal = dict(exx=self.exx_n, ezz=self.ezz_n, exz=self.exz_n, q=self.q, T=self.T if c.solve_T else None)
        ops.interp_material(b, self.active, self.r, self.t, self.iel, self.mat, nodal, self.material, P)
        # elements and nodes (meeuuw.py:1194, 1344-1405)
        ops.bin_particles(self.nel, self.active, self.iel, self.counts, self.offsets, self.order, self.err)
        ops.project_elements(self.nel, self.offsets, self.order, P["rho"], P["eta"], c.averaging, self.rho_e,
                             self.eta_e, self.err)
        nd = self.nodal
        ops.project_nodes(b, c.nodal_projection_type, [(P["rho"], "arithmetic"), (P["eta"], c.averaging)],
                          self.offsets, self.order, self.r, self.t, [nd["rho"], nd["eta"]])
        if c.solve_T:
            ops.project_nodes(b, 2, [(P[k], "arithmetic") for k in ("hcond", "hcapa", "hprod", "alpha")],
                              self.offsets, self.order, self.r, self.t, [nd[k] for k in ("hcond", "hcapa", "hprod",
                                                                                        "alpha")])
        # qpoint fields (meeuuw.py:1503-1590, "elemental" rho/eta, or the least-squares fits)
        qf = self.qf
        ops.elemental_to_qpoints(self.rho_e, self.eta_e, qf["rhoq"], qf["etaq"])
        if c.ls_order:                                                   # meeuuw.py:1225-1297
            cnt, off, order = self.ls_bins
            ops.bin_particles(self.nel, self.every, self.iel, cnt, off, order, self.err)
            (cr, _, _), (ce, _, _) = ops.ls_fit(b, c.ls_order, off, order, self.x, self.z, [P["rho"], P["eta"]],
                                                limit_h=b.hx if c.ls_order == 3 else 0.0, err=self.err)
            if c.particle_rho_projection.startswith("least_squares"):
                ops.ls_to_qpoints(b, cr, self.xq, self.zq, qf["rhoq"])
            if c.particle_eta_projection.startswith("least_squares"):
                ops.ls_to_qpoints(b, ce, self.xq, self.zq, qf["etaq"])
        if c.solve_T:
            ops.nodal_to_qpoints(b, L.SPACE_Q2, tb["N_V"], self.T, qf["Tq"])
            for k in ("hcapa", "hcond", "hprod", "alpha"):
                ops.nodal_to_qpoints(b, L.SPACE_Q1_ON_V, tb["N_P"], nd[k], qf[k + "q"])
        if c.formulation == "EBA":
            for k in ("exx", "ezz", "exz"):
                ops.nodal_to_qpoints(b, L.SPACE_Q2, tb["N_V"], getattr(self, k + "_n"), qf[k + "q"])
        self._mark("stokes")
        # Stokes (meeuuw.py:1705-1851): right-hand side, matrix-free solve
        if self.zero_bc_values:
            ops.stokes_rhs_body(b, qf["rhoq"], self.gxq, self.gzq, self.geo["JxWq"], tb["N_V"], self.bc_fix_V,
                                self.rhs_f, self.rhs_h)
        else:
            ops.assemble_stokes(b, False, 0, self.stokes_inputs(), tb, self.bc_fix_V, self.bc_val_V, c.eta_ref,
                                self.L_ref, out=dict(rhs_f=self.rhs_f, rhs_h=self.rhs_h))
        self.solver.set_viscosity(qf["etaq"], self.eta_e)
        if self.guess is not None:
            if not self._capturing:
                self.guess(self)
        elif self.warm_start != "previous":
            self.solV.zero_()
            self.solP.zero_()

    def _step_post(self):
        """The step after the Stokes solve: velocity and pressure fields, dt, energy, Nu, strain
        rate, vrms, advection and locate."""
        c, b, tb = self.cfg, self.box, self.tables
        P = self.props
        qf, nd = self.qf, self.nodal
        ops.split_solution(self.solV, self.solP, c.eta_ref / self.L_ref, self.u, self.w, self.p)
        self._mark("post+dt")
        # pressure normalisation and nodal pressure (meeuuw.py:1958-2051)
        ops.pressure_offset(b, c.pressure_normalisation, self.p, tb["N_P"], self.geo["JxWq"], self.volume, self.offset)
        ops.nodal_pressure(b, self.p, self.offset, tb["N_P_n"], self.q, subtract=True)
        # time step (meeuuw.py:2112-2139)
        ops.compute_dt(self.u, self.w, P["hcond"], P["hcapa"], P["rho"], c.CFLnb, b.hx, b.hz, c.dt_max, c.solve_T,
                       self.dt_state, self.dt_out)
        ops.nodal_to_qpoints(b, L.SPACE_Q2, tb["N_V"], self.u, qf["uq"])
        ops.nodal_to_qpoints(b, L.SPACE_Q2, tb["N_V"], self.w, qf["wq"])
        if c.solve_T:
            self._mark("energy")
            # energy (meeuuw.py:2186-2235); T on entry is T_mem
            q = {k: qf[k] for k in ("rhoq", "etaq", "Tq", "uq", "wq", "hcondq", "hcapaq", "alphaq", "hprodq")}
            for k in ("exxq", "ezzq", "exzq"):
                q[k] = qf.get(k)
            q.update(self.geo)
            if self.energy_op is not None:
                ops.energy_op_setup(b, self.T, q, tb, self.bc_fix_T, self.bc_val_T, 0.0, c.rho0, c.formulation,
                                    self.energy_op, self.rhs_T, dt_dev=self.dt_out)
                self.energy_info = ops.energy_op_solve(b, self.energy_op, self.rhs_T, self.T, rtol=self.energy_rtol,
                                                       maxit=300)
            else:
                ops.assemble_energy(b, 0, self.T, q, tb, self.bc_fix_T, self.bc_val_T, 0.0, c.rho0, c.formulation,
                                    self.VV_T, self.rhs_T, dt_dev=self.dt_out)
                self.energy_info = ops.energy_solve(b, self.VV_T, self.rhs_T, self.T, rtol=self.energy_rtol,
                                                    maxit=300)
            # heat flux and Nu (meeuuw.py:2259-2308)
            ops.nodal_heat_flux(b, self.T, nd["hcond"], tb, out=self.hf)
            ops.compute_nu(b, self.T, self.hf[0], self.hf[1], nd["hcond"], self.nu_out)
        self._mark("strain+vrms")
        # nodal strain rate for the next step's particles (meeuuw.py:2385)
        ops.nodal_strain_rate(b, self.u, self.w, tb, out=[self.exx_n, self.ezz_n, self.exz_n])
        # vrms (meeuuw.py:2512; uses the Tq of this step as the reference does)
        ops.global_quantities(qf["uq"], qf["wq"], qf["Tq"] if c.solve_T else None, qf["rhoq"], self.geo["JxWq"],
                              self.volume, self.gq_out)
        self._mark("advect+locate")
        # advect and locate (meeuuw.py:2726, 2862)
        ops.advect(b, c.RKorder, 0.0, self.x, self.z, self.active, self.u, self.w, self.up, self.wp, self.err,
                   dt_dev=self.dt_out)
        if c.allow_population_control and c.RKorder > 0:                 # meeuuw.py:2846-2850
            ops.population_control(b, c.nmin, self.counts, self.offsets, self.order, self.active, self.iel, self.r,
                                   self.t, self.x, self.z, mat=self.mat, avg=(P["eta"], self.up, self.wp),
                                   seed=c.population_seed(self.istep), added=self.pc_added, err=self.err)
        ops.locate(b, self.active, self.x, self.z, self.r, self.t, self.iel, self.err)
        self._mark("end")
        self.istep += 1

    def diagnostics(self):
        """Reads the step's scalars (synchronises) and applies the reference's exit checks."""
        if self._replayed:              # a recorded step ran: the solvers' outcomes are on the device
            with ops.workspace_scope(self):
                self.last_solve = self.solver.device_info(self.tol)
                if self.cfg.solve_T:
                    self.energy_info = ops.energy_device_info(self.box, op=self.energy_op is not None)
            self._replayed = False
        err = int(self.err.item())
        d = dict(istep=self.istep, dt=float(self.dt_out[0].item()), vrms=float(self.gq_out[0].item()),
                 Tavrg=float(self.gq_out[1].item()), Nu=float(self.nu_out[12].item()) if self.cfg.solve_T else None,
                 err=err, stokes=dict(self.last_solve))
        return d

    def check(self):
        """SystemExit with the reference's message when a device flag is set."""
        err = int(self.err.item())
        if err & L.FLAG_EMPTY_ELEMENT:
            raise SystemExit("ABORT: an element contains no particle!")          # meeuuw.py:1198-1199
        if err & L.FLAG_R_OUT:
            raise SystemExit("r value out of bounds")                             # locate_particles.py:61-62
        if err & L.FLAG_T_OUT:
            raise SystemExit("t value out of bounds")                             # locate_particles.py:63-64
        if err & L.FLAG_ELEMENT_RANGE:
            raise SystemExit("particle outside the mesh")
        if err & L.FLAG_POP_UNAVAILABLE:
            raise ValueError("population_control: not available yet")          # pic_functions.py:1722-1733
        if err & L.FLAG_POP_MASK_EMPTY:
            raise ValueError("population_control: mask empty")                  # pic_functions.py:1747-1748
