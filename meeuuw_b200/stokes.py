"""Device Stokes solver handle (matrix-free operator + multigrid PCG + Uzawa), over the C ABI.

Mirrors the reference's block solvers ``uzawa3_solver_L2`` (uzawa3_solver_L2.py:21-99) and
``cd_u_eta`` (cd_u_eta.py:13-99): the Schur-complement PCG with step lengths and the FP64
stopping test on the device, K^-1 by geometric-multigrid PCG instead of SuperLU.
"""
import ctypes

import torch

from . import _lib as L
from ._lib import c_double, c_int32, c_size_t, c_void_p, call, ptr, stream_ptr


class MwStokesParams(ctypes.Structure):
    _fields_ = [("eta_ref", c_double), ("L_ref", c_double), ("precisions", c_int32), ("coarse_min", c_int32),
                ("dense_max", c_int32), ("cheb_degree", c_int32), ("cheb_ratio", c_double),
                ("cheb_safety", c_double), ("power_iters", c_int32), ("power_iters_warm", c_int32),
                ("tail_nel", c_int32), ("cheb_degree_coarse", c_int32), ("coarsen_odd", c_int32),
                ("coarse_dense_max", c_int32)]


class MwSolveParams(ctypes.Structure):
    _fields_ = [("scheme", c_int32), ("precision", c_int32), ("tol", c_double), ("max_outer", c_int32),
                ("max_inner", c_int32), ("inner_rtol", c_double), ("max_refine", c_int32),
                ("sweep_reduction", c_double), ("mass_iters", c_int32),
                ("use_guess", c_int32), ("history", c_void_p), ("history_len", c_int32),
                ("host_loops", c_int32), ("sweep_target", c_double)]


class MwSolveInfo(ctypes.Structure):
    _fields_ = [("outer_iters", c_int32), ("inner_iters", c_int32), ("refinements", c_int32), ("converged", c_int32),
                ("rel_residual", c_double), ("initial_rel_residual", c_double)]


L.extra_protos({
    "mw_stokes_default_params": (None, [c_void_p]),
    "mw_solve_default_params": (None, [c_void_p]),
    "mw_stokes_workspace_bytes": (c_size_t, [L.MwBox, MwStokesParams]),
    "mw_stokes_create": (c_int32, [L.MwBox, MwStokesParams, c_void_p, c_void_p, c_size_t, c_void_p]),
    "mw_stokes_destroy": (c_int32, [c_void_p]),
    "mw_stokes_device_loops": (c_int32, [c_void_p]),
    "mw_stokes_device_info": (c_int32, [c_void_p, c_double, c_void_p, c_void_p]),
    "mw_stokes_uzawa_residual": (c_int32, [c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_double, c_int32,
                                           c_void_p, c_void_p, c_void_p]),
    "mw_stokes_levels": (c_int32, [c_void_p, c_int32]),
    "mw_stokes_set_viscosity": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_stokes_apply": (c_int32, [c_void_p] * 6),
    "mw_stokes_apply_f32": (c_int32, [c_void_p] * 6),
    "mw_stokes_grad": (c_int32, [c_void_p] * 4),
    "mw_stokes_cheb_step_f32": (c_int32, [c_void_p] * 5 + [c_int32, c_void_p]),
    "mw_stokes_div": (c_int32, [c_void_p] * 4),
    "mw_stokes_vcycle": (c_int32, [c_void_p, c_int32, c_void_p, c_void_p, c_void_p]),
    "mw_stokes_solve_K": (c_int32, [c_void_p, c_int32, c_void_p, c_void_p, c_double, c_int32,
                                    ctypes.POINTER(c_int32), ctypes.POINTER(c_double), c_void_p]),
    "mw_stokes_residual": (c_int32, [c_void_p] * 7 + [c_void_p, c_void_p]),
    "mw_stokes_solve": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, MwSolveParams, c_void_p,
                                  c_void_p]),
    "mw_stokes_prepare": (c_int32, [c_void_p, c_int32, c_void_p]),
    "mw_stokes_transfer": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_void_p]),
    "mw_stokes_level_shape": (c_int32, [c_void_p, c_int32, c_int32, ctypes.POINTER(c_int32),
                                        ctypes.POINTER(c_int32)]),
    "mw_stokes_ensemble_create": (c_int32, [c_void_p] * 5 + [c_int32, c_void_p]),
    "mw_stokes_ensemble_solve": (c_int32, [c_void_p, MwSolveParams, c_void_p]),
    "mw_stokes_ensemble_destroy": (c_int32, [c_void_p]),
})

SCHEME = {"cd_u_eta": 0, "uzawa3": 1}
PREC = {"f64": 0, "f32": 1, "mixed": 1}


class StokesSolver:
    """One box mesh's Stokes solver; owns its device workspace (a torch uint8 tensor)."""

    def __init__(self, box, bc_fix_V, eta_ref=1.0, L_ref=1.0, precisions=("f64", "f32"), **kw):
        L.require_cuda()
        self.box = box
        self.fix = bc_fix_V.view(torch.uint8) if bc_fix_V.dtype == torch.bool else bc_fix_V
        prm = MwStokesParams()
        L.lib().mw_stokes_default_params(ctypes.byref(prm))
        prm.eta_ref, prm.L_ref = float(eta_ref), float(L_ref)
        prm.precisions = (1 if "f64" in precisions else 0) | (2 if ("f32" in precisions or "mixed" in precisions) else 0)
        for k, v in kw.items():
            setattr(prm, k, v)
        self.prm = prm
        nbytes = L.lib().mw_stokes_workspace_bytes(box, prm)
        self.work = torch.empty(int(nbytes), dtype=torch.uint8, device="cuda")
        h = c_void_p()
        call("mw_stokes_create", box, prm, ptr(self.fix), ptr(self.work), c_size_t(self.work.numel()), ctypes.byref(h))
        self.h = h
        self.nv = 2 * (2 * box.nelx + 1) * (2 * box.nelz + 1)
        self.np = (box.nelx + 1) * (box.nelz + 1)

    def __del__(self):
        if getattr(self, "h", None) is not None and L._lib is not None:
            L.lib().mw_stokes_destroy(self.h)
            self.h = None

    def levels(self, precision="f64"):
        return L.lib().mw_stokes_levels(self.h, PREC[precision])

    def set_viscosity(self, etaq, eta_e=None):
        self._eta = etaq
        call("mw_stokes_set_viscosity", self.h, ptr(etaq), ptr(eta_e), stream_ptr())

    def prepare(self, precision="mixed"):
        """Set up the multigrid hierarchy for the current viscosity (coarse viscosities, diagonals,
        Chebyshev intervals, the coarsest inverse) on the current stream; a solve does this itself,
        an ensemble solve (StokesEnsembleSolve) needs it done per model first."""
        call("mw_stokes_prepare", self.h, PREC[precision], stream_ptr())

    def level_shape(self, level, precision="f64"):
        """(nx, nz) elements of multigrid level `level` (0: the mesh)."""
        nx, nz = c_int32(), c_int32()
        call("mw_stokes_level_shape", self.h, PREC[precision], int(level), ctypes.byref(nx), ctypes.byref(nz))
        return nx.value, nz.value

    def restrict(self, level, r_fine, precision="f64"):
        """P^T r from level `level` to level + 1 (fixed coarse dofs zero)."""
        nx, nz = self.level_shape(level + 1, precision)
        out = torch.zeros(2 * (2 * nx + 1) * (2 * nz + 1), dtype=r_fine.dtype, device="cuda")
        call("mw_stokes_transfer", self.h, PREC[precision], int(level), 1, ptr(r_fine), ptr(out), stream_ptr())
        return out

    def prolong(self, level, x_coarse, precision="f64"):
        """P x_c from level `level` + 1 to level `level` (zero on the fixed fine dofs)."""
        nx, nz = self.level_shape(level, precision)
        out = torch.zeros(2 * (2 * nx + 1) * (2 * nz + 1), dtype=x_coarse.dtype, device="cuda")
        call("mw_stokes_transfer", self.h, PREC[precision], int(level), 0, ptr(x_coarse), ptr(out), stream_ptr())
        return out

    def apply(self, u=None, p=None, yV=None, yP=None, precision="f64"):
        dt = torch.float32 if precision == "f32" else torch.float64
        if yV is None:
            yV = torch.empty(self.nv, dtype=dt, device="cuda")
        if yP is None:
            yP = torch.empty(self.np, dtype=dt, device="cuda")
        name = "mw_stokes_apply_f32" if precision == "f32" else "mw_stokes_apply"
        call(name, self.h, ptr(u), ptr(p), ptr(yV), ptr(yP), stream_ptr())
        return yV, yP

    def cheb_step_f32(self, b, x, xo, d, step=1):
        """One Chebyshev smoothing step of the FP32 finest level (coefficient pair `step`)."""
        call("mw_stokes_cheb_step_f32", self.h, ptr(b), ptr(x), ptr(xo), ptr(d), int(step), stream_ptr())
        return xo

    def grad(self, p, yV=None):
        """yV = G p (the Schur iterations' stencil form of the G block)."""
        yV = torch.empty(self.nv, dtype=torch.float64, device="cuda") if yV is None else yV
        call("mw_stokes_grad", self.h, ptr(p), ptr(yV), stream_ptr())
        return yV

    def div(self, u, yP=None):
        """yP = G^T u (fixed velocity entries ignored)."""
        yP = torch.empty(self.np, dtype=torch.float64, device="cuda") if yP is None else yP
        call("mw_stokes_div", self.h, ptr(u), ptr(yP), stream_ptr())
        return yP

    def solve_K(self, b, precision="f64", rtol=1e-10, maxit=500):
        x = torch.empty_like(b)
        it = c_int32()
        rr = c_double()
        rc = L.lib().mw_stokes_solve_K(self.h, PREC[precision], ptr(b), ptr(x), float(rtol), int(maxit), ctypes.byref(it),
                                       ctypes.byref(rr), stream_ptr())
        if rc not in (0, 3):
            raise RuntimeError(f"mw_stokes_solve_K returned {L.STATUS.get(rc, rc)}")
        return x, it.value, rr.value

    def vcycle(self, b, precision="f64"):
        x = torch.empty_like(b)
        call("mw_stokes_vcycle", self.h, PREC[precision], ptr(b), ptr(x), stream_ptr())
        return x

    def device_info(self, tol=1e-8):
        """Outcome of the last solve read from its device scalars (after a recorded-graph replay)."""
        info = MwSolveInfo()
        call("mw_stokes_device_info", self.h, float(tol), ctypes.byref(info), stream_ptr())
        out = {k: getattr(info, k) for k, _ in MwSolveInfo._fields_}
        out["status"] = "MW_OK" if info.converged else "MW_ERR_NOT_CONVERGED"
        return out

    def device_loops(self):
        """True once a solve ran as one recorded graph with its loops on the device."""
        return bool(L.lib().mw_stokes_device_loops(self.h))

    def uzawa_residual(self, f, h, P, precision="f32", rtol=1e-3, maxit=100, V=None):
        """||G^T K^-1 (f - G P) - h|| (mean removed): how far pressure P is from the Schur solution,
        the quantity the Uzawa iteration starts from."""
        prec = PREC[precision]
        nrm = c_double()
        call("mw_stokes_uzawa_residual", self.h, prec, ptr(f), ptr(h), ptr(P), float(rtol), int(maxit), ptr(V),
             ctypes.byref(nrm), stream_ptr())
        return nrm.value

    def residual(self, V, P, f, h):
        RV = torch.empty(self.nv, dtype=torch.float64, device="cuda")
        RP = torch.empty(self.np, dtype=torch.float64, device="cuda")
        nrm = c_double()
        call("mw_stokes_residual", self.h, ptr(V), ptr(P), ptr(f), ptr(h), ptr(RV), ptr(RP), ctypes.byref(nrm),
             stream_ptr())
        return RV, RP, nrm.value

    def solve(self, f, h, V=None, P=None, scheme="cd_u_eta", precision="f64", tol=1e-8, raise_on_fail=False, **kw):
        """Returns (solV, solP, info dict).  V/P given -> warm start (overwritten in place)."""
        sp = MwSolveParams()
        L.lib().mw_solve_default_params(ctypes.byref(sp))
        sp.scheme, sp.precision, sp.tol = SCHEME[scheme], PREC[precision], float(tol)
        for k, v in kw.items():
            setattr(sp, k, v)
        if V is None or P is None:
            V = torch.zeros(self.nv, dtype=torch.float64, device="cuda")
            P = torch.zeros(self.np, dtype=torch.float64, device="cuda")
            sp.use_guess = 0
        else:
            sp.use_guess = 1
        info = MwSolveInfo()
        rc = L.lib().mw_stokes_solve(self.h, ptr(f), ptr(h), ptr(V), ptr(P), sp, ctypes.byref(info), stream_ptr())
        out = {k: getattr(info, k) for k, _ in MwSolveInfo._fields_}
        out["status"] = L.STATUS.get(rc, rc)
        if rc not in (0, 3) or (raise_on_fail and rc != 0):
            raise RuntimeError(f"mw_stokes_solve returned {out['status']} ({out})")
        return V, P, out


def solve_params(scheme="cd_u_eta", precision="f64", tol=1e-8, use_guess=True, **kw):
    sp = MwSolveParams()
    L.lib().mw_solve_default_params(ctypes.byref(sp))
    sp.scheme, sp.precision, sp.tol = SCHEME[scheme], PREC[precision], float(tol)
    sp.use_guess = 1 if use_guess else 0
    for k, v in kw.items():
        setattr(sp, k, v)
    return sp


class StokesEnsembleSolve:
    """The Stokes solves of many models in one launch: one thread-block cluster per model runs that
    model's whole mixed-precision solve (FP64 refinement, Schur-complement CG, FP32 multigrid-PCG)
    with its own hierarchy and convergence tests.  Binds each solver to its right-hand side (f, h)
    and solution (V, P) tensors, which must stay in place.  Before solve(), every model's viscosity
    is set and its hierarchy prepared (StokesSolver.prepare) on streams the current stream waits for;
    the outcomes are read per model with StokesSolver.device_info."""

    def __init__(self, solvers, f, h, V, P):
        n = len(solvers)
        if not (n == len(f) == len(h) == len(V) == len(P)) or n == 0:
            raise ValueError("one (f, h, V, P) per solver")
        self.solvers = list(solvers)
        self._keep = (list(f), list(h), list(V), list(P))     # the bound tensors stay alive
        arr = lambda xs: (c_void_p * n)(*[x.data_ptr() for x in xs])
        hs = (c_void_p * n)(*[s.h.value for s in self.solvers])
        e = c_void_p()
        call("mw_stokes_ensemble_create", hs, arr(f), arr(h), arr(V), arr(P), n, ctypes.byref(e))
        self.h = e

    def __del__(self):
        if getattr(self, "h", None) is not None and L._lib is not None:
            L.lib().mw_stokes_ensemble_destroy(self.h)
            self.h = None

    def solve(self, scheme="cd_u_eta", tol=1e-8, use_guess=True, **kw):
        sp = solve_params(scheme, "mixed", tol, use_guess, **kw)
        call("mw_stokes_ensemble_solve", self.h, sp, stream_ptr())

