"""The Stokes operator behind the solver drop-ins.

The reference assembles COO values (build_matrix_stokes), the driver turns them into SciPy
matrices (meeuuw.py:1784-1800) and hands those to the solver (meeuuw.py:1813-1818).  The device
solver is matrix-free: it applies the same operator element by element from the quadrature-point
viscosity.  The assembly drop-in therefore records, next to the values it returns, what the
matrix-free operator needs (viscosity, box, Dirichlet mask, eta_ref / L_ref) and a fingerprint of
the K block (its dimension and the FP64 sum of its values).  The solver drop-in checks the
matrices it receives against that fingerprint and refuses matrices it did not see assembled.
"""
import numpy as np
import torch

from ..stokes import StokesSolver

_current = None
_solvers = {}


class Operator:
    def __init__(self, box, etaq, eta_e, fix_u8, eta_ref, L_ref, nfem_V, nfem_P, k_sum, k_abs):
        self.box, self.etaq, self.eta_e, self.fix = box, etaq, eta_e, fix_u8
        self.eta_ref, self.L_ref = float(eta_ref), float(L_ref)
        self.nfem_V, self.nfem_P = nfem_V, nfem_P
        self.k_sum, self.k_abs = k_sum, k_abs
        self.viscosity_set = False

    def matches(self, K):
        if tuple(K.shape) != (self.nfem_V, self.nfem_V):
            return False
        data = K.data if hasattr(K, "data") and not isinstance(K, torch.Tensor) else None
        if data is None:
            return True
        return abs(float(np.sum(data)) - self.k_sum) <= 1e-9 * max(self.k_abs, 1e-300)

    def solver(self, precision):
        key = (self.box.nelx, self.box.nelz, self.box.hx, self.box.hz, self.fix.data_ptr(), self.eta_ref, self.L_ref,
               precision)
        S = _solvers.get(key)
        if S is None:
            precs = ("f32",) if precision == "mixed" else ("f64",)
            # the time stepper's smoothing settings per arithmetic (meeuuw_b200/timestep.py)
            S = StokesSolver(self.box, self.fix, eta_ref=self.eta_ref, L_ref=self.L_ref, precisions=precs,
                             cheb_degree=2 if precision == "mixed" else 1,
                             power_iters_warm=6 if precision == "mixed" else 3)
            _solvers.clear()          # one operator size at a time keeps the device memory bounded
            _solvers[key] = S
        if getattr(S, "_op", None) is not self:
            S.set_viscosity(self.etaq, self.eta_e)
            S._op = self
        return S


def record(op):
    global _current
    _current = op


def current(K):
    if _current is None:
        raise RuntimeError("the device Stokes solver needs the operator assembled by the build_matrix_stokes drop-in")
    if not _current.matches(K):
        raise RuntimeError("K does not match the operator last assembled by the build_matrix_stokes drop-in")
    return _current
