"""Shared body of the two Schur-complement solver drop-ins."""
import torch

from .._lib import ptr
from . import _operator
from ._common import back, dev, host_mode, f64

# Stopping rule of the device solver: FP64 relative true residual ||(f,h) - A(V,P)|| / ||(f,h)||.
# (The reference stops on the absolute step sizes ||alpha p||, ||alpha d|| < 1e-6, at most 100
# iterations; the relative residual is the criterion that is independent of the problem's units.)
TOL = 1e-8
# "mixed" (default, the time stepper's product path): FP32 inner multigrid-PCG with FP64 iterative
# refinement; "f64": FP64 throughout.
PRECISION = "mixed"
NITER = 100
# Per-precision solver settings, the ones GPUModel uses (meeuuw_b200/timestep.py): the mixed arm's
# inner tolerance, M_eta Chebyshev steps and refinement-sweep target; the FP64 arm's inner tolerance
# (the loosest that converges from a cold start on the 512x512 FK model).
SETTINGS = {"mixed": dict(inner_rtol=2e-2, mass_iters=6, sweep_target=0.1),
            "f64": dict(inner_rtol=1e-9, mass_iters=6)}


def solve(scheme, K, f, h, Nfem_P, V0=None, P0=None):
    op = _operator.current(K)
    if Nfem_P != op.nfem_P:
        raise ValueError("Nfem_P does not match the assembled operator")
    host = host_mode(f, h)
    S = op.solver(PRECISION)
    hist = torch.zeros(4, NITER, dtype=f64, device="cuda")
    fd, hd = dev(f, f64), dev(h, f64)
    if V0 is not None and P0 is not None:
        V, P = dev(V0, f64).clone(), dev(P0, f64).clone()
    else:
        V, P = None, None
    V, P, info = S.solve(fd, hd, V, P, scheme=scheme, precision=PRECISION, tol=TOL, history=ptr(hist),
                         history_len=NITER, **SETTINGS[PRECISION])
    if info["status"] != "MW_OK":
        raise RuntimeError(f"device Stokes solve did not converge: {info}")
    n = int(info["outer_iters"])
    h_out = back(hist, host)
    return back(V, host), back(P, host), n, h_out[0], h_out[1], h_out[2], h_out[3]
