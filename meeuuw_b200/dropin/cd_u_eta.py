"""Device drop-in for ``cd_u_eta`` (cd_u_eta.py:13-99): the Schur-complement CG preconditioned with
the viscosity-weighted pressure mass matrix M_eta, run matrix-free on the device with multigrid-PCG
inner K solves.  Returns (solV, solP, iterations, array_xiV, array_xiP, array_alpha, array_beta);
the history arrays have the reference's length 100.  Optional V0, P0 start the iteration from a
previous solution.  The stopping rule is the FP64 relative true residual ``_schur.TOL``."""
from . import _schur


def cd_u_eta(K, G, GT, M, M_eta, H, f, h, Nfem_P, V0=None, P0=None):
    return _schur.solve("cd_u_eta", K, f, h, Nfem_P, V0, P0)


__all__ = ["cd_u_eta"]
