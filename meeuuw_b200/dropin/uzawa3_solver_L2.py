"""Device drop-in for ``uzawa3_solver_L2`` (uzawa3_solver_L2.py:21-99): the Schur-complement CG in
the pressure-mass-matrix inner product, run matrix-free on the device with multigrid-PCG inner K
solves.  Returns (solV, solP, iterations, array_xiV, array_xiP, array_alpha) with the reference's
history length 100.  Optional V0, P0 start from a previous solution."""
from . import _schur


def uzawa3_solver_L2(K_mat, G_mat, GT_mat, MP_mat, H_mat, f_rhs, h_rhs, Nfem_P, V0=None, P0=None):
    V, P, n, xiV, xiP, alpha, _ = _schur.solve("uzawa3", K_mat, f_rhs, h_rhs, Nfem_P, V0, P0)
    return V, P, n, xiV, xiP, alpha


__all__ = ["uzawa3_solver_L2"]
