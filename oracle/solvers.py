"""Oracle: the reference's Stokes and energy linear solves (SciPy sparse).

Test infrastructure only.

* COO -> CSR/CSC with duplicates summed    ``meeuuw.py:1784-1800``
* direct saddle-point solve                 ``meeuuw.py:1829-1833``
* ``uzawa3_solver_L2``                      ``uzawa3_solver_L2.py:21-99``
* ``cd_u_eta``                              ``cd_u_eta.py:13-99``
* energy solve                              ``meeuuw.py:2232-2235``

The sparse direct factorisations are SciPy's SuperLU (scipy 1.18.1 in this
image), exactly what the reference calls; they are third-party arithmetic and are
pinned only through residuals.
"""
import numpy as np
import scipy.sparse as sps
import scipy.sparse.linalg as sla


def stokes_blocks(mesh, VV_K, VV_G, VV_GT, VV_M, VV_M_eta, VV_H):
    """meeuuw.py:1786-1791."""
    IK, JK = mesh.coo_K()
    IG, JG, IGT, JGT = mesh.coo_G()
    IM, JM = mesh.coo_MP()
    nv, npp = mesh.Nfem_V, mesh.Nfem_P
    K = sps.coo_matrix((VV_K, (IK, JK)), shape=(nv, nv)).tocsc()
    M = sps.coo_matrix((VV_M, (IM, JM)), shape=(npp, npp)).tocsc()
    Me = sps.coo_matrix((VV_M_eta, (IM, JM)), shape=(npp, npp)).tocsc()
    G = sps.coo_matrix((VV_G, (IG, JG)), shape=(nv, npp)).tocsr()
    GT = sps.coo_matrix((VV_GT, (IGT, JGT)), shape=(npp, nv)).tocsr()
    H = sps.coo_matrix((VV_H, (IGT, JGT)), shape=(npp, nv)).tocsr()
    return K, G, GT, M, Me, H


def stokes_full(mesh, VV_Stokes):
    """meeuuw.py:1798."""
    II, JJ = mesh.coo_stokes()
    n = mesh.Nfem_V + mesh.Nfem_P
    return sps.coo_matrix((VV_Stokes, (II, JJ)), shape=(n, n)).tocsr()


def direct_solve(A, rhs_f, rhs_h):
    """meeuuw.py:1829-1833."""
    b = np.concatenate([rhs_f, rhs_h])
    return sla.spsolve(A, b)


def uzawa3_solver_L2(K_mat, G_mat, GT_mat, MP_mat, H_mat, f_rhs, h_rhs, Nfem_P, tol=1e-6, niter=100):
    """uzawa3_solver_L2.py:21-99 with innerK = innerMp = 'splu'."""
    xiV = np.zeros(niter)
    xiP = np.zeros(niter)
    alphas = np.zeros(niter)
    solP = np.zeros(Nfem_P)
    LU = sla.splu(K_mat)
    solV = LU.solve(f_rhs)                                             # :37-38
    LU_Mp = sla.splu(MP_mat)
    r = LU_Mp.solve(GT_mat.dot(solV) - h_rhs)                         # :46-47
    p = r.copy()
    k = 0
    for k in range(niter):                                            # :51-95
        d = LU.solve(G_mat.dot(p))
        alpha = r.dot(MP_mat.dot(r)) / p.dot(H_mat.dot(d))
        alphas[k] = alpha
        solP += alpha * p
        solV -= alpha * d
        rn = r + LU_Mp.solve(-alpha * GT_mat.dot(d))
        beta = rn.dot(MP_mat.dot(rn)) / r.dot(MP_mat.dot(r))
        pn = rn + beta * p
        xiP[k] = np.linalg.norm(alpha * p)
        xiV[k] = np.linalg.norm(alpha * d)
        if xiP[k] < tol and xiV[k] < tol:
            break
        r, p = rn, pn
    return solV, solP, k + 1, xiV, xiP, alphas


def _splu_spd(K, permc_spec):
    """SuperLU of the symmetric positive definite K with a symmetric fill-reducing ordering:
    the same factorisation up to round-off as ``splu(K)``, with far less fill on large meshes."""
    if permc_spec is None:
        return sla.splu(K)
    return sla.splu(K, permc_spec=permc_spec, diag_pivot_thresh=0.0, options=dict(SymmetricMode=True))


def cd_u_eta(K, G, GT, M, M_eta, H, f, h, Nfem_P, tol=1e-6, niter=100, permc_spec=None):
    """cd_u_eta.py:13-99 with innerK = innerM = 'splu'.  ``permc_spec`` (e.g. "MMD_AT_PLUS_A")
    only reorders K's factorisation (SuperLU's default COLAMD runs out of memory at 512x512)."""
    xiV = np.zeros(niter)
    xiP = np.zeros(niter)
    alphas = np.zeros(niter)
    betas = np.zeros(niter)
    solP = np.zeros(Nfem_P)
    LU_K = _splu_spd(K, permc_spec)
    solV = LU_K.solve(f)                                               # (B)
    LU_M = sla.splu(M)
    LU_Me = sla.splu(M_eta)
    q = LU_M.solve(-GT @ solV + M @ h)                                 # (C)
    w = LU_Me.solve(-GT @ solV + M @ h)                                # (D)
    d = -w.copy()
    k = 0
    for k in range(niter):
        z = LU_K.solve(G @ d)                                          # (E)
        alpha = q.dot(M.dot(w)) / d.dot(H.dot(z))                      # (F)
        alphas[k] = alpha
        solP += alpha * d                                              # (G)
        solV -= alpha * z                                              # (H)
        qn = LU_M.solve(-GT @ solV + M @ h)                            # (I)
        wn = LU_Me.solve(M @ qn)                                       # (J)
        beta = qn.dot(M.dot(wn)) / q.dot(M.dot(w))                     # (K)
        betas[k] = beta
        dn = -wn + beta * d
        xiP[k] = np.linalg.norm(alpha * d)
        xiV[k] = np.linalg.norm(alpha * z)
        if xiP[k] < tol and xiV[k] < tol:
            break
        w, d, q = wn, dn, qn
    return solV, solP, k + 1, xiV, xiP, alphas, betas


def energy_solve(mesh, VV_T, rhs, permc_spec=None):
    """meeuuw.py:2232-2235 (``permc_spec`` only reorders the factorisation)."""
    II, JJ = mesh.coo_T()
    A = sps.coo_matrix((VV_T, (II, JJ)), shape=(mesh.nn_V, mesh.nn_V)).tocsr()
    if permc_spec is None:
        return sla.spsolve(A, rhs)
    return sla.spsolve(A, rhs, permc_spec=permc_spec)


def stokes_relative_residual(A, sol, rhs_f, rhs_h):
    """FP64 relative true residual ||b - A x|| / ||b|| of the full saddle system."""
    b = np.concatenate([rhs_f, rhs_h])
    r = b - A @ sol
    return float(np.linalg.norm(r) / np.linalg.norm(b))
