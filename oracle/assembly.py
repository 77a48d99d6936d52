"""Oracle: Stokes and energy element assembly (vectorised over elements).

Test infrastructure only.  Same signatures and return tuples as the reference:

* ``build_matrix_stokes``  -- ``build_matrix_stokes.py:18-278`` (box, plane strain)
* ``build_matrix_energy``  -- ``build_matrix_energy.py:12-141``

The per-element arithmetic follows the reference line by line; the loops over
elements become numpy axes.  Right-hand sides are accumulated with
``np.add.at`` in element-major, local-dof-minor order, which is the order of the
reference's scatter loops (``build_matrix_stokes.py:223-229``,
``build_matrix_energy.py:133-139``).
"""
import numpy as np


def _stokes_element_blocks(nel, N_V, N_P, dNdr_V, dNdt_V, dNdr_P, dNdt_P, rhoq, etaq, JxWq,
                           gxq, gyq, jcbi00q, jcbi01q, jcbi10q, jcbi11q):
    """Per-element K_el, G_el (unscaled), M_el, H_el, f_el: build_matrix_stokes.py:130-154."""
    K = np.zeros((nel, 18, 18))
    G = np.zeros((nel, 18, 4))
    M = np.zeros((nel, 4, 4))
    H = np.zeros((nel, 4, 18))
    f = np.zeros((nel, 18))
    C = np.array([[2.0, 0, 0], [0, 2.0, 0], [0, 0, 1.0]])          # :77
    for iq in range(9):
        j00, j01 = jcbi00q[:, iq:iq + 1], jcbi01q[:, iq:iq + 1]
        j10, j11 = jcbi10q[:, iq:iq + 1], jcbi11q[:, iq:iq + 1]
        dNdx_V = j00 * dNdr_V[iq] + j01 * dNdt_V[iq]                # :131
        dNdz_V = j10 * dNdr_V[iq] + j11 * dNdt_V[iq]                # :132
        dNdx_P = j00 * dNdr_P[iq] + j01 * dNdt_P[iq]                # :133
        dNdz_P = j10 * dNdr_P[iq] + j11 * dNdt_P[iq]                # :134
        B = np.zeros((nel, 3, 18))
        B[:, 0, 0::2] = dNdx_V                                      # :135-139
        B[:, 1, 1::2] = dNdz_V
        B[:, 2, 0::2] = dNdz_V
        B[:, 2, 1::2] = dNdx_V
        jxw = JxWq[:, iq]
        BtCB = np.einsum("erp,rs,esq->epq", B, C, B)
        K += BtCB * etaq[:, iq, None, None] * jxw[:, None, None]     # :140
        f[:, 0::2] += N_V[iq][None, :] * jxw[:, None] * rhoq[:, iq, None] * gxq[:, iq, None]  # :142
        f[:, 1::2] += N_V[iq][None, :] * jxw[:, None] * rhoq[:, iq, None] * gyq[:, iq, None]  # :143
        BtN = (B[:, 0, :] + B[:, 1, :])[:, :, None] * N_P[iq][None, None, :]
        G -= BtN * jxw[:, None, None]                                # :144-146
        M += np.outer(N_P[iq], N_P[iq])[None] * jxw[:, None, None]   # :147
        Hq = np.zeros((nel, 4, 18))
        Hq[:, :, 0::2] = dNdx_P[:, :, None] * N_V[iq][None, None, :]  # :148-153
        Hq[:, :, 1::2] = dNdz_P[:, :, None] * N_V[iq][None, None, :]
        H += Hq * jxw[:, None, None]
    return K, G, M, H, f


def build_matrix_stokes(bignb_Stokes, bignb_K, bignb_M, bignb_G, nel, nq_per_element, m_V, m_P,
                        ndof_V, Nfem_V, Nfem_P, ndof_V_el, icon_V, icon_P, rhoq, etaq, JxWq,
                        local_to_globalV, gxq, gyq, N_V, N_P, dNdr_V, dNdt_V, dNdr_P, dNdt_P,
                        jcbi00q, jcbi01q, jcbi10q, jcbi11q, eta_e, eta_ref, L_ref, bc_fix_V,
                        bc_val_V, bot_element, top_element, bot_free_slip, top_free_slip,
                        geometry, theta_V, axisymmetric, xq, blocks):
    """build_matrix_stokes.py:18-278 restricted to the Cartesian, plane-strain path."""
    if axisymmetric or geometry != "box":
        raise NotImplementedError("oracle covers the Cartesian box path only")
    K, G, M, H, f = _stokes_element_blocks(nel, N_V, N_P, dNdr_V, dNdt_V, dNdr_P, dNdt_P, rhoq,
                                           etaq, JxWq, gxq, gyq, jcbi00q, jcbi01q, jcbi10q, jcbi11q)
    G *= eta_ref / L_ref                                             # :157
    h = np.zeros((nel, 4))
    l2g = local_to_globalV
    for ikk in range(18):                                            # :206-217
        m1 = l2g[ikk]
        fix = bc_fix_V[m1]
        if not fix.any():
            continue
        e = np.nonzero(fix)[0]
        val = bc_val_V[m1[e]]
        K_ref = K[e, ikk, ikk].copy()
        f[e, :] -= K[e, :, ikk] * val[:, None]
        K[e, ikk, :] = 0
        K[e, :, ikk] = 0
        K[e, ikk, ikk] = K_ref
        f[e, ikk] = K_ref * val
        h[e, :] -= G[e, ikk, :] * val[:, None]
        G[e, ikk, :] = 0
    rhs_f = np.zeros(Nfem_V)
    rhs_h = np.zeros(Nfem_P)
    np.add.at(rhs_f, l2g.T.ravel(), f.ravel())                      # :223-225
    np.add.at(rhs_h, icon_P.T.ravel(), h.ravel())                   # :227-229
    empty = np.zeros(0)
    if blocks:                                                      # :235-265
        VV_K = K.reshape(-1).copy()
        VV_G = G.reshape(-1).copy()
        VV_GT = np.transpose(G, (0, 2, 1)).reshape(-1).copy()
        VV_H = H.reshape(-1).copy()
        VV_M = M.reshape(-1).copy()
        VV_M_eta = (M / eta_e[:, None, None]).reshape(-1).copy()
        return empty, rhs_f, rhs_h, VV_K, VV_G, VV_GT, VV_M, VV_M_eta, VV_H
    full = np.zeros((nel, 18, 26))                                  # :267-276
    full[:, :, :18] = K
    full[:, :, 18::2] = G
    full[:, :, 19::2] = G
    return full.reshape(-1), rhs_f, rhs_h, empty, empty, empty, empty, empty, empty


def build_matrix_energy(bignb, nel, nq_per_element, m_T, Nfem_T, T, icon_T, rhoq, etaq, Tq, uq, wq,
                        hcondq, hcapaq, alphaq, hprodq, exxq, ezzq, exzq, dpdxq, dpdzq, JxWq, N_T,
                        dNdr_T, dNds_T, jcbi00q, jcbi01q, jcbi10q, jcbi11q, bc_fix_T, bc_val_T, dt,
                        formulation, rho0):
    """build_matrix_energy.py:12-141 (Crank-Nicolson element systems + Dirichlet elimination)."""
    MM = np.zeros((nel, 9, 9))
    Kd = np.zeros((nel, 9, 9))
    Ka = np.zeros((nel, 9, 9))
    b = np.zeros((nel, 9))
    Tvect = T[icon_T].T                                             # :63
    for iq in range(9):
        N = N_T[iq]
        u = uq[:, iq:iq + 1]
        w = wq[:, iq:iq + 1]
        dNdx = jcbi00q[:, iq:iq + 1] * dNdr_T[iq] + jcbi01q[:, iq:iq + 1] * dNds_T[iq]   # :71
        dNdy = jcbi10q[:, iq:iq + 1] * dNdr_T[iq] + jcbi11q[:, iq:iq + 1] * dNds_T[iq]   # :72
        jxw = JxWq[:, iq, None, None]
        hc = hcapaq[:, iq, None, None]
        MM += np.outer(N, N)[None] * rho0 * hc * jxw                                    # :77
        BtB = dNdx[:, :, None] * dNdx[:, None, :] + dNdy[:, :, None] * dNdy[:, None, :]
        Kd += BtB * hcondq[:, iq, None, None] * jxw                                     # :79
        vB = u * dNdx + w * dNdy
        Ka += (N[None, :, None] * vB[:, None, :]) * rho0 * hc * jxw                      # :81
        b += N[None, :] * hprodq[:, iq:iq + 1] * JxWq[:, iq:iq + 1]                     # :83
        if formulation == "EBA":                                                         # :85-110
            exx, ezz, exz = exxq[:, iq:iq + 1], ezzq[:, iq:iq + 1], exzq[:, iq:iq + 1]
            b += (N[None, :] * 2 * etaq[:, iq:iq + 1]
                  * (2.0 / 3.0 * exx ** 2 + 2.0 / 3.0 * ezz ** 2 - 2.0 / 3.0 * exx * ezz + 2 * exz ** 2)
                  * JxWq[:, iq:iq + 1])
            b += (N[None, :] * alphaq[:, iq:iq + 1] * Tq[:, iq:iq + 1]
                  * (-w * rho0 * 10) * JxWq[:, iq:iq + 1])
    b *= dt                                                                             # :112
    A = MM + (Ka + Kd) * dt * 0.5                                                       # :114
    b += np.einsum("eij,ej->ei", MM - (Ka + Kd) * dt * 0.5, Tvect)                     # :115
    for k1 in range(9):                                                                 # :118-130
        m1 = icon_T[k1]
        fix = bc_fix_T[m1]
        if not fix.any():
            continue
        e = np.nonzero(fix)[0]
        val = bc_val_T[m1[e]]
        Aref = A[e, k1, k1].copy()
        b[e, :] -= A[e, :, k1] * val[:, None]
        A[e, k1, :] = 0
        A[e, :, k1] = 0
        A[e, k1, k1] = Aref
        b[e, k1] = Aref * val
    rhs = np.zeros(Nfem_T)
    np.add.at(rhs, icon_T.T.ravel(), b.ravel())                                        # :133-139
    return A.reshape(-1).copy(), rhs
