"""Oracle: nodal<->qpoint projections and the FP64 reductions.

Test infrastructure only.  Sequential sums of the reference (``+=`` inside a
loop over elements and qpoints) are reproduced with ``np.cumsum(...)[-1]``,
which accumulates in the same order.

* ``project_nodal_{P,V,T}field_onto_qpoints``  ``project_nodal_field_onto_qpoints.py:12-62``
* ``compute_pressure_offset``                   ``compute_pressure_offset.py:12-66``
* ``compute_nodal_pressure``                    ``compute_nodal_pressure.py:8-21``
* ``compute_nodal_strain_rate``                 ``compute_strain_rate.py:51-73``
* ``compute_nodal_heat_flux``                   ``compute_nodal_heat_flux.py:12-40``
* ``compute_Nu``                                ``postprocessors.py:114-248``
* ``compute_global_quantities``                 ``postprocessors.py:14-83``
* time step                                     ``meeuuw.py:2112-2139``
"""
import numpy as np

from .fe import basis_V


def _seqsum(a):
    a = np.ascontiguousarray(a).ravel()
    return float(np.cumsum(a)[-1]) if a.size else 0.0


def project_nodal_field_onto_qpoints(phi_nodal, N, icon):
    """phiq[e, q] = sum_k N[q, k] phi[icon[k, e]] (k ascending)."""
    m = N.shape[1]
    acc = N[None, :, 0] * phi_nodal[icon[0]][:, None]
    for k in range(1, m):
        acc = acc + N[None, :, k] * phi_nodal[icon[k]][:, None]
    return acc


def compute_pressure_offset(pressure_normalisation, top_element, nelx, N_P, JxWq, p, icon_P, volume):
    """compute_pressure_offset.py:12-66 (Cartesian, non-axisymmetric)."""
    if pressure_normalisation == "none":
        return 0.0
    if pressure_normalisation == "surface":                        # :219-223
        e = np.nonzero(top_element)[0]
        return _seqsum(0.5 * (p[icon_P[2, e]] + p[icon_P[3, e]])) / nelx
    if pressure_normalisation == "volume":                         # :234-238
        pq = project_nodal_field_onto_qpoints(p, N_P, icon_P)
        return _seqsum(pq * JxWq) / volume
    raise ValueError("compute_pressure_offset: unknown pressure_normalisation value")


def compute_nodal_pressure(nn_V, icon_V, icon_P, p, N_P_n):
    """compute_nodal_pressure.py:8-21: q on V nodes by averaging element-local Q1 values."""
    q = np.zeros(nn_V)
    cnt = np.zeros(nn_V, dtype=np.int32)
    vals = np.zeros((icon_V.shape[1], 9))
    for k in range(9):
        vals[:, k] = project_nodal_field_onto_qpoints(p, N_P_n[k:k + 1], icon_P)[:, 0]
    np.add.at(q, icon_V.T.ravel(), vals.ravel())
    np.add.at(cnt, icon_V.T.ravel(), 1)
    return q / cnt


def compute_nodal_strain_rate(icon_V, u, v, nn_V, dNdr_V_n, dNds_V_n, jcbi00n, jcbi01n, jcbi10n, jcbi11n):
    """compute_strain_rate.py:51-73."""
    nel = icon_V.shape[1]
    ue, ve = u[icon_V].T, v[icon_V].T
    exx = np.zeros((nel, 9))
    eyy = np.zeros((nel, 9))
    exy = np.zeros((nel, 9))
    for i in range(9):
        dNdx = jcbi00n[:, i:i + 1] * dNdr_V_n[i] + jcbi01n[:, i:i + 1] * dNds_V_n[i]
        dNdy = jcbi10n[:, i:i + 1] * dNdr_V_n[i] + jcbi11n[:, i:i + 1] * dNds_V_n[i]
        exx[:, i] = np.sum(dNdx * ue, axis=1)
        eyy[:, i] = np.sum(dNdy * ve, axis=1)
        exy[:, i] = 0.5 * np.sum(dNdx * ve, axis=1) + 0.5 * np.sum(dNdy * ue, axis=1)
    out = []
    cnt = np.zeros(nn_V)
    np.add.at(cnt, icon_V.T.ravel(), 1.0)
    for a in (exx, eyy, exy):
        n = np.zeros(nn_V)
        np.add.at(n, icon_V.T.ravel(), a.ravel())
        out.append(n / cnt)
    return tuple(out)


def compute_nodal_heat_flux(icon_T, T, hcond_nodal, nn_T, dNdr_T_n, dNds_T_n, jcbi00_T, jcbi01_T,
                            jcbi10_T, jcbi11_T):
    """compute_nodal_heat_flux.py:12-40 -> (dTdx_n, dTdy_n, qx_n, qy_n)."""
    nel = icon_T.shape[1]
    Te = T[icon_T].T
    gx = np.zeros((nel, 9))
    gy = np.zeros((nel, 9))
    for i in range(9):
        dNdx = jcbi00_T[:, i:i + 1] * dNdr_T_n[i] + jcbi01_T[:, i:i + 1] * dNds_T_n[i]
        dNdy = jcbi10_T[:, i:i + 1] * dNdr_T_n[i] + jcbi11_T[:, i:i + 1] * dNds_T_n[i]
        gx[:, i] = np.sum(dNdx * Te, axis=1)
        gy[:, i] = np.sum(dNdy * Te, axis=1)
    nodes = icon_T.T.ravel()
    hc = hcond_nodal[icon_T].T
    res = []
    for a in (-gx, -gy, -(hc * gx), -(hc * gy)):
        n = np.zeros(nn_T)
        np.add.at(n, nodes, a.ravel())
        res.append(n)
    cnt = np.zeros(nn_T)
    np.add.at(cnt, nodes, 1.0)
    dTdx, dTdy, qx, qy = (r / cnt for r in res)
    return dTdx, dTdy, qx, qy


def compute_Nu(Lx, Lz, x_V, z_V, nel, left_element, right_element, top_element, bottom_element,
               icon_V, T, dTdx_nodal, dTdz_nodal, nq_per_dim, qcoords, qweights, hcond_n):
    """postprocessors.py:114-248 -> the 13-tuple ending in Nu."""
    qc = np.asarray(qcoords, dtype=np.float64)
    qw = np.asarray(qweights, dtype=np.float64)

    def side(mask, rfix, tfix, grad, jac, nsign):
        e = np.nonzero(mask)[0]
        if rfix is not None:
            N = basis_V(np.full(3, float(rfix)), qc)
        else:
            N = basis_V(qc, np.full(3, float(tfix)))
        Tq = (T[icon_V[:, e]].T @ N.T)                 # (ne, 3)
        hq = (hcond_n[icon_V[:, e]].T @ N.T)
        gq = (grad[icon_V[:, e]].T @ N.T)
        jc = jac(e)[:, None]
        aT = _seqsum(Tq * jc * qw[None, :])
        ag = _seqsum(gq * jc * qw[None, :] * nsign)
        q = -_seqsum(hq * gq * jc * qw[None, :] * nsign)
        return aT, ag, q

    aTl, agl, qxl = side(left_element, -1, None, dTdx_nodal,
                         lambda e: (z_V[icon_V[3, e]] - z_V[icon_V[0, e]]) / 2, -1)
    aTr, agr, qxr = side(right_element, +1, None, dTdx_nodal,
                         lambda e: (z_V[icon_V[2, e]] - z_V[icon_V[1, e]]) / 2, +1)
    aTt, agt, qzt = side(top_element, None, +1, dTdz_nodal,
                         lambda e: (x_V[icon_V[2, e]] - x_V[icon_V[3, e]]) / 2, +1)
    aTb, agb, qzb = side(bottom_element, None, -1, dTdz_nodal,
                         lambda e: (x_V[icon_V[1, e]] - x_V[icon_V[0, e]]) / 2, -1)
    aTl /= Lz
    aTr /= Lz
    aTb /= Lx
    aTt /= Lx
    agl /= Lz
    agr /= Lz
    agb /= Lx
    agt /= Lx
    Nu = np.abs(agt) / (aTb - aTt) * Lz                                 # :232
    return aTl, aTr, aTb, aTt, agl, agr, agb, agt, qxl, qxr, qzb, qzt, Nu


def compute_global_quantities(uq, wq, Tq, rhoq, JxWq, volume):
    """postprocessors.py:53-78: the vrms, mass and mean-T sums."""
    vrms = np.sqrt(_seqsum((uq ** 2 + wq ** 2) * JxWq) / volume)
    Tavrg = _seqsum(Tq * JxWq) / volume
    TM = _seqsum(rhoq * JxWq)
    return vrms, Tavrg, TM


def compute_global_quantities_full(uq, wq, Tq, rhoq, hcapaq, etaq, exxq, ezzq, exzq, gxq, gzq, JxWq, volume):
    """postprocessors.py:42-83, the whole returned tuple (vrms, EK, WAG, TVD, GPE, ITE, TM, Tavrg,
    eta_avrg); GPE stays 0 (its accumulation is commented out at :69); eta_avrg is None when the
    strain-rate sum is zero (the reference leaves the name unassigned)."""
    eII = exxq ** 2 + ezzq ** 2 + 2 * exzq ** 2
    TM = _seqsum(rhoq * JxWq)
    EK = _seqsum(0.5 * rhoq * (uq ** 2 + wq ** 2) * JxWq)
    WAG = -_seqsum(rhoq * (uq * gxq + wq * gzq) * JxWq)
    TVD = _seqsum(2 * etaq * (2 * exxq ** 2 / 3 + 2 * ezzq ** 2 / 3 - 2 * exxq * ezzq / 3 + 2 * exzq ** 2) * JxWq)
    ITE = _seqsum(rhoq * hcapaq * Tq * JxWq)
    vrms = np.sqrt(_seqsum((uq ** 2 + wq ** 2) * JxWq) / volume)
    Tavrg = _seqsum(Tq * JxWq) / volume
    num, denom = _seqsum(etaq * eII * JxWq), _seqsum(eII * JxWq)
    eta_avrg = num / denom if denom > 0 else None
    return vrms, EK, WAG, TVD, 0, ITE, TM, Tavrg, eta_avrg


def compute_dt(CFLnb, hx, hz, u, w, swarm_hcond, swarm_hcapa, swarm_rho, dt1_mem, dt2_mem, dt_max,
               solve_T=True):
    """meeuuw.py:2112-2139 (box): CFL and diffusion limits, 25 % growth limiter."""
    vel = np.sqrt(u ** 2 + w ** 2)
    dt1 = CFLnb * min(hx, hz) / np.max(vel)
    if solve_T:
        kappa = np.average(swarm_hcond) / np.average(swarm_hcapa) / np.average(swarm_rho)
        dt2 = CFLnb * min(hx, hz) ** 2 / kappa
    else:
        dt2 = 1e50
    dt1 = min(dt1, 1.25 * dt1_mem)
    dt2 = min(dt2, 1.25 * dt2_mem)
    return float(np.min([dt1, dt2, dt_max])), dt1, dt2
