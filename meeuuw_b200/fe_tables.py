"""Basis tables at the 3x3 Gauss points and at the Q2 nodes (set-up, host side).

Same values as the reference's set-up (quadrature_setup.py:13-15, basis_functions.py:16-138,
basis_functions_setup_q.py:47-76, basis_functions_setup_Vnodes.py); computed once and uploaded.
For the uniform box the Jacobian is constant: J = diag(hx/2, hz/2), JxW = hx*hz/4*w_q.
"""
import numpy as np
import torch

R_NODE = np.array([-1, 1, 1, -1, 0, 1, 0, -1, 0], dtype=np.float64)
T_NODE = np.array([-1, -1, 1, 1, -1, 0, 1, 0, 0], dtype=np.float64)


def gauss3():
    qc = np.array([-np.sqrt(3.0 / 5.0), 0.0, np.sqrt(3.0 / 5.0)])
    qw = np.array([5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0])
    return qc, qw


def _q2(r, s):
    return np.stack([0.5 * r * (r - 1.0) * 0.5 * s * (s - 1.0), 0.5 * r * (r + 1.0) * 0.5 * s * (s - 1.0),
                     0.5 * r * (r + 1.0) * 0.5 * s * (s + 1.0), 0.5 * r * (r - 1.0) * 0.5 * s * (s + 1.0),
                     (1.0 - r * r) * 0.5 * s * (s - 1.0), 0.5 * r * (r + 1.0) * (1.0 - s * s),
                     (1.0 - r * r) * 0.5 * s * (s + 1.0), 0.5 * r * (r - 1.0) * (1.0 - s * s),
                     (1.0 - r * r) * (1.0 - s * s)], axis=-1)


def _q2_dr(r, s):
    return np.stack([0.5 * (2.0 * r - 1.0) * 0.5 * s * (s - 1), 0.5 * (2.0 * r + 1.0) * 0.5 * s * (s - 1),
                     0.5 * (2.0 * r + 1.0) * 0.5 * s * (s + 1), 0.5 * (2.0 * r - 1.0) * 0.5 * s * (s + 1),
                     (-2.0 * r) * 0.5 * s * (s - 1), 0.5 * (2.0 * r + 1.0) * (1.0 - s * s),
                     (-2.0 * r) * 0.5 * s * (s + 1), 0.5 * (2.0 * r - 1.0) * (1.0 - s * s),
                     (-2.0 * r) * (1.0 - s * s)], axis=-1)


def _q2_dt(r, s):
    return np.stack([0.5 * r * (r - 1.0) * 0.5 * (2.0 * s - 1.0), 0.5 * r * (r + 1.0) * 0.5 * (2.0 * s - 1.0),
                     0.5 * r * (r + 1.0) * 0.5 * (2.0 * s + 1.0), 0.5 * r * (r - 1.0) * 0.5 * (2.0 * s + 1.0),
                     (1.0 - r * r) * 0.5 * (2.0 * s - 1.0), 0.5 * r * (r + 1.0) * (-2.0 * s),
                     (1.0 - r * r) * 0.5 * (2.0 * s + 1.0), 0.5 * r * (r - 1.0) * (-2.0 * s),
                     (1.0 - r * r) * (-2.0 * s)], axis=-1)


def _q1(r, s):
    return np.stack([0.25 * (1 - r) * (1 - s), 0.25 * (1 + r) * (1 - s), 0.25 * (1 + r) * (1 + s),
                     0.25 * (1 - r) * (1 + s)], axis=-1)


def _q1_dr(r, s):
    return np.stack([-0.25 * (1 - s), 0.25 * (1 - s), 0.25 * (1 + s), -0.25 * (1 + s)], axis=-1)


def _q1_dt(r, s):
    return np.stack([-0.25 * (1 - r), -0.25 * (1 + r), 0.25 * (1 + r), 0.25 * (1 - r)], axis=-1)


def host_tables():
    qc, qw = gauss3()
    rq = np.array([qc[i] for i in range(3) for j in range(3)])
    tq = np.array([qc[j] for i in range(3) for j in range(3)])
    wq = np.array([qw[i] * qw[j] for i in range(3) for j in range(3)])
    return dict(rq=rq, tq=tq, weightq=wq, N_V=_q2(rq, tq), dNdr_V=_q2_dr(rq, tq), dNdt_V=_q2_dt(rq, tq),
                N_P=_q1(rq, tq), dNdr_P=_q1_dr(rq, tq), dNdt_P=_q1_dt(rq, tq), N_P_n=_q1(R_NODE, T_NODE),
                dNdr_V_n=_q2_dr(R_NODE, T_NODE), dNdt_V_n=_q2_dt(R_NODE, T_NODE), qcoords=qc, qweights=qw)


_cache = {}


def device_tables(device="cuda"):
    key = str(device)
    if key not in _cache:
        _cache[key] = {k: torch.as_tensor(np.ascontiguousarray(v), dtype=torch.float64, device=device)
                       for k, v in host_tables().items()}
    return _cache[key]


def uniform_geometry(nel, hx, hz, device="cuda"):
    """JxWq and inverse-Jacobian arrays (nel, 9) of the uniform box (basis_functions_setup_q.py:60-70)."""
    t = host_tables()
    J00, J11 = hx / 2.0, hz / 2.0
    jxw = torch.as_tensor(J00 * J11 * t["weightq"], dtype=torch.float64, device=device).expand(nel, 9).contiguous()
    one = torch.ones(nel, 9, dtype=torch.float64, device=device)
    return dict(JxWq=jxw, jcbi00q=one * (1.0 / J00), jcbi01q=one * 0.0, jcbi10q=one * 0.0, jcbi11q=one * (1.0 / J11))
