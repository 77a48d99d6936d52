"""Device drop-in for ``build_matrix_stokes`` (build_matrix_stokes.py:19-278), plane-strain box.

Returns the reference's 9-tuple (VV_Stokes, rhs_f, rhs_h, VV_K, VV_G, VV_GT, VV_M, VV_M_eta, VV_H)
with the same element-major value layouts (full: per row 18 K values then 4 (G, G^T) pairs,
:268-276; blocks: VV_K [e, i, j], VV_G [e, i, k], VV_GT and VV_H [e, k, i], VV_M and VV_M_eta
[e, k, l]) and zero-length arrays for the layout not requested.  Dirichlet rows and columns are
eliminated as at :206-217.  The values are assembled in FP64 on the device; the operator is also
recorded for the solver drop-ins.
"""
import numpy as np
import torch

from .. import ops
from . import _operator
from ._common import back, box, box_dims, check_icon_P, dev, dev_u8, host_mode, require_box, f64

_geometry_checked = {}


def _uniform_spacing(jcbi00q, jcbi01q, jcbi10q, jcbi11q):
    """hx, hz of an axis-aligned uniform mesh (jcbi = diag(2/hx, 2/hz) everywhere, to 1e-10
    relative), else raise."""
    key = tuple(int(t.data_ptr()) for t in (jcbi00q, jcbi01q, jcbi10q, jcbi11q))
    hit = _geometry_checked.get(key)
    if hit is not None:
        return hit
    # the reference computes the Jacobian numerically: off-diagonal terms carry rounding noise
    a, b = float(jcbi00q.mean().item()), float(jcbi11q.mean().item())
    tol = 1e-10 * max(abs(a), abs(b))
    ok = float((jcbi00q - a).abs().max().item()) <= tol and float((jcbi11q - b).abs().max().item()) <= tol and \
        float(jcbi01q.abs().max().item()) <= tol and float(jcbi10q.abs().max().item()) <= tol
    if not ok:
        raise NotImplementedError("the device path covers uniform axis-aligned box meshes")
    hit = (2.0 / a, 2.0 / b)
    _geometry_checked[key] = hit
    return hit


def build_matrix_stokes(bignb_Stokes, bignb_K, bignb_M, bignb_G, nel, nq_per_element, m_V, m_P, ndof_V, Nfem_V, Nfem_P,
                        ndof_V_el, icon_V, icon_P, rhoq, etaq, JxWq, local_to_globalV, gxq, gyq, N_V, N_P, dNdr_V,
                        dNdt_V, dNdr_P, dNdt_P, jcbi00q, jcbi01q, jcbi10q, jcbi11q, eta_e, eta_ref, L_ref, bc_fix_V,
                        bc_val_V, bot_element, top_element, bot_free_slip, top_free_slip, geometry, theta_V,
                        axisymmetric, xq, blocks):
    require_box(geometry, axisymmetric)
    if (nq_per_element, m_V, m_P, ndof_V, ndof_V_el) != (9, 9, 4, 2, 18):
        raise NotImplementedError("the device path covers Q2xQ1 elements with 3x3 Gauss quadrature")
    nx, nz = box_dims(icon_V, nel)
    check_icon_P(icon_P, nx, nz)
    if Nfem_V != 2 * (2 * nx + 1) * (2 * nz + 1) or Nfem_P != (nx + 1) * (nz + 1):
        raise ValueError("Nfem_V / Nfem_P do not match the connectivity")
    host = host_mode(rhoq, etaq, JxWq)
    q = dict(rhoq=dev(rhoq, f64), etaq=dev(etaq, f64), JxWq=dev(JxWq, f64), jcbi00q=dev(jcbi00q, f64),
             jcbi01q=dev(jcbi01q, f64), jcbi10q=dev(jcbi10q, f64), jcbi11q=dev(jcbi11q, f64), gxq=dev(gxq, f64),
             gzq=dev(gyq, f64), eta_e=dev(eta_e, f64))
    tables = dict(N_V=dev(N_V, f64), N_P=dev(N_P, f64), dNdr_V=dev(dNdr_V, f64), dNdt_V=dev(dNdt_V, f64),
                  dNdr_P=dev(dNdr_P, f64), dNdt_P=dev(dNdt_P, f64))
    hx, hz = _uniform_spacing(q["jcbi00q"], q["jcbi01q"], q["jcbi10q"], q["jcbi11q"])
    b = box(nx, nz, hx, hz)
    fix = dev_u8(bc_fix_V)
    out = ops.assemble_stokes(b, bool(blocks), 0, q, tables, fix, dev(bc_val_V, f64), eta_ref, L_ref)
    Kvals = out["VV_K"] if blocks else out["VV_Stokes"].view(nel, 18, 26)[:, :, :18]
    _operator.record(_operator.Operator(b, q["etaq"], q["eta_e"], fix, eta_ref, L_ref, Nfem_V, Nfem_P,
                                        float(Kvals.sum().item()), float(Kvals.abs().sum().item())))
    empty = np.zeros(0) if host else torch.zeros(0, dtype=f64, device="cuda")
    r = lambda k: back(out[k], host)
    if blocks:
        return (empty, r("rhs_f"), r("rhs_h"), r("VV_K"), r("VV_G"), r("VV_GT"), r("VV_M"), r("VV_M_eta"), r("VV_H"))
    return (r("VV_Stokes"), r("rhs_f"), r("rhs_h"), empty, empty, empty, empty, empty, empty)


__all__ = ["build_matrix_stokes"]
