"""Device drop-in for ``build_matrix_energy`` (build_matrix_energy.py:12-141), box mesh.

Crank-Nicolson element systems A_el = MM + dt/2 (Ka + Kd) and right-hand sides (BA and EBA
formulations), Dirichlet values eliminated symmetrically (:118-130).  Returns (VV_T [e, i, j]
element-major, rhs).  dpdxq, dpdzq are accepted and unused, as in the reference (:107 is
commented out).
"""
from .. import ops
from ._common import back, box, box_dims, dev, dev_u8, host_mode, f64


def build_matrix_energy(bignb, nel, nq_per_element, m_T, Nfem_T, T, icon_T, rhoq, etaq, Tq, uq, wq, hcondq, hcapaq,
                        alphaq, hprodq, exxq, ezzq, exzq, dpdxq, dpdzq, JxWq, N_T, dNdr_T, dNds_T, jcbi00q, jcbi01q,
                        jcbi10q, jcbi11q, bc_fix_T, bc_val_T, dt, formulation, rho0):
    if (nq_per_element, m_T) != (9, 9):
        raise NotImplementedError("the device path covers Q2 temperature with 3x3 Gauss quadrature")
    if formulation not in ("BA", "EBA"):
        raise NotImplementedError(f"formulation {formulation!r}")
    nx, nz = box_dims(icon_T, nel)
    if Nfem_T != (2 * nx + 1) * (2 * nz + 1):
        raise ValueError("Nfem_T does not match the connectivity")
    host = host_mode(T, rhoq, uq)
    names = dict(rhoq=rhoq, etaq=etaq, Tq=Tq, uq=uq, wq=wq, hcondq=hcondq, hcapaq=hcapaq, alphaq=alphaq,
                 hprodq=hprodq, JxWq=JxWq, jcbi00q=jcbi00q, jcbi01q=jcbi01q, jcbi10q=jcbi10q, jcbi11q=jcbi11q)
    if formulation == "EBA":
        names.update(exxq=exxq, ezzq=ezzq, exzq=exzq)
    q = {k: dev(v, f64) for k, v in names.items()}
    tables = dict(N_V=dev(N_T, f64), dNdr_V=dev(dNdr_T, f64), dNdt_V=dev(dNds_T, f64))
    VV, rhs = ops.assemble_energy(box(nx, nz), 0, dev(T, f64), q, tables, dev_u8(bc_fix_T), dev(bc_val_T, f64),
                                  float(dt), float(rho0), formulation)
    return back(VV, host), back(rhs, host)


__all__ = ["build_matrix_energy"]
