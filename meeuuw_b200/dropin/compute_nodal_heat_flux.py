"""Device drop-in for ``compute_nodal_heat_flux`` (compute_nodal_heat_flux.py:12-40): nodal -grad T
and -k grad T averaged over the incident elements.  Returns (dTdx_n, dTdy_n, qx_n, qy_n)."""
from .. import ops
from ._common import back, box, box_dims, dev, host_mode, f64


def compute_nodal_heat_flux(icon_T, T, hcond_nodal, nn_T, m_T, nel, dNdr_T_n, dNds_T_n, jcbi00_T, jcbi01_T, jcbi10_T,
                            jcbi11_T):
    nx, nz = box_dims(icon_T, nel)
    if m_T != 9 or nn_T != (2 * nx + 1) * (2 * nz + 1):
        raise ValueError("m_T / nn_T do not match the connectivity")
    tables = dict(dNdr_V_n=dev(dNdr_T_n, f64), dNdt_V_n=dev(dNds_T_n, f64))
    jc = tuple(dev(a, f64) for a in (jcbi00_T, jcbi01_T, jcbi10_T, jcbi11_T))
    out = ops.nodal_heat_flux(box(nx, nz), dev(T, f64), dev(hcond_nodal, f64), tables, jcbi=jc)
    host = host_mode(T)
    return tuple(back(o, host) for o in out)


__all__ = ["compute_nodal_heat_flux"]
