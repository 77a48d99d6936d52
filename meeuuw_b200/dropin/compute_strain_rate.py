"""Device drop-in for ``compute_nodal_strain_rate`` (compute_strain_rate.py:51-73): element-local
strain rates at the element's nodes, averaged over the incident elements."""
from .. import ops
from ._common import back, box, box_dims, dev, host_mode, f64


def compute_nodal_strain_rate(icon_V, u, v, nn_V, m_V, nel, dNdr_V_n, dNds_V_n, jcbi00n, jcbi01n, jcbi10n, jcbi11n):
    nx, nz = box_dims(icon_V, nel)
    if m_V != 9 or nn_V != (2 * nx + 1) * (2 * nz + 1):
        raise ValueError("m_V / nn_V do not match the connectivity")
    tables = dict(dNdr_V_n=dev(dNdr_V_n, f64), dNdt_V_n=dev(dNds_V_n, f64))
    jc = tuple(dev(a, f64) for a in (jcbi00n, jcbi01n, jcbi10n, jcbi11n))
    exx, ezz, exz = ops.nodal_strain_rate(box(nx, nz), dev(u, f64), dev(v, f64), tables, jcbi=jc)
    host = host_mode(u, v)
    return back(exx, host), back(ezz, host), back(exz, host)


__all__ = ["compute_nodal_strain_rate"]
