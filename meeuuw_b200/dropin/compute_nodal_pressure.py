"""Device drop-in for ``compute_nodal_pressure`` (compute_nodal_pressure.py:8-21): q on the V nodes
as the average over incident elements of the Q1 pressure evaluated at the node (N_P_n)."""
import torch

from .. import ops
from ._common import back, box, box_dims, check_icon_P, dev, host_mode, f64


def compute_nodal_pressure(m_V, nn_V, icon_V, icon_P, p, N_P_n):
    nel = icon_V.shape[1]
    nx, nz = box_dims(icon_V, nel)
    check_icon_P(icon_P, nx, nz)
    if m_V != 9 or nn_V != (2 * nx + 1) * (2 * nz + 1):
        raise ValueError("m_V / nn_V do not match the connectivity")
    zero = torch.zeros(1, dtype=f64, device="cuda")
    q = ops.nodal_pressure(box(nx, nz), dev(p, f64), zero, dev(N_P_n, f64), subtract=False)
    return back(q, host_mode(p))


__all__ = ["compute_nodal_pressure"]
