"""Device drop-ins for ``project_nodal_{P,V,T}field_onto_qpoints``
(project_nodal_field_onto_qpoints.py:12-62): phiq[e, q] = sum_k N[q, k] phi[icon[k, e]].

The P variant is also called with icon_V and a nodal field on the V nodes (meeuuw.py:1516, 1549,
1581-1584): it then reads the 4 corner V nodes.  Both uses are recognised from the connectivity
passed in.
"""
from .. import _lib as L
from .. import ops
from ._common import back, box, box_dims, check_icon_P, dev, host_mode, f64


def _dims_from_P(icon, nel):
    """(nelx, nelz, space) for a Q1 table: the pressure connectivity or the V connectivity."""
    if icon.shape[0] == 9:
        nx, nz = box_dims(icon, nel)
        return nx, nz, L.SPACE_Q1_ON_V
    # icon_P (4, nel): nelx from the first element's top-left node (nelx + 1)
    ic0 = icon[:, 0].tolist() if hasattr(icon, "tolist") else list(icon[:, 0])
    nx = int(ic0[3]) - int(ic0[0]) - 1
    if nx < 1 or nel % nx:
        raise NotImplementedError("icon_P is not the box mesh's Q1 numbering")
    nz = nel // nx
    check_icon_P(icon, nx, nz)
    return nx, nz, L.SPACE_Q1


def project_nodal_Pfield_onto_qpoints(phi_nodal, nq_per_element, nel, m_P, N_P, icon_P):
    if (nq_per_element, m_P) != (9, 4):
        raise NotImplementedError("Q1 field with 3x3 Gauss quadrature")
    nx, nz, space = _dims_from_P(icon_P, nel)
    out = ops.nodal_to_qpoints(box(nx, nz), space, dev(N_P, f64), dev(phi_nodal, f64))
    return back(out, host_mode(phi_nodal))


def project_nodal_Vfield_onto_qpoints(phi_nodal, nq_per_element, nel, m_V, N_V, icon_V):
    if (nq_per_element, m_V) != (9, 9):
        raise NotImplementedError("Q2 field with 3x3 Gauss quadrature")
    nx, nz = box_dims(icon_V, nel)
    out = ops.nodal_to_qpoints(box(nx, nz), L.SPACE_Q2, dev(N_V, f64), dev(phi_nodal, f64))
    return back(out, host_mode(phi_nodal))


def project_nodal_Tfield_onto_qpoints(phi_nodal, nq_per_element, nel, m_T, N_T, icon_T):
    return project_nodal_Vfield_onto_qpoints(phi_nodal, nq_per_element, nel, m_T, N_T, icon_T)


__all__ = ["project_nodal_Pfield_onto_qpoints", "project_nodal_Vfield_onto_qpoints",
           "project_nodal_Tfield_onto_qpoints"]
