"""Device drop-ins for ``compute_global_quantities`` (postprocessors.py:14-83) and ``compute_Nu``
(postprocessors.py:114-248), box geometry.  Both are FP64 reductions on the device in a fixed
(deterministic) order; the scalars come back as numpy float64 values."""
import ctypes

import numpy as np
import torch

from .. import _lib as L
from .. import ops
from .._lib import call, ptr, stream_ptr
from ._common import box, box_dims, check_coords, dev, f64

L.extra_protos({
    "mw_global_quantities_full": (ctypes.c_int32, [ctypes.c_int64] + [ctypes.c_void_p] * 12 +
                                  [ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                   ctypes.c_void_p]),
})


def compute_global_quantities(nel, nq_per_element, xq, zq, uq, wq, Tq, rhoq, hcapaq, alphaq, etaq, exxq, ezzq, exzq,
                              dxxq, dzzq, dxzq, volume, JxWq, gxq, gzq):
    arrs = [dev(a, f64) for a in (uq, wq, Tq, rhoq, hcapaq, etaq, exxq, ezzq, exzq, gxq, gzq, JxWq)]
    nq = nel * nq_per_element
    if any(a.numel() != nq for a in arrs):
        raise ValueError("qpoint arrays must hold nel * nq_per_element values")
    out = torch.empty(9, dtype=f64, device="cuda")
    wp, wb = ops.workspace("post").get(L.lib().mw_post_workspace_bytes())
    call("mw_global_quantities_full", nq, *[ptr(a) for a in arrs], float(volume), ptr(out), wp, wb, stream_ptr())
    v = out.cpu().numpy()
    if np.isnan(v[8]):
        # the reference assigns eta_avrg only when the strain-rate sum is positive (:80-81)
        raise UnboundLocalError("cannot access local variable 'eta_avrg' where it is not associated with a value")
    vrms, EK, WAG, TVD, GPE, ITE, TM, Tavrg, eta_avrg = (np.float64(x) for x in v)
    return vrms, EK, WAG, TVD, 0, ITE, TM, Tavrg, eta_avrg


def compute_Nu(Lx, Lz, x_V, z_V, nel, left_element, right_element, top_element, bottom_element, icon_V, T, dTdx_nodal,
               dTdz_nodal, nq_per_dim, qcoords, qweights, hcond_n):
    nx, nz = box_dims(icon_V, nel)
    if nq_per_dim != 3:
        raise NotImplementedError("boundary integrals with 3 Gauss points per edge")
    check_coords(x_V, z_V, nx, nz, Lx / nx, Lz / nz)
    g = L.MwGauss3()
    for i in range(3):
        g.c[i], g.w[i] = float(qcoords[i]), float(qweights[i])
    out = torch.empty(13, dtype=f64, device="cuda")
    b = box(nx, nz, Lx=Lx, Lz=Lz)
    wp, wb = ops.workspace("nu").get(L.lib().mw_nu_workspace_bytes(b))
    # keep the device copies referenced until the kernels have run (the caching allocator would
    # otherwise hand a freed copy's memory to the next one)
    args = [dev(a, f64) for a in (T, dTdx_nodal, dTdz_nodal, hcond_n)]
    call("mw_compute_nu", b, *[ptr(a) for a in args], g, ptr(out), wp, wb, stream_ptr())
    res = out.cpu().numpy()
    del args
    return tuple(np.float64(x) for x in res)


__all__ = ["compute_global_quantities", "compute_Nu"]
