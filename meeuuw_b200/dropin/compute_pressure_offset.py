"""Device drop-in for ``compute_pressure_offset`` (compute_pressure_offset.py:12-66), box
geometry: "none" -> 0, "surface" -> mean of the top-edge midpoints (:41-46), "volume" -> the
volume average of p (:56-61), any other value -> the reference's ValueError.  FP64 reductions in a
fixed order on the device."""
import numpy as np

from .. import ops
from ._common import box, check_icon_P, dev, require_box, f64


def _check_top(top_element, nelx, nel):
    te = top_element.cpu().numpy() if hasattr(top_element, "cpu") else np.asarray(top_element)
    want = np.zeros(nel, dtype=bool)
    want[nel - nelx:] = True
    if te.shape != (nel,) or not np.array_equal(te.astype(bool), want):
        raise NotImplementedError("top_element is not the top row of the box mesh")


def compute_pressure_offset(geometry, pressure_normalisation, axisymmetric, top_element, nel, nelx, nq_per_element, N_P,
                            JxWq, p, icon_P, theta_P, xq, volume):
    if pressure_normalisation not in ("none", "surface", "volume"):
        raise ValueError("compute_pressure_offset: unknown pressure_normalisation value")
    if pressure_normalisation == "none":
        return 0.
    require_box(geometry, axisymmetric)
    if nel % nelx:
        raise ValueError("nel is not a multiple of nelx")
    nz = nel // nelx
    check_icon_P(icon_P, nelx, nz)
    if pressure_normalisation == "surface":
        _check_top(top_element, nelx, nel)
    out = ops.pressure_offset(box(nelx, nz), pressure_normalisation, dev(p, f64), dev(N_P, f64), dev(JxWq, f64),
                              float(volume))
    return float(out.item())


__all__ = ["compute_pressure_offset"]
