"""Device drop-in for ``locate_particles`` (locate_particles.py:12-66), box geometry.

The reference's dispatcher calls the per-geometry locator and then exits with "r value out of
bounds" / "t value out of bounds" when a reduced coordinate leaves [-1, 1]
(locate_particles.py:61-64).  Here the bounds are tested on the device while locating and the
same SystemExit messages are raised.  Its diagnostic min/max prints (:57-59) are not repeated.
"""
import torch

from .. import _lib as L
from .. import ops
from ._common import back, box, box_dims, check_coords, dev, dev_u8, host_mode, raise_flags, f64


def locate_particles(geometry, nparticle, swarm_active, swarm_x, swarm_z, swarm_rad, swarm_theta, hx, hz, hrad,
                     htheta, x_V, z_V, rad_V, theta_V, icon_V, nelx, Rinner):
    if geometry != "box":
        raise NotImplementedError(f"the device path locates particles in the box geometry (got {geometry!r})")
    nel = icon_V.shape[1]
    nx, nz = box_dims(icon_V, nel)
    if nx != nelx:
        raise NotImplementedError("nelx does not match the connectivity")
    check_coords(x_V, z_V, nx, nz, hx, hz)
    host = host_mode(swarm_x, swarm_z, swarm_active)
    x, z, act = dev(swarm_x, f64)[:nparticle], dev(swarm_z, f64)[:nparticle], dev_u8(swarm_active)[:nparticle]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    r, t, iel = ops.locate(box(nx, nz, hx, hz), act, x, z, err=err)
    raise_flags(err, [(L.FLAG_ELEMENT_RANGE, "r value out of bounds"), (L.FLAG_R_OUT, "r value out of bounds"),
                      (L.FLAG_T_OUT, "t value out of bounds")])
    return back(r, host), back(t, host), back(iel, host)


__all__ = ["locate_particles"]
