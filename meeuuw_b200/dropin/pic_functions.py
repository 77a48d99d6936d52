"""Device drop-ins for the particle-in-cell functions of ``pic_functions.py`` (box geometry).

Same names, positional arguments, return tuples and in-place contracts as the reference:
  * ``locate_particles___box``            pic_functions.py:108-137
  * ``interpolate_field_on_particles``    pic_functions.py:85-101
  * ``advect_particles___box``            pic_functions.py:180-292 (mutates swarm_x, swarm_z,
                                          swarm_active in place and returns them)
  * ``project_particles_on_elements``     pic_functions.py:603-650
  * ``project_particle_field_on_nodes_{1,2,3,4}``  pic_functions.py:659-1053
Per-node sums of the nodal projections run in the library's deterministic per-element order
(particles of an element in index order, elements ascending); ``EXACT_ORDER = True`` switches to
the reference's particle-index order (bit-identical sums, slower).
"""
import torch

from .. import _lib as L
from .. import ops
from ._common import back, box, box_dims, check_coords, copy_into, dev, dev_u8, host_mode, i32, f64

EXACT_ORDER = False


def locate_particles___box(nparticle, swarm_active, swarm_x, swarm_z, hx, hz, x_V, z_V, icon, nelx):
    nel = icon.shape[1]
    nx, nz = box_dims(icon, nel)
    if nx != nelx:
        raise NotImplementedError("nelx does not match the connectivity")
    check_coords(x_V, z_V, nx, nz, hx, hz)
    host = host_mode(swarm_x, swarm_z, swarm_active)
    b = box(nx, nz, hx, hz)
    x, z, act = dev(swarm_x, f64)[:nparticle], dev(swarm_z, f64)[:nparticle], dev_u8(swarm_active)[:nparticle]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    r, t, iel = ops.locate(b, act, x, z, err=err)
    if int(err.item()) & L.FLAG_ELEMENT_RANGE:
        raise IndexError("a particle lies outside the mesh (element index out of range)")
    return back(r, host), back(t, host), back(iel, host)


def interpolate_field_on_particles(nparticle, swarm_active, swarm_r, swarm_t, swarm_iel, phi, icon):
    nel = icon.shape[1]
    nx, nz = box_dims(icon, nel)
    host = host_mode(swarm_r, phi)
    (out,) = ops.interp(box(nx, nz), dev_u8(swarm_active)[:nparticle], dev(swarm_r, f64)[:nparticle],
                        dev(swarm_t, f64)[:nparticle], dev(swarm_iel, i32)[:nparticle], [dev(phi, f64)])
    return back(out, host)


def advect_particles___box(RKorder, dt, nparticle, swarm_x, swarm_z, swarm_active, u, w, Lx, Lz, hx, hz, nelx, icon,
                           x_V, z_V):
    nel = icon.shape[1]
    nx, nz = box_dims(icon, nel)
    if RKorder not in (1, 2, 4):
        raise ValueError(f"RKorder {RKorder} not available")
    check_coords(x_V, z_V, nx, nz, hx, hz)
    host = host_mode(swarm_x, swarm_z, u)
    b = box(nx, nz, hx, hz, Lx, Lz)
    x, z = dev(swarm_x, f64), dev(swarm_z, f64)
    act = dev_u8(swarm_active)
    up = torch.zeros(nparticle, dtype=f64, device="cuda")
    wp = torch.zeros(nparticle, dtype=f64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ops.advect(b, RKorder, float(dt), x[:nparticle], z[:nparticle], act[:nparticle], dev(u, f64), dev(w, f64), up, wp,
               err)
    # in-place contract of the reference (pic_functions.py:226-229)
    copy_into(swarm_x, x)
    copy_into(swarm_z, z)
    copy_into(swarm_active, act)
    return swarm_x, swarm_z, back(up, host), back(wp, host), swarm_active


def project_particles_on_elements(nel, nparticle, swarm_active, swarm_rho, swarm_eta, swarm_iel, averaging):
    if averaging not in L.AVG:
        raise ValueError(f"unknown averaging {averaging!r}")
    host = host_mode(swarm_rho, swarm_eta, swarm_iel)
    act, iel = dev_u8(swarm_active)[:nparticle], dev(swarm_iel, i32)[:nparticle]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    counts, offsets, order = ops.bin_particles(nel, act, iel, err=err)
    rho_e, eta_e = ops.project_elements(nel, offsets, order, dev(swarm_rho, f64)[:nparticle],
                                        dev(swarm_eta, f64)[:nparticle], averaging, err=err)
    return back(rho_e, host), back(eta_e, host), back(counts, host)


def _project_nodes(flavour, nel, nn_V, nparticle, swarm_active, swarm_phi, icon, swarm_iel, swarm_r, swarm_t,
                   averaging):
    if averaging not in L.AVG:
        raise ValueError(f"unknown averaging {averaging!r}")
    nx, nz = box_dims(icon, nel)
    if nn_V != (2 * nx + 1) * (2 * nz + 1):
        raise ValueError("nn_V does not match the connectivity")
    host = host_mode(swarm_phi, swarm_iel)
    act, iel = dev_u8(swarm_active)[:nparticle], dev(swarm_iel, i32)[:nparticle]
    counts, offsets, order = ops.bin_particles(nel, act, iel)
    (out,) = ops.project_nodes(box(nx, nz), flavour, [(dev(swarm_phi, f64)[:nparticle], averaging)], offsets, order,
                               dev(swarm_r, f64)[:nparticle], dev(swarm_t, f64)[:nparticle], exact_order=EXACT_ORDER)
    return back(out, host)


def project_particle_field_on_nodes_1(nel, nn_V, nparticle, swarm_active, swarm_phi, icon, swarm_iel, swarm_r,
                                      swarm_t, averaging):
    return _project_nodes(1, nel, nn_V, nparticle, swarm_active, swarm_phi, icon, swarm_iel, swarm_r, swarm_t,
                          averaging)


def project_particle_field_on_nodes_2(nel, nn_V, nparticle, swarm_active, swarm_phi, icon, swarm_iel, swarm_r,
                                      swarm_t, averaging):
    return _project_nodes(2, nel, nn_V, nparticle, swarm_active, swarm_phi, icon, swarm_iel, swarm_r, swarm_t,
                          averaging)


def project_particle_field_on_nodes_3(nel, nn_V, nparticle, swarm_active, swarm_phi, icon, swarm_iel, swarm_r,
                                      swarm_t, averaging):
    return _project_nodes(3, nel, nn_V, nparticle, swarm_active, swarm_phi, icon, swarm_iel, swarm_r, swarm_t,
                          averaging)


def project_particle_field_on_nodes_4(nel, nn_V, nparticle, swarm_active, swarm_phi, icon, swarm_iel, swarm_r,
                                      swarm_t, averaging):
    return _project_nodes(4, nel, nn_V, nparticle, swarm_active, swarm_phi, icon, swarm_iel, swarm_r, swarm_t,
                          averaging)


__all__ = ["locate_particles___box", "interpolate_field_on_particles", "advect_particles___box",
           "project_particles_on_elements", "project_particle_field_on_nodes_1", "project_particle_field_on_nodes_2",
           "project_particle_field_on_nodes_3", "project_particle_field_on_nodes_4"]
