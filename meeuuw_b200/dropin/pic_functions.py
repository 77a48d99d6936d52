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


# ---------------------------------------------------------------- least squares, population control
def _ls(order, nel, x_e, z_e, swarm_x, swarm_z, swarm_iel, swarm_rho, swarm_eta):
    nelx, nelz = _box_of_centres(x_e, z_e, nel)
    host = host_mode(swarm_x, swarm_rho)
    n = len(swarm_x)
    iel = dev(swarm_iel, i32)[:n]
    every = torch.ones(n, dtype=torch.uint8, device="cuda")        # the reference's mask: swarm_iel == iel
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    counts, offsets, order_ = ops.bin_particles(nel, every, iel, err=err)
    b = box(nelx, nelz, 2 * float(x_e[0]), 2 * float(z_e[0]))
    out = ops.ls_fit(b, order, offsets, order_, dev(swarm_x, f64)[:n], dev(swarm_z, f64)[:n],
                     [dev(swarm_rho, f64)[:n], dev(swarm_eta, f64)[:n]], err=err)
    if int(err.item()) & L.FLAG_EMPTY_ELEMENT:
        raise ValueError("least squares fit: an element contains no particle")
    (cr, rmin, rmax), (ce, emin, emax) = out
    coefs = [back(cr[:, j].contiguous(), host) for j in range(order)] + \
            [back(ce[:, j].contiguous(), host) for j in range(order)]
    return tuple(coefs) + (back(rmin, host), back(rmax, host), back(emin, host), back(emax, host))


def _box_of_centres(x_e, z_e, nel):
    """(nelx, nelz) of a uniform box from its element centres (x_V of node 8)."""
    xe = x_e.detach().cpu().numpy() if isinstance(x_e, torch.Tensor) else x_e
    ze = z_e.detach().cpu().numpy() if isinstance(z_e, torch.Tensor) else z_e
    nelx = int(round(float(xe.max() - xe.min()) / float(2 * xe[0]))) + 1 if nel > 1 else 1
    if nelx < 1 or nel % nelx:
        raise NotImplementedError("least squares fits: element centres of a uniform box expected")
    return nelx, nel // nelx


def compute_ls_coefficients_P1(nel, x_e, z_e, swarm_x, swarm_z, swarm_iel, swarm_rho, swarm_eta):
    """pic_functions.py:1098-1172: (rho a, b, c, eta a, b, c, rho min, max, eta min, max)."""
    return _ls(3, nel, x_e, z_e, swarm_x, swarm_z, swarm_iel, swarm_rho, swarm_eta)


def compute_ls_coefficients_Q1(nel, x_e, z_e, swarm_x, swarm_z, swarm_iel, swarm_rho, swarm_eta):
    """pic_functions.py:1182-1285: (rho a, b, c, d, eta a, b, c, d, rho min, max, eta min, max)."""
    return _ls(4, nel, x_e, z_e, swarm_x, swarm_z, swarm_iel, swarm_rho, swarm_eta)


def population_control(istep, x_V, z_V, icon_V, nel, nparticle_min, nparticle, nparticle_e, swarm_active, swarm_id,
                       swarm_iel, swarm_r, swarm_t, swarm_x, swarm_z, swarm_u, swarm_w, swarm_strain, swarm_eta,
                       swarm_wf, swarm_F, swarm_paint, use_melting, nmat, ptcl_active_file, output_folder):
    """pic_functions.py:1621-1812 on the device, in place.  The reduced coordinates come from
    Python's `random` exactly as the reference draws them (random.uniform(-0.95, 0.95), r then t,
    per added particle); the weight fractions of each new particle are copied from the nearest
    particle, strain (and melt fraction) averaged over its element, paint set to -1."""
    import random

    import numpy as np
    nx, nz = box_dims(icon_V, nel)
    ne = np.asarray(nparticle_e.detach().cpu().numpy() if isinstance(nparticle_e, torch.Tensor) else nparticle_e)
    needed = int(np.maximum(0, nparticle_min - ne).sum())
    print("     -> nparticle_min=", nparticle_min)
    print("     -> number of needed particles", needed)
    if needed == 0:
        print("     -> no population control needed")
        return
    act = dev_u8(swarm_active)
    available = int(nparticle - int(act.sum().item()))
    ptcl_active_file.write("%d %d %d %d\n" % (istep, nparticle - available, needed, available))
    ptcl_active_file.flush()
    if needed > available:
        raise ValueError("population_control: not available yet")
    draws = torch.tensor([random.random() for _ in range(2 * needed)], dtype=f64, device="cuda")
    xv = x_V.detach().cpu().numpy() if isinstance(x_V, torch.Tensor) else np.asarray(x_V)
    zv = z_V.detach().cpu().numpy() if isinstance(z_V, torch.Tensor) else np.asarray(z_V)
    hx, hz = 2 * float(xv[1] - xv[0]), 2 * float(zv[2 * nx + 1] - zv[0])   # x-fastest Q2 lattice
    check_coords(x_V, z_V, nx, nz, hx, hz)
    b = box(nx, nz, hx, hz)
    iel = dev(swarm_iel, i32)
    counts, offsets, order = ops.bin_particles(nel, act, iel)      # the mask: active, swarm_iel == iel
    x, z, r, t = dev(swarm_x, f64), dev(swarm_z, f64), dev(swarm_r, f64), dev(swarm_t, f64)
    avg = [dev(a, f64) for a in (swarm_eta, swarm_u, swarm_w, swarm_strain)]
    if use_melting:
        avg.append(dev(swarm_F, f64))
    src = torch.full((nparticle,), -1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ops.population_control(b, int(nparticle_min), dev(ne, i32), offsets, order, act, iel, r, t, x, z, avg=avg,
                           source=src, draws=draws, err=err)
    flags = int(err.item())
    if flags & L.FLAG_POP_MASK_EMPTY:
        raise ValueError("population_control: mask empty")
    if flags & L.FLAG_POP_UNAVAILABLE:
        raise ValueError("population_control: not available yet")
    new = torch.nonzero(src >= 0).flatten()
    wf = dev(swarm_wf, f64)
    wf[:, new] = wf[:, src[new].long()]
    paint = dev(swarm_paint)
    paint[new] = -1
    for dst, s in ((swarm_active, act), (swarm_iel, iel), (swarm_r, r), (swarm_t, t), (swarm_x, x), (swarm_z, z),
                   (swarm_eta, avg[0]), (swarm_u, avg[1]), (swarm_w, avg[2]), (swarm_strain, avg[3]),
                   (swarm_wf, wf), (swarm_paint, paint)):
        copy_into(dst, s)
    if use_melting:
        copy_into(swarm_F, avg[4])


__all__ += ["compute_ls_coefficients_P1", "compute_ls_coefficients_Q1", "population_control"]
