"""Oracle: particle-in-cell functions for the Cartesian box (vectorised over particles).

Test infrastructure only.  Restates ``pic_functions.py``:

* ``interpolate_vel_on_pt___box``        ``pic_functions.py:18-37``
* ``interpolate_field_on_particles``     ``pic_functions.py:85-101``
* ``locate_particles___box``             ``pic_functions.py:108-137`` (+ bounds check ``locate_particles.py:61-64``)
* ``advect_particles___box``             ``pic_functions.py:180-292``
* ``project_particles_on_elements``      ``pic_functions.py:603-650``
* ``project_particle_field_on_nodes_N``  ``pic_functions.py:659-1053``

Accumulations use ``np.add.at`` over particle-major arrays, so every node and
element receives its contributions in particle-index order, as in the
reference's sequential loops.
"""
import numpy as np

from .fe import basis_V


def _q2_dot(N, phi, icon, iel):
    """Sum_k N[:,k] * phi[icon[k, iel]] in k order (a 9-term dot product)."""
    acc = N[:, 0] * phi[icon[0, iel]]
    for k in range(1, 9):
        acc = acc + N[:, k] * phi[icon[k, iel]]
    return acc


def locate_particles___box(nparticle, swarm_active, swarm_x, swarm_z, hx, hz, x_V, z_V, icon, nelx):
    """pic_functions.py:108-137.  Inactive particles keep r=t=0, iel=0."""
    r = np.zeros(nparticle)
    t = np.zeros(nparticle)
    iel = np.zeros(nparticle, dtype=np.int32)
    a = np.asarray(swarm_active, dtype=bool)
    x, z = swarm_x[a], swarm_z[a]
    ielx = (x / hx).astype(np.int64)          # int() truncation, :131
    ielz = (z / hz).astype(np.int64)
    e = nelx * ielz + ielx
    r[a] = ((x - x_V[icon[0, e]]) / hx - 0.5) * 2
    t[a] = ((z - z_V[icon[0, e]]) / hz - 0.5) * 2
    iel[a] = e
    return r, t, iel


def locate_bounds_ok(r, t):
    """locate_particles.py:61-64: the driver exits if any r or t leaves [-1, 1]."""
    return not (r.min() < -1 or r.max() > 1 or t.min() < -1 or t.max() > 1)


def interpolate_field_on_particles(nparticle, swarm_active, swarm_r, swarm_t, swarm_iel, phi, icon):
    """pic_functions.py:85-101; inactive particles get 0."""
    out = np.zeros(nparticle)
    a = np.asarray(swarm_active, dtype=bool)
    N = basis_V(swarm_r[a], swarm_t[a])
    out[a] = _q2_dot(N, phi, icon, swarm_iel[a])
    return out


def interpolate_vel_on_pt___box(xp, zp, u, w, hx, hz, nelx, icon, x_V, z_V):
    """pic_functions.py:18-37 for arrays of points."""
    ielx = (xp / hx).astype(np.int64)
    ielz = (zp / hz).astype(np.int64)
    e = nelx * ielz + ielx
    rp = ((xp - x_V[icon[0, e]]) / hx - 0.5) * 2
    tp = ((zp - z_V[icon[0, e]]) / hz - 0.5) * 2
    N = basis_V(rp, tp)
    return _q2_dot(N, u, icon, e), _q2_dot(N, w, icon, e), e


def advect_particles___box(RKorder, dt, nparticle, swarm_x, swarm_z, swarm_active, u, w, Lx, Lz,
                           hx, hz, nelx, icon, x_V, z_V):
    """pic_functions.py:180-292.  Mutates swarm_x, swarm_z, swarm_active in place and returns them."""
    su = np.zeros(nparticle)
    sw = np.zeros(nparticle)
    act = swarm_active

    def out(x, z):
        return (x < 0) | (x > Lx) | (z < 0) | (z > Lz)

    idx = np.nonzero(act)[0]
    xA, zA = swarm_x[idx].copy(), swarm_z[idx].copy()
    uA, wA, _ = interpolate_vel_on_pt___box(xA, zA, u, w, hx, hz, nelx, icon, x_V, z_V)
    if RKorder == 1:                                                     # :220-231
        swarm_x[idx] = xA + uA * dt
        swarm_z[idx] = zA + wA * dt
        su[idx], sw[idx] = uA, wA
        act[idx[out(swarm_x[idx], swarm_z[idx])]] = False
    elif RKorder in (2, 4):
        xB = xA + uA * dt / 2.0                                          # :239
        zB = zA + wA * dt / 2.0
        bad = out(xB, zB)
        act[idx[bad]] = False
        ok = ~bad
        i2 = idx[ok]
        xA, zA, uA, wA, xB, zB = xA[ok], zA[ok], uA[ok], wA[ok], xB[ok], zB[ok]
        uB, wB, _ = interpolate_vel_on_pt___box(xB, zB, u, w, hx, hz, nelx, icon, x_V, z_V)
        if RKorder == 2:                                                 # :244-248
            swarm_x[i2] = xA + uB * dt
            swarm_z[i2] = zA + wB * dt
            su[i2], sw[i2] = uB, wB
        else:                                                            # :264-280
            xC = xA + uB * dt / 2.0
            zC = zA + wB * dt / 2.0
            bad = out(xC, zC)
            act[i2[bad]] = False
            ok = ~bad
            i3 = i2[ok]
            xA, zA, uA, wA, uB, wB, xC, zC = (v[ok] for v in (xA, zA, uA, wA, uB, wB, xC, zC))
            uC, wC, _ = interpolate_vel_on_pt___box(xC, zC, u, w, hx, hz, nelx, icon, x_V, z_V)
            xD = xA + uC * dt
            zD = zA + wC * dt
            bad = out(xD, zD)
            act[i3[bad]] = False
            ok = ~bad
            i4 = i3[ok]
            xA, zA, uA, wA, uB, wB, uC, wC, xD, zD = (v[ok] for v in (xA, zA, uA, wA, uB, wB, uC, wC, xD, zD))
            uD, wD, _ = interpolate_vel_on_pt___box(xD, zD, u, w, hx, hz, nelx, icon, x_V, z_V)
            su[i4] = (uA + 2 * uB + 2 * uC + uD) / 6
            sw[i4] = (wA + 2 * wB + 2 * wC + wD) / 6
            swarm_x[i4] = xA + su[i4] * dt
            swarm_z[i4] = zA + sw[i4] * dt
    else:
        raise ValueError("RKorder must be 1, 2 or 4")
    dead = ~act                                                          # :287-290
    swarm_x[dead] = 0
    swarm_z[dead] = 0
    return swarm_x, swarm_z, su, sw, act


def project_particles_on_elements(nel, nparticle, swarm_active, swarm_rho, swarm_eta, swarm_iel, averaging):
    """pic_functions.py:603-650 (counts int32; rho arithmetic; eta by ``averaging``)."""
    a = np.asarray(swarm_active, dtype=bool)
    e = swarm_iel[a]
    rho_e = np.zeros(nel)
    eta_e = np.zeros(nel)
    cnt = np.zeros(nel, dtype=np.int32)
    np.add.at(rho_e, e, swarm_rho[a])
    np.add.at(cnt, e, 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        rho_e /= cnt
        if averaging == "arithmetic":
            np.add.at(eta_e, e, swarm_eta[a])
            eta_e /= cnt
        elif averaging == "geometric":
            np.add.at(eta_e, e, np.log10(swarm_eta[a]))
            eta_e = 10.0 ** (eta_e / cnt)
        elif averaging == "harmonic":
            np.add.at(eta_e, e, 1.0 / swarm_eta[a])
            eta_e = cnt / eta_e
        else:
            raise ValueError("unknown averaging")
    return rho_e, eta_e, cnt


def _transform(phi, averaging):
    if averaging == "arithmetic":
        return phi
    if averaging == "geometric":
        return np.log10(phi)
    if averaging == "harmonic":
        return 1.0 / phi
    raise ValueError("unknown averaging")


def _finish(phi_nodal, count_nodal, averaging):
    with np.errstate(divide="ignore", invalid="ignore"):
        if averaging == "arithmetic":
            return phi_nodal / count_nodal
        if averaging == "geometric":
            return 10 ** (phi_nodal / count_nodal)
        return count_nodal / phi_nodal


def _fill_q2(phi_nodal, icon):
    """pic_functions.py:801-809: edge/centre nodes from the 4 corners."""
    c0, c1, c2, c3 = (phi_nodal[icon[k]] for k in range(4))
    phi_nodal[icon[4]] = 0.50 * (c0 + c1)
    phi_nodal[icon[5]] = 0.50 * (c1 + c2)
    phi_nodal[icon[6]] = 0.50 * (c2 + c3)
    phi_nodal[icon[7]] = 0.50 * (c0 + c3)
    phi_nodal[icon[8]] = 0.25 * (c0 + c1 + c2 + c3)
    return phi_nodal


def project_particle_field_on_nodes(flavour, nel, nn_V, nparticle, swarm_active, swarm_phi, icon,
                                    swarm_iel, swarm_r, swarm_t, averaging):
    """pic_functions.py:659-1053, flavours 1..4, in particle-index order per node."""
    a = np.nonzero(np.asarray(swarm_active, dtype=bool))[0]
    e = swarm_iel[a]
    r, t = swarm_r[a], swarm_t[a]
    v = _transform(swarm_phi[a], averaging)
    nodes = np.stack([icon[k, e] for k in range(4)], axis=1)          # (np, 4) particle-major
    if flavour == 1:                                                  # :678-700
        w = np.ones((len(a), 4))
        use = np.ones((len(a), 4), dtype=bool)
    elif flavour == 2:                                                # :756-783
        w = np.stack([0.25 * (1 - r) * (1 - t), 0.25 * (1 + r) * (1 - t),
                      0.25 * (1 + r) * (1 + t), 0.25 * (1 - r) * (1 + t)], axis=1)
        use = np.ones((len(a), 4), dtype=bool)
    elif flavour in (3, 4):                                           # :845-858, :961-979
        use = np.stack([(r <= 0) & (t <= 0), (r >= 0) & (t <= 0),
                        (r >= 0) & (t >= 0), (r <= 0) & (t >= 0)], axis=1)
        if flavour == 3:
            w = np.ones((len(a), 4))
        else:
            w = np.stack([-r * -t, (1 - r) * -t, (1 - r) * (1 - t), -r * (1 - t)], axis=1)
    else:
        raise ValueError("flavour must be 1..4")
    phi_nodal = np.zeros(nn_V)
    if flavour in (1, 3):
        count = np.zeros(nn_V, dtype=np.int16)                        # :676, :838
        np.add.at(count, nodes[use], 1)
    else:
        count = np.zeros(nn_V)
        np.add.at(count, nodes[use], (1 * w)[use])
    if flavour in (1, 3):
        np.add.at(phi_nodal, nodes[use], np.broadcast_to(v[:, None], w.shape)[use])
    else:
        np.add.at(phi_nodal, nodes[use], (v[:, None] * w)[use])
    return _fill_q2(_finish(phi_nodal, count, averaging), icon)
