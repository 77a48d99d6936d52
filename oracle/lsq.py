"""Oracle: least-squares particle projections, their slope limiter, and population control.

Test infrastructure only.  Restates:

* ``limiter``                      ``pic_functions.py:1068-1089`` (slope limiter of a P1 fit)
* ``compute_ls_coefficients_P1``   ``pic_functions.py:1098-1172`` (a + b dx + c dz per element)
* ``compute_ls_coefficients_Q1``   ``pic_functions.py:1182-1285`` (+ d dx dz)
* the qpoint evaluation of the fits ``meeuuw.py:1517-1532`` / ``:1547-1562``
* the limiter loop of the driver    ``meeuuw.py:1241-1248`` (P1 only; h = hx)
* ``population_control``           ``pic_functions.py:1621-1812``

The fits follow the reference's mask ``swarm_iel == iel`` (active or not: inactive particles
carry iel = 0 after locate and so take part in element 0's fit), accumulate the normal
equations particle by particle in index order, and solve them with numpy's LAPACK solve.
"""
import numpy as np


def _sign(v):
    """pic_functions.py:1061-1064: -1 for negative values, +1 otherwise (also for -0.0)."""
    return -1.0 if v < 0 else 1.0


def limiter(c_0, c_1, c_2, S=0, L=1, h=1):
    """pic_functions.py:1068-1089."""
    k_u = min(c_0 - S, L - c_0)
    k_l = (abs(c_1) + abs(c_2)) * h / 2
    if k_l > k_u:
        c_max = k_u * 2 / h
        c_1 = _sign(c_1) * min(abs(c_1), c_max)
        c_2 = _sign(c_2) * min(abs(c_2), c_max)
    k_l = (abs(c_1) + abs(c_2)) * h / 2
    if k_l > k_u:
        c_change = (k_l - k_u) / h
        c_1 = _sign(c_1) * (abs(c_1) - c_change)
        c_2 = _sign(c_2) * (abs(c_2) - c_change)
    return c_1, c_2


def ls_coefficients(order, nel, x_e, z_e, swarm_x, swarm_z, swarm_iel, fields):
    """compute_ls_coefficients_P1 (order 3) / _Q1 (order 4) for any number of particle fields.

    Returns (coefs, fmin, fmax): coefs[f] is (nel, order); fmin/fmax[f] the particle extrema per
    element."""
    nf = len(fields)
    coefs = [np.zeros((nel, order)) for _ in range(nf)]
    fmin = [np.zeros(nel) for _ in range(nf)]
    fmax = [np.zeros(nel) for _ in range(nf)]
    order_p = np.argsort(swarm_iel, kind="stable")                 # particles of each element, index order
    bounds = np.searchsorted(swarm_iel[order_p], np.arange(nel + 1))
    for e in range(nel):
        idx = order_p[bounds[e]:bounds[e + 1]]
        sx = swarm_x[idx] - x_e[e]
        sz = swarm_z[idx] - z_e[e]
        A = np.zeros((order, order))
        rhs = np.zeros((nf, order))
        A[0, 0] = len(idx)
        for ip in range(len(idx)):                                 # :1134-1146 / :1226-1246
            x, z = sx[ip], sz[ip]
            A[0, 1] += x
            A[0, 2] += z
            if order == 4:
                A[0, 3] += x * z
            A[1, 1] += x ** 2
            A[1, 2] += x * z
            if order == 4:
                A[1, 3] += x ** 2 * z
            A[2, 2] += z ** 2
            if order == 4:
                A[2, 3] += x * z ** 2
                A[3, 3] += x ** 2 * z ** 2
            for f in range(nf):
                v = fields[f][idx[ip]]
                rhs[f, 0] += v
                rhs[f, 1] += v * x
                rhs[f, 2] += v * z
                if order == 4:
                    rhs[f, 3] += v * x * z
        for i in range(order):
            for j in range(i):
                A[i, j] = A[j, i]
        for f in range(nf):
            coefs[f][e] = np.linalg.solve(A, rhs[f])
            vals = fields[f][idx]
            fmin[f][e] = np.min(vals)
            fmax[f][e] = np.max(vals)
    return coefs, fmin, fmax


def limit_p1(coef, fmin, fmax, h):
    """meeuuw.py:1241-1248: the slopes of every element's P1 fit through limiter(), h = hx."""
    out = coef.copy()
    for e in range(len(coef)):
        out[e, 1], out[e, 2] = limiter(coef[e, 0], coef[e, 1], coef[e, 2], fmin[e], fmax[e], h)
    return out


def ls_to_qpoints(coef, xq, zq, x_e, z_e):
    """meeuuw.py:1517-1532: a + b (xq - x_e) + c (zq - z_e) [+ d (xq - x_e)(zq - z_e)]."""
    dx = xq - x_e[:, None]
    dz = zq - z_e[:, None]
    out = coef[:, 0:1] + coef[:, 1:2] * dx + coef[:, 2:3] * dz
    if coef.shape[1] == 4:
        out = out + coef[:, 3:4] * dx * dz
    return out


def population_control(x_V, z_V, icon_V, nel, nparticle_min, nparticle_e, swarm_active, swarm_iel, swarm_r,
                       swarm_t, swarm_x, swarm_z, swarm_u, swarm_w, swarm_eta, swarm_mat, draws):
    """pic_functions.py:1621-1812 on the arrays the box path carries (material id in place of the
    weight fractions; no strain, paint or melt fields).  Mutates the swarm arrays in place.
    draws: the uniform [0, 1) numbers the reference's random.uniform(-0.95, 0.95) calls consume,
    two per added particle (r then t).  Returns the number of particles added; raises ValueError
    with the reference's messages."""
    from .fe import basis_V
    need = np.maximum(0, nparticle_min - nparticle_e)
    needed = int(need.sum())                                        # :1655-1657
    if needed == 0:
        return 0
    available = np.flatnonzero(~swarm_active.astype(bool))          # :1680-1688
    if needed > len(available):
        raise ValueError("population_control: not available yet")   # :1722-1733
    counter = 0
    lo, hi = -0.95, 0.95
    for e in np.flatnonzero(nparticle_e < nparticle_min):           # :1739-1799
        mask = (swarm_iel == e) & swarm_active.astype(bool)
        if mask.sum() == 0:
            raise ValueError("population_control: mask empty")
        ids = np.flatnonzero(mask)
        mx, mz = swarm_x[mask].copy(), swarm_z[mask].copy()
        avg_eta, avg_u, avg_w = np.average(swarm_eta[mask]), np.average(swarm_u[mask]), np.average(swarm_w[mask])
        for _ in range(int(need[e])):
            pid = available[counter]
            swarm_active[pid] = True
            swarm_iel[pid] = e
            swarm_r[pid] = lo + (hi - lo) * draws[2 * counter]
            swarm_t[pid] = lo + (hi - lo) * draws[2 * counter + 1]
            N = basis_V(np.array([swarm_r[pid]]), np.array([swarm_t[pid]]))[0]
            swarm_x[pid] = np.dot(N, x_V[icon_V[:, e]])
            swarm_z[pid] = np.dot(N, z_V[icon_V[:, e]])
            dist = (mx - swarm_x[pid]) ** 2 + (mz - swarm_z[pid]) ** 2
            swarm_mat[pid] = swarm_mat[ids[np.argmin(dist)]]
            swarm_eta[pid] = avg_eta
            swarm_u[pid] = avg_u
            swarm_w[pid] = avg_w
            counter += 1
    return counter


def splitmix_u01(seed, n):
    """The device generator of population control (k_pc_fill's splitmix_u01): n uniform [0, 1)
    numbers for key `seed`, the k-th from the SplitMix64 finaliser of seed + (k + 1) * golden."""
    with np.errstate(over="ignore"):
        k = np.arange(n, dtype=np.uint64)
        z = np.uint64(seed) + (k + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
