"""Oracle: structured Q2xQ1 box mesh, basis tables and COO index arrays.

Test infrastructure only (see ``oracle/__init__.py``).  Restates the reference's
set-up stage for the Cartesian box:

* Gauss rules ............ ``quadrature_setup.py:13-15``
* Q2 / Q1 bases .......... ``basis_functions.py:16-138``
* V nodes ................ ``build_velocity_mesh.py:113-145``
* icon_V ................. ``build_velocity_connectivity.py:63-92``
* P nodes / icon_P ....... ``build_pressure_mesh.py``, ``build_pressure_connectivity.py``
* Jacobians at qpoints ... ``basis_functions_setup_q.py:47-76``
* Jacobians at V nodes ... ``basis_functions_setup_Vnodes.py``
* local_to_globalV, II/JJ  ``meeuuw.py:874-1017``
"""
import numpy as np

R_V = np.array([-1, 1, 1, -1, 0, 1, 0, -1, 0], dtype=np.float64)  # basis_functions.py:16
T_V = np.array([-1, -1, 1, 1, -1, 0, 1, 0, 0], dtype=np.float64)  # basis_functions.py:17


def quadrature_setup(nq_per_dim=3):
    """quadrature_setup.py:13-15 (3-point Gauss-Legendre)."""
    if nq_per_dim != 3:
        raise ValueError("only nq_per_dim=3 is on the hot path")
    qcoords = [-np.sqrt(3.0 / 5.0), 0.0, np.sqrt(3.0 / 5.0)]
    qweights = [5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0]
    return qcoords, qweights


def basis_V(r, s):
    """basis_functions.py:20-30, same operation order."""
    r = np.asarray(r, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    N0 = 0.5 * r * (r - 1.0) * 0.5 * s * (s - 1.0)
    N1 = 0.5 * r * (r + 1.0) * 0.5 * s * (s - 1.0)
    N2 = 0.5 * r * (r + 1.0) * 0.5 * s * (s + 1.0)
    N3 = 0.5 * r * (r - 1.0) * 0.5 * s * (s + 1.0)
    N4 = (1.0 - r * r) * 0.5 * s * (s - 1.0)
    N5 = 0.5 * r * (r + 1.0) * (1.0 - s * s)
    N6 = (1.0 - r * r) * 0.5 * s * (s + 1.0)
    N7 = 0.5 * r * (r - 1.0) * (1.0 - s * s)
    N8 = (1.0 - r * r) * (1.0 - s * s)
    return np.stack([N0, N1, N2, N3, N4, N5, N6, N7, N8], axis=-1)


def basis_V_dr(r, s):
    """basis_functions.py:34-44."""
    r = np.asarray(r, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    d = [0.5 * (2.0 * r - 1.0) * 0.5 * s * (s - 1),
         0.5 * (2.0 * r + 1.0) * 0.5 * s * (s - 1),
         0.5 * (2.0 * r + 1.0) * 0.5 * s * (s + 1),
         0.5 * (2.0 * r - 1.0) * 0.5 * s * (s + 1),
         (-2.0 * r) * 0.5 * s * (s - 1),
         0.5 * (2.0 * r + 1.0) * (1.0 - s * s),
         (-2.0 * r) * 0.5 * s * (s + 1),
         0.5 * (2.0 * r - 1.0) * (1.0 - s * s),
         (-2.0 * r) * (1.0 - s * s)]
    return np.stack(d, axis=-1)


def basis_V_dt(r, s):
    """basis_functions.py:48-58."""
    r = np.asarray(r, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    d = [0.5 * r * (r - 1.0) * 0.5 * (2.0 * s - 1.0),
         0.5 * r * (r + 1.0) * 0.5 * (2.0 * s - 1.0),
         0.5 * r * (r + 1.0) * 0.5 * (2.0 * s + 1.0),
         0.5 * r * (r - 1.0) * 0.5 * (2.0 * s + 1.0),
         (1.0 - r * r) * 0.5 * (2.0 * s - 1.0),
         0.5 * r * (r + 1.0) * (-2.0 * s),
         (1.0 - r * r) * 0.5 * (2.0 * s + 1.0),
         0.5 * r * (r - 1.0) * (-2.0 * s),
         (1.0 - r * r) * (-2.0 * s)]
    return np.stack(d, axis=-1)


def basis_P(r, s):
    """basis_functions.py:115-120."""
    r = np.asarray(r, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    return np.stack([0.25 * (1 - r) * (1 - s), 0.25 * (1 + r) * (1 - s),
                     0.25 * (1 + r) * (1 + s), 0.25 * (1 - r) * (1 + s)], axis=-1)


def basis_P_dr(r, s):
    """basis_functions.py:124-129."""
    r = np.asarray(r, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    return np.stack([-0.25 * (1 - s), 0.25 * (1 - s), 0.25 * (1 + s), -0.25 * (1 + s)], axis=-1)


def basis_P_dt(r, s):
    """basis_functions.py:133-138."""
    r = np.asarray(r, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    return np.stack([-0.25 * (1 - r), -0.25 * (1 + r), 0.25 * (1 + r), 0.25 * (1 - r)], axis=-1)


class BoxMesh:
    """Uniform nelx x nelz Q2xQ1 box, numbered exactly as the reference."""

    def __init__(self, nelx, nelz, Lx=1.0, Lz=1.0):
        self.nelx, self.nelz, self.Lx, self.Lz = int(nelx), int(nelz), float(Lx), float(Lz)
        nelx, nelz = self.nelx, self.nelz
        self.nel = nelx * nelz
        self.hx = Lx / nelx                      # build_velocity_mesh.py:19
        self.hz = Lz / nelz
        self.nnx, self.nnz = 2 * nelx + 1, 2 * nelz + 1
        self.nn_V = self.nnx * self.nnz
        self.nn_P = (nelx + 1) * (nelz + 1)
        self.Nfem_V, self.Nfem_P = 2 * self.nn_V, self.nn_P
        self.volume = Lx * Lz
        self.L_ref = (Lx + Lz) / 2               # meeuuw.py:341
        j, i = np.meshgrid(np.arange(self.nnz), np.arange(self.nnx), indexing="ij")
        i, j = i.ravel(), j.ravel()
        self.x_V = i * self.hx / 2               # build_velocity_mesh.py:116
        self.z_V = j * self.hz / 2
        self.left_Vnodes, self.right_Vnodes = i == 0, i == 2 * nelx
        self.bot_Vnodes, self.top_Vnodes = j == 0, j == 2 * nelz
        self.cornerBL = 0
        self.cornerBR = self.nnx - 1
        self.cornerTL = self.nnx * (self.nnz - 1)
        self.cornerTR = self.nn_V - 1
        ez, ex = np.meshgrid(np.arange(nelz), np.arange(nelx), indexing="ij")
        ex, ez = ex.ravel(), ez.ravel()
        nnx = self.nnx
        b = ex * 2 + ez * 2 * nnx                # build_velocity_connectivity.py:66-74
        self.icon_V = np.stack([b, b + 2, b + 2 + 2 * nnx, b + 2 * nnx, b + 1, b + 2 + nnx,
                                b + 1 + 2 * nnx, b + nnx, b + 1 + nnx]).astype(np.int32)
        self.left_element, self.right_element = ex == 0, ex == nelx - 1
        self.bot_element, self.top_element = ez == 0, ez == nelz - 1
        p = ex + ez * (nelx + 1)                 # build_pressure_connectivity.py
        self.icon_P = np.stack([p, p + 1, p + 1 + (nelx + 1), p + (nelx + 1)]).astype(np.int32)
        jp, ip = np.meshgrid(np.arange(nelz + 1), np.arange(nelx + 1), indexing="ij")
        self.x_P = ip.ravel() * self.hx
        self.z_P = jp.ravel() * self.hz
        # meeuuw.py:874-882
        l2g = np.empty((18, self.nel), dtype=np.int32)
        for k in range(9):
            for c in range(2):
                l2g[2 * k + c] = 2 * self.icon_V[k] + c
        self.local_to_globalV = l2g
        self.setup_q()
        self.setup_nodes()

    def setup_q(self):
        """basis_functions_setup_q.py:47-76 for straight-edged elements."""
        qc, qw = quadrature_setup(3)
        self.qcoords, self.qweights = qc, qw
        rq = np.array([qc[iq] for iq in range(3) for jq in range(3)])
        tq = np.array([qc[jq] for iq in range(3) for jq in range(3)])
        wq = np.array([qw[iq] * qw[jq] for iq in range(3) for jq in range(3)])
        self.rq, self.tq, self.weightq = rq, tq, wq
        self.N_V = basis_V(rq, tq)
        self.N_P = basis_P(rq, tq)
        self.N_T = self.N_V.copy()
        self.dNdr_V, self.dNdt_V = basis_V_dr(rq, tq), basis_V_dt(rq, tq)
        self.dNdr_P, self.dNdt_P = basis_P_dr(rq, tq), basis_P_dt(rq, tq)
        self.dNdr_T, self.dNdt_T = self.dNdr_V.copy(), self.dNdt_V.copy()
        xe = self.x_V[self.icon_V].T  # (nel,9)
        ze = self.z_V[self.icon_V].T
        J00 = xe @ self.dNdr_V.T      # (nel,9q)
        J01 = ze @ self.dNdr_V.T
        J10 = xe @ self.dNdt_V.T
        J11 = ze @ self.dNdt_V.T
        det = J00 * J11 - J01 * J10
        self.JxWq = det * wq[None, :]
        self.jcbi00q = J11 / det
        self.jcbi01q = -J01 / det
        self.jcbi10q = -J10 / det
        self.jcbi11q = J00 / det
        self.xq = xe @ self.N_V.T
        self.zq = ze @ self.N_V.T

    def setup_nodes(self):
        """basis_functions_setup_Vnodes.py (N_P_n, dN_V at V nodes, jcbi at V nodes)."""
        self.N_P_n = basis_P(R_V, T_V)
        self.dNdr_V_n, self.dNdt_V_n = basis_V_dr(R_V, T_V), basis_V_dt(R_V, T_V)
        xe = self.x_V[self.icon_V].T
        ze = self.z_V[self.icon_V].T
        J00 = xe @ self.dNdr_V_n.T
        J01 = ze @ self.dNdr_V_n.T
        J10 = xe @ self.dNdt_V_n.T
        J11 = ze @ self.dNdt_V_n.T
        det = J00 * J11 - J01 * J10
        self.jcbi00n, self.jcbi01n = J11 / det, -J01 / det
        self.jcbi10n, self.jcbi11n = -J10 / det, J00 / det

    # ---- COO index arrays, meeuuw.py:884-1017 ----
    def coo_stokes(self):
        l2g, iP = self.local_to_globalV, self.icon_P + self.Nfem_V
        rows = []
        cols = []
        for ikk in range(18):
            m1 = l2g[ikk]
            for jkk in range(18):
                rows.append(m1)
                cols.append(l2g[jkk])
            for jkk in range(4):
                rows += [m1, iP[jkk]]
                cols += [iP[jkk], m1]
        return np.stack(rows, 1).ravel(), np.stack(cols, 1).ravel()

    def coo_K(self):
        l2g = self.local_to_globalV
        II = np.repeat(l2g.T[:, :, None], 18, axis=2).ravel()
        JJ = np.repeat(l2g.T[:, None, :], 18, axis=1).ravel()
        return II, JJ

    def coo_G(self):
        l2g, iP = self.local_to_globalV, self.icon_P
        II_G = np.repeat(l2g.T[:, :, None], 4, axis=2).ravel()
        JJ_G = np.repeat(iP.T[:, None, :], 18, axis=1).ravel()
        II_GT = np.repeat(iP.T[:, :, None], 18, axis=2).ravel()
        JJ_GT = np.repeat(l2g.T[:, None, :], 4, axis=1).ravel()
        return II_G, JJ_G, II_GT, JJ_GT

    def coo_MP(self):
        iP = self.icon_P
        return (np.repeat(iP.T[:, :, None], 4, axis=2).ravel(),
                np.repeat(iP.T[:, None, :], 4, axis=1).ravel())

    def coo_T(self):
        ic = self.icon_V
        return (np.repeat(ic.T[:, :, None], 9, axis=2).ravel(),
                np.repeat(ic.T[:, None, :], 9, axis=1).ravel())
