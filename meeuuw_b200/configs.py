"""Problem set-up for the box configurations (host side, run once per model).

The reference builds its mesh, boundary conditions, initial temperature and swarm
in pure-Python set-up loops (``build_velocity_mesh.py:113-145``,
``build_velocity_connectivity.py:63-92``, ``experiment0.py:91-95``,
``experiment0.py:112-175``, ``swarm_coordinates_setup.py:60-100``).  This module
produces the same arrays with numpy, once, before anything goes to the GPU; the
per-timestep work never comes back here.

The reference seeds nothing (``random.uniform`` in ``swarm_coordinates_setup.py:75``);
here every random draw comes from ``numpy.random.default_rng(seed)``.
"""
from dataclasses import dataclass, field, replace

import numpy as np


@dataclass(frozen=True)
class StepConfig:
    """One model's settings (the reference's experiment globals for the box path)."""
    name: str
    nelx: int
    nelz: int
    Lx: float = 1.0
    Lz: float = 1.0
    Ra: float = 1e4
    alphaT: float = 1e-2
    rho0: float = 1.0
    hcond: float = 1.0
    hcapa: float = 1.0
    hprod: float = 0.0
    eta_ref: float = 1.0
    fk_gamma: float = 0.0            # eta = exp(-fk_gamma * T)  (0 -> isoviscous)
    material: str = "boussinesq"     # or "two_material"
    mat_rho: tuple = (0.99, 1.0)     # two_material: below / above the interface
    mat_eta: tuple = (1.0, 100.0)
    gravity: tuple = None            # (gx, gz); None -> (0, -Ra/alphaT)
    bc_V: str = "free_slip"          # or "noslip_tb"  (no slip top/bottom, free slip sides)
    solve_T: bool = True
    Ttop: float = 0.0
    Tbottom: float = 1.0
    T_noise: float = 0.0
    particle_distribution: int = 1   # 0 random (seeded), 1 regular
    nparticle_per_dim: int = 4
    RKorder: int = 2
    averaging: str = "harmonic"
    nodal_projection_type: int = 2
    pressure_normalisation: str = "surface"
    CFLnb: float = 0.25
    dt_max: float = 1e30
    formulation: str = "BA"
    nstep: int = 20
    seed: int = 0
    # qpoint density / viscosity from the particles (meeuuw.py:1503-1562): "elemental" (element
    # means) or the least-squares fits "least_squares_P1" (with the slope limiter) / "least_squares_Q1"
    particle_rho_projection: str = "elemental"
    particle_eta_projection: str = "elemental"
    # population control after advection (pic_functions.py:1621-1812); 0 -> the reference's default
    # int(0.85 nparticle_per_dim^2) (set_default_parameters.py:112)
    allow_population_control: bool = False
    nparticle_min: int = 0

    @property
    def nmin(self):
        return self.nparticle_min if self.nparticle_min > 0 else int(self.nparticle_per_dim ** 2 * 0.85)

    @property
    def ls_order(self):
        """3 (P1) or 4 (Q1) when a least-squares projection is used, else 0 (meeuuw.py:1225-1297)."""
        p = (self.particle_rho_projection, self.particle_eta_projection)
        if "least_squares_P1" in p:
            return 3
        if "least_squares_Q1" in p:
            return 4
        return 0

    def population_seed(self, istep):
        """Key of the device generator that draws population control's reduced coordinates."""
        return (self.seed * 1000003 + istep) & 0xFFFFFFFFFFFFFFFF

    @property
    def nel(self):
        return self.nelx * self.nelz

    @property
    def nparticle(self):
        return self.nel * self.nparticle_per_dim ** 2

    @property
    def gxz(self):
        if self.gravity is not None:
            return self.gravity
        return (0.0, -self.Ra / self.alphaT)        # experiment0.py:270-272


def blankenbach(n=32, **kw):
    """Isoviscous Boussinesq convection, Ra=1e4, free slip, 4x4 regular particles, RK2."""
    return replace(StepConfig(name=f"blankenbach{n}", nelx=n, nelz=n), **kw)


def fk_convection(n=512, **kw):
    """Frank-Kamenetskii viscosity exp(-ln(1e5) T), Ra=1e6, 16 random particles/element, RK4."""
    base = StepConfig(name=f"fk{n}", nelx=n, nelz=n, Ra=1e6, fk_gamma=float(np.log(1e5)),
                      averaging="geometric", T_noise=1e-3, particle_distribution=0,
                      nparticle_per_dim=4, RKorder=4, nstep=10)
    return replace(base, **kw)


def rayleigh_taylor(n=256, **kw):
    """Two-material Rayleigh-Taylor, 0.9142 x 1 box, no slip top/bottom, 25 particles/element."""
    base = StepConfig(name=f"rt{n}", nelx=n, nelz=n, Lx=0.9142, Lz=1.0, material="two_material",
                      gravity=(0.0, -10.0), bc_V="noslip_tb", solve_T=False, eta_ref=100.0,
                      particle_distribution=0, nparticle_per_dim=5, RKorder=2,
                      pressure_normalisation="volume", nstep=200)
    return replace(base, **kw)


def q2_basis(r, s):
    """Q2 Lagrange basis in the reference's node order (basis_functions.py:20-30)."""
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


@dataclass
class HostModel:
    """Numpy arrays of one model, laid out as the reference lays them out."""
    cfg: StepConfig
    hx: float = 0.0
    hz: float = 0.0
    arrays: dict = field(default_factory=dict)

    def __getattr__(self, k):
        a = self.__dict__.get("arrays", {})
        if k in a:
            return a[k]
        raise AttributeError(k)


def build_host_model(cfg: StepConfig) -> HostModel:
    """Mesh, BCs, initial T and seeded swarm for one box model."""
    nelx, nelz, Lx, Lz = cfg.nelx, cfg.nelz, cfg.Lx, cfg.Lz
    hx, hz = Lx / nelx, Lz / nelz
    nnx, nnz = 2 * nelx + 1, 2 * nelz + 1
    nn_V = nnx * nnz
    j, i = np.meshgrid(np.arange(nnz), np.arange(nnx), indexing="ij")
    i, j = i.ravel(), j.ravel()
    x_V = i * hx / 2
    z_V = j * hz / 2
    ez, ex = np.meshgrid(np.arange(nelz), np.arange(nelx), indexing="ij")
    ex, ez = ex.ravel(), ez.ravel()
    b = ex * 2 + ez * 2 * nnx
    icon_V = np.stack([b, b + 2, b + 2 + 2 * nnx, b + 2 * nnx, b + 1, b + 2 + nnx,
                       b + 1 + 2 * nnx, b + nnx, b + 1 + nnx]).astype(np.int32)
    p = ex + ez * (nelx + 1)
    icon_P = np.stack([p, p + 1, p + 1 + (nelx + 1), p + (nelx + 1)]).astype(np.int32)
    eps = 1e-8
    bc_fix_V = np.zeros(2 * nn_V, dtype=bool)
    xl, xr = x_V / Lx < eps, x_V / Lx > 1 - eps
    zb, zt = z_V / Lz < eps, z_V / Lz > 1 - eps
    bc_fix_V[0::2] |= xl | xr                                    # experiment0.py:135-146
    bc_fix_V[1::2] |= zb | zt
    if cfg.bc_V == "noslip_tb":                                  # experiment1.py:61-77
        bc_fix_V[0::2] |= zb | zt
    bc_val_V = np.zeros(2 * nn_V)
    bc_fix_T = np.zeros(nn_V, dtype=bool)
    bc_val_T = np.zeros(nn_V)
    bc_fix_T[z_V < eps] = True                                   # experiment0.py:196-201
    bc_val_T[z_V < eps] = cfg.Tbottom
    bc_fix_T[z_V > Lz - eps] = True
    bc_val_T[z_V > Lz - eps] = cfg.Ttop
    rng = np.random.default_rng(cfg.seed)
    T = ((cfg.Tbottom - cfg.Ttop) * (Lz - z_V) / Lz + cfg.Ttop
         + 0.01 * np.cos(np.pi * x_V / Lx) * np.sin(np.pi * z_V / Lz))   # experiment0.py:91-95
    if cfg.T_noise > 0:
        T = T + rng.normal(0.0, cfg.T_noise, size=nn_V)
    if not cfg.solve_T:
        T = np.zeros(nn_V)
    else:
        T[bc_fix_T] = bc_val_T[bc_fix_T]                         # meeuuw.py:693-695
    npd = cfg.nparticle_per_dim
    ppe = npd * npd
    nel = nelx * nelz
    if cfg.particle_distribution == 1:                           # swarm_coordinates_setup.py:86-100
        jj, ii = np.meshgrid(np.arange(npd), np.arange(npd), indexing="ij")
        r1 = -1.0 + ii.ravel() * 2.0 / npd + 1.0 / npd
        t1 = -1.0 + jj.ravel() * 2.0 / npd + 1.0 / npd
        r = np.tile(r1, nel)
        t = np.tile(t1, nel)
    else:                                                        # swarm_coordinates_setup.py:72-83 (seeded)
        r = rng.uniform(-1.0, 1.0, size=nel * ppe)
        t = rng.uniform(-1.0, 1.0, size=nel * ppe)
    iel = np.repeat(np.arange(nel, dtype=np.int32), ppe)
    N = q2_basis(r, t)
    swarm_x = np.einsum("pk,pk->p", N, x_V[icon_V[:, iel].T])
    swarm_z = np.einsum("pk,pk->p", N, z_V[icon_V[:, iel].T])
    swarm_mat = np.zeros(nel * ppe, dtype=np.int8)
    if cfg.material == "two_material":                           # experiment1.py:25-36
        above = swarm_z >= 0.2 + 0.02 * np.cos(swarm_x * np.pi / 0.9142)
        swarm_mat[above] = 1
    m = HostModel(cfg=cfg, hx=hx, hz=hz)
    m.arrays.update(dict(x_V=x_V, z_V=z_V, icon_V=icon_V, icon_P=icon_P, bc_fix_V=bc_fix_V,
                         bc_val_V=bc_val_V, bc_fix_T=bc_fix_T, bc_val_T=bc_val_T, T=T,
                         swarm_x=swarm_x, swarm_z=swarm_z, swarm_r=r, swarm_t=t, swarm_iel=iel,
                         swarm_active=np.ones(nel * ppe, dtype=bool), swarm_mat=swarm_mat,
                         top_element=ez == nelz - 1, bot_element=ez == 0,
                         left_element=ex == 0, right_element=ex == nelx - 1))
    return m
