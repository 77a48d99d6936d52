"""The matrix-free energy operator (mw_energy_op_*) against the element-matrix path.

The element-matrix path (mw_assemble_energy + the summed-COO matvec) is pinned to the
reference's build_matrix_energy fixtures (test_gpu_parity.py); the matrix-free operator forms the
same A = M + (dt/2)(Ka + Kd) from Gauss-point coefficients, so both agree to rounding:
* right-hand side and A x: 1e-12 relative to the largest entry (FP64, another association);
* solutions of both solvers at rtol 1e-12: 1e-10;
* tiles: meshes that are and are not multiples of the 16 x 8 element tile, with Dirichlet
  nodes on two or four sides and random coefficient fields (BA and EBA).
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

f64 = torch.float64


def D(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def H(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("case", ["energy_BA", "energy_EBA"])
def test_energy_op_against_reference_fixture(case):
    from meeuuw_b200 import _lib, ops
    _lib.require_cuda()
    M = golden("mesh_6x4")
    g = golden(case)
    box = _lib.box_of(6, 4, 1.5, 1.0)
    # the box's Jacobian is diagonal (the reference's computed off-diagonal entries are rounding)
    assert max(np.abs(M["jcbi01q"]).max(), np.abs(M["jcbi10q"]).max()) < 1e-13 * np.abs(M["jcbi00q"]).max()
    q = {k: D(g[k]) for k in ("rhoq", "etaq", "Tq", "uq", "wq", "hcondq", "hcapaq", "alphaq", "hprodq", "exxq", "ezzq",
                              "exzq")}
    for k in ("JxWq", "jcbi00q", "jcbi01q", "jcbi10q", "jcbi11q"):
        q[k] = D(M[k])
    tables = {k: D(M[k]) for k in ("N_V", "dNdr_V", "dNdt_V")}
    args = (D(g["T"]), q, tables, D(g["bc_fix_T"]), D(g["bc_val_T"]), float(g["dt"]), float(g["rho0"]),
            str(g["formulation"]))
    op, rhs = ops.energy_op_setup(box, *args)
    assert rel_err(H(rhs), g["out_rhs"]) < 1e-12
    VV = D(g["out_VV_T"])
    x = torch.randn(rhs.numel(), dtype=f64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    assert rel_err(H(ops.energy_op_apply(box, op, x)), H(ops.energy_matvec(box, VV, x))) < 1e-12
    T0 = torch.zeros_like(rhs)
    T1 = torch.zeros_like(rhs)
    ops.energy_solve(box, VV, rhs, T0, rtol=1e-13, maxit=200)
    ops.energy_op_solve(box, op, rhs, T1, rtol=1e-13, maxit=200)
    assert rel_err(H(T1), H(T0)) < 1e-10


def _random_case(nelx, nelz, formulation, seed, sides):
    from meeuuw_b200 import _lib, fe_tables
    Lx, Lz = 1.3, 1.0
    box = _lib.box_of(nelx, nelz, Lx, Lz)
    nel = nelx * nelz
    nnx, nnz = 2 * nelx + 1, 2 * nelz + 1
    gen = torch.Generator("cuda").manual_seed(seed)
    R = lambda *s, lo=0.5, hi=1.5: lo + (hi - lo) * torch.rand(*s, dtype=f64, device="cuda", generator=gen)
    q = {k: R(nel, 9) for k in ("rhoq", "etaq", "Tq", "hcondq", "hcapaq", "alphaq", "hprodq")}
    for k in ("exxq", "ezzq", "exzq"):
        q[k] = R(nel, 9, lo=-300.0, hi=300.0)
    # velocities at a Courant number of at most 0.25 (dt = 2.5e-4), random per Gauss point
    umax = 0.25 * min(box.hx, box.hz) / 2.5e-4
    for k in ("uq", "wq"):
        q[k] = R(nel, 9, lo=-umax, hi=umax)
    q.update(fe_tables.uniform_geometry(nel, box.hx, box.hz))
    tables = fe_tables.device_tables()
    T = R(nnx * nnz, lo=0.0, hi=1.0)
    fix = torch.zeros(nnz, nnx, dtype=torch.bool, device="cuda")
    if "z" in sides:
        fix[0, :] = True
        fix[-1, :] = True
    if "x" in sides:
        fix[:, 0] = True
        fix[:, -1] = True
    val = torch.where(fix, R(nnz, nnx, lo=0.0, hi=1.0), torch.zeros(nnz, nnx, dtype=f64, device="cuda"))
    return box, (T, q, tables, fix.reshape(-1), val.reshape(-1), 2.5e-4, 1.0, formulation)


@pytest.mark.parametrize("nelx,nelz,sides", [(32, 16, "z"), (40, 17, "xz"), (7, 3, "xz"), (48, 24, "x")])
@pytest.mark.parametrize("formulation", ["BA", "EBA"])
def test_energy_op_tiles_random(nelx, nelz, sides, formulation):
    from meeuuw_b200 import ops
    box, args = _random_case(nelx, nelz, formulation, 11 + nelx + nelz, sides)
    VV, rhs0 = ops.assemble_energy(box, 0, *args)
    op, rhs1 = ops.energy_op_setup(box, *args)
    assert rel_err(H(rhs1), H(rhs0)) < 1e-12
    gen = torch.Generator("cuda").manual_seed(5)
    for _ in range(2):
        x = torch.randn(rhs0.numel(), dtype=f64, device="cuda", generator=gen)
        assert rel_err(H(ops.energy_op_apply(box, op, x)), H(ops.energy_matvec(box, VV, x))) < 1e-12
    T0 = args[0].clone()
    T1 = args[0].clone()
    i0, r0 = ops.energy_solve(box, VV, rhs0, T0, rtol=1e-12, maxit=300)
    i1, r1 = ops.energy_op_solve(box, op, rhs1, T1, rtol=1e-12, maxit=300)
    assert r0 <= 1e-12 and r1 <= 1e-12 and abs(i1 - i0) <= 2, (i0, r0, i1, r1)
    assert rel_err(H(T1), H(T0)) < 1e-10
    fixed = args[3]
    assert torch.allclose(T1[fixed], args[4][fixed], rtol=1e-12, atol=1e-14)    # Dirichlet values


def test_time_step_energy_forms_agree():
    """Three FK steps with the matrix-free operator and with the element matrices."""
    from meeuuw_b200 import configs
    from meeuuw_b200.timestep import GPUModel
    cfg = configs.fk_convection(48, seed=7)
    host = configs.build_host_model(cfg)
    out = {}
    for form in ("matrix_free", "matrices"):
        m = GPUModel(cfg, host, stokes="f64", tol=1e-10, energy=form)
        for _ in range(3):
            m.step()
        d = m.diagnostics()
        m.check()
        out[form] = (d["vrms"], d["Nu"], H(m.T))
    a, b = out["matrix_free"], out["matrices"]
    assert abs(a[0] / b[0] - 1) < 1e-8 and abs(a[1] / b[1] - 1) < 1e-8
    assert np.max(np.abs(a[2] - b[2])) < 1e-8
