"""GPU parity of the matrix-free Stokes operator and the device Uzawa / multigrid solvers.

* operator: equal to SpMV with the reference-assembled, Dirichlet-eliminated COO matrix
  (meeuuw.py:1798), FP64 relative 1e-12, FP32 relative 1e-5;
* K solve: relative residual below the requested tolerance;
* Stokes solve: FP64 relative true residual <= 1e-8; the velocity then
  agrees with SciPy's direct solve of the same system to 2e-5 (max norm) / 5e-6 (2-norm), the
  forward error a 1e-8 residual allows at these viscosity contrasts.
"""
import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


def make_case(nelx, nelz, Lx=1.0, contrast=1e3, bc="free_slip", eta_ref=1.0, seed=0):
    from oracle import assembly, solvers
    from oracle.fe import BoxMesh
    m = BoxMesh(nelx, nelz, Lx, 1.0)
    rng = np.random.default_rng(seed)
    T = (1 - m.zq) + 0.05 * np.cos(np.pi * m.xq / Lx) * np.sin(np.pi * m.zq) + 0.01 * rng.standard_normal(m.xq.shape)
    etaq = np.exp(-np.log(contrast) * T)
    eta_e = etaq.mean(axis=1)
    rhoq = 1 - 1e-2 * T
    fix = np.zeros(m.Nfem_V, dtype=bool)
    x, z = m.x_V, m.z_V
    fix[0::2] |= (x / Lx < 1e-8) | (x / Lx > 1 - 1e-8)
    fix[1::2] |= (z < 1e-8) | (z > 1 - 1e-8)
    if bc == "noslip_tb":
        fix[0::2] |= (z < 1e-8) | (z > 1 - 1e-8)
    val = np.zeros(m.Nfem_V)
    gx = np.zeros((m.nel, 9))
    gz = np.full((m.nel, 9), -1e6)
    res = assembly.build_matrix_stokes(0, 0, 0, 0, m.nel, 9, 9, 4, 2, m.Nfem_V, m.Nfem_P, 18, m.icon_V, m.icon_P,
                                       rhoq, etaq, m.JxWq, m.local_to_globalV, gx, gz, m.N_V, m.N_P, m.dNdr_V,
                                       m.dNdt_V, m.dNdr_P, m.dNdt_P, m.jcbi00q, m.jcbi01q, m.jcbi10q, m.jcbi11q,
                                       eta_e, eta_ref, m.L_ref, fix, val, m.bot_element, m.top_element, False, False,
                                       "box", None, False, m.xq, False)
    A = solvers.stokes_full(m, res[0])
    return dict(m=m, etaq=etaq, eta_e=eta_e, fix=fix, A=A, f=res[1], h=res[2], eta_ref=eta_ref)


def solver_for(c, **kw):
    from meeuuw_b200 import _lib
    from meeuuw_b200.stokes import StokesSolver
    m = c["m"]
    box = _lib.box_of(m.nelx, m.nelz, m.Lx, m.Lz)
    S = StokesSolver(box, torch.as_tensor(c["fix"]).cuda(), eta_ref=c["eta_ref"], L_ref=m.L_ref, **kw)
    S.set_viscosity(torch.as_tensor(c["etaq"]).cuda(), torch.as_tensor(c["eta_e"]).cuda())
    return S


@pytest.mark.parametrize("shape", [(6, 4), (16, 12), (32, 32)])
def test_apply_matches_assembled_coo(shape):
    c = make_case(*shape, Lx=1.3, eta_ref=2.0)
    S = solver_for(c)
    m = c["m"]
    rng = np.random.default_rng(1)
    u = rng.standard_normal(m.Nfem_V)
    p = rng.standard_normal(m.Nfem_P)
    yref = c["A"] @ np.concatenate([u, p])
    yV, yP = S.apply(torch.as_tensor(u).cuda(), torch.as_tensor(p).cuda())
    assert rel_err(yV.cpu().numpy(), yref[:m.Nfem_V]) < 1e-12
    assert rel_err(yP.cpu().numpy(), yref[m.Nfem_V:]) < 1e-12
    yV32, yP32 = S.apply(torch.as_tensor(u).float().cuda(), torch.as_tensor(p).float().cuda(), precision="f32")
    assert rel_err(yV32.double().cpu().numpy(), yref[:m.Nfem_V]) < 1e-5
    assert rel_err(yP32.double().cpu().numpy(), yref[m.Nfem_V:]) < 1e-5
    # the G and G^T blocks alone, as the Schur iterations apply them (node stencils)
    A = c["A"]
    G, GT = A[:m.Nfem_V, m.Nfem_V:], A[m.Nfem_V:, :m.Nfem_V]
    assert rel_err(S.grad(torch.as_tensor(p).cuda()).cpu().numpy(), G @ p) < 1e-12
    assert rel_err(S.div(torch.as_tensor(u).cuda()).cpu().numpy(), GT @ u) < 1e-12


@pytest.mark.parametrize("precision,tol,true_tol", [("f64", 1e-10, 3e-10), ("f32", 1e-4, 2e-3)])
def test_multigrid_pcg_K(precision, tol, true_tol):
    """FP32: the recursive residual drifts from the true one (FP32 rounding of K at 1e4 viscosity
    contrast); the mixed-precision Stokes path absorbs that with FP64 refinement."""
    c = make_case(64, 64, contrast=1e4)
    S = solver_for(c)
    m = c["m"]
    K = c["A"][:m.Nfem_V, :m.Nfem_V]
    b = torch.as_tensor(c["f"]).cuda()
    x, it, rr = S.solve_K(b, precision=precision, rtol=tol, maxit=300)
    xr = x.cpu().numpy()
    res = np.linalg.norm(c["f"] - K @ xr) / np.linalg.norm(c["f"])
    assert res < true_tol, (res, it)
    assert it < 100, it


@pytest.mark.parametrize("scheme", ["cd_u_eta", "uzawa3"])
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_stokes_solve_to_1e8(scheme, precision):
    import scipy.sparse.linalg as sla
    contrast = 1e3 if scheme == "cd_u_eta" else 1.0
    c = make_case(32, 32, contrast=contrast)
    S = solver_for(c)
    m = c["m"]
    f, h = torch.as_tensor(c["f"]).cuda(), torch.as_tensor(c["h"]).cuda()
    V, P, info = S.solve(f, h, scheme=scheme, precision=precision, tol=1e-8)
    assert info["converged"] == 1, info
    sol = np.concatenate([V.cpu().numpy(), P.cpu().numpy()])
    b = np.concatenate([c["f"], c["h"]])
    res = np.linalg.norm(b - c["A"] @ sol) / np.linalg.norm(b)
    assert res <= 1.05e-8, (res, info)
    ref = sla.spsolve(c["A"], b)
    # forward error a 1e-8 residual allows: the M-preconditioned uzawa3 iteration stops on the
    # residual with a larger error left in the velocity than cd_u_eta's M_eta-preconditioned one
    fwd = 2e-5 if scheme == "cd_u_eta" else 1e-4
    assert rel_err(sol[:m.Nfem_V], ref[:m.Nfem_V]) < fwd
    assert np.linalg.norm(sol[:m.Nfem_V] - ref[:m.Nfem_V]) < fwd / 2 * np.linalg.norm(ref[:m.Nfem_V])


def test_noslip_rayleigh_taylor_box_solve():
    c = make_case(32, 32, Lx=0.9142, contrast=100.0, bc="noslip_tb", eta_ref=100.0)
    S = solver_for(c)
    f, h = torch.as_tensor(c["f"]).cuda(), torch.as_tensor(c["h"]).cuda()
    V, P, info = S.solve(f, h, precision="mixed", tol=1e-8)
    assert info["converged"] == 1, info


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_device_loops_reproduce_host_loops(precision):
    """The solve recorded as one CUDA graph (loops as conditional nodes, decided on the device) runs
    the same kernels in the same order as the host-driven loops: same iterates, same counts.  Two
    solves in a row exercise the replay of the recorded graph."""
    c = make_case(32, 32, contrast=1e3)
    f, h = torch.as_tensor(c["f"]).cuda(), torch.as_tensor(c["h"]).cuda()
    out = {}
    for host in (1, 0):
        S = solver_for(c)
        runs = []
        for _ in range(2):
            V, P, info = S.solve(f, h, precision=precision, tol=1e-8, host_loops=host)
            runs.append((V.cpu().numpy(), P.cpu().numpy(), info))
        assert S.device_loops() == (host == 0)
        out[host] = runs
    for (Vh, Ph, ih), (Vd, Pd, idv) in zip(out[1], out[0]):
        assert idv["converged"] == 1 and ih["converged"] == 1, (ih, idv)
        for k in ("outer_iters", "inner_iters", "refinements"):
            assert idv[k] == ih[k], (k, ih, idv)
        assert abs(idv["rel_residual"] - ih["rel_residual"]) <= 1e-6 * ih["rel_residual"]
        assert rel_err(Vd, Vh) < 1e-12 and rel_err(Pd, Ph) < 1e-12


@pytest.mark.parametrize("tail_nel", [1024, 256])
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_coarse_tail_matches_level_launches(precision, tail_nel):
    """The coarse multigrid levels run as one launch per V-cycle (tail_nel: levels of at most 1024
    elements as an 8-CTA cluster through global memory; of at most 256 as one CTA with every
    vector in shared memory) repeat the multi-launch V-cycle bit for bit: same V-cycle output, same
    solve iterates and counts."""
    c = make_case(64, 64, contrast=1e4, seed=3)
    f, h = torch.as_tensor(c["f"]).cuda(), torch.as_tensor(c["h"]).cuda()
    hier = "f32" if precision == "mixed" else "f64"
    dt = torch.float32 if hier == "f32" else torch.float64
    g = torch.Generator(device="cuda").manual_seed(5)
    out = {}
    for tail in (tail_nel, 0):
        S = solver_for(c, tail_nel=tail)
        b = torch.randn(S.nv, dtype=dt, device="cuda", generator=g) if tail else b
        x = S.vcycle(b, precision=hier)
        V, P, info = S.solve(f, h, precision=precision, tol=1e-8)
        out[tail] = (x.cpu().numpy(), V.cpu().numpy(), P.cpu().numpy(), info)
    (x1, V1, P1, i1), (x0, V0, P0, i0) = out[tail_nel], out[0]
    assert np.array_equal(x1, x0)
    assert i1["converged"] == 1 and i0["converged"] == 1
    for k in ("outer_iters", "inner_iters", "refinements"):
        assert i1[k] == i0[k], (k, i1, i0)
    assert np.array_equal(V1, V0) and np.array_equal(P1, P0)


_FUSED_SCRIPT = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from meeuuw_b200 import _lib
from meeuuw_b200.stokes import StokesSolver
nel = 64
box = _lib.box_of(nel, nel, 1.0, 1.0)
nn1 = 2 * nel + 1
X, Z = np.meshgrid(np.arange(nn1), np.arange(nn1))
fix = np.zeros((nn1 * nn1, 2), dtype=bool)
fix[:, 0] = ((X == 0) | (X == nn1 - 1)).ravel()            # free slip: one component fixed on each side
fix[:, 1] = ((Z == 0) | (Z == nn1 - 1)).ravel()
rng = np.random.default_rng(4)
etaq = np.exp(np.repeat(rng.uniform(-4.0, 4.0, nel * nel), 9).reshape(nel * nel, 9))
S = StokesSolver(box, torch.as_tensor(fix.ravel()).cuda(), eta_ref=1.0, L_ref=1.0)
S.set_viscosity(torch.as_tensor(etaq).cuda(), torch.as_tensor(etaq[:, 0]).cuda())
g = torch.Generator(device="cuda").manual_seed(9)
out = {}
for prec, dt in (("f32", torch.float32), ("f64", torch.float64)):
    b = torch.randn(S.nv, dtype=dt, device="cuda", generator=g)
    out["v_" + prec] = S.vcycle(b, precision=prec).cpu().numpy()
    x, it, rr = S.solve_K(b.double(), precision=prec, rtol=1e-9 if prec == "f64" else 1e-4, maxit=300)
    out["x_" + prec] = x.cpu().numpy()
    out["it_" + prec] = np.array([it])
np.savez(sys.argv[2], **out)
"""


def test_fused_prolongation_matches_separate_launch(tmp_path):
    """The prolongation folded into the first post-smoothing step (MW_FUSED_PROLONG=1) and launched
    on its own (the default) give the same V-cycle and multigrid-PCG iterates bit for bit, on a mesh
    with free-slip sides (nodes with one fixed and one free component)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = {}
    for flag in ("1", "0"):
        path = str(tmp_path / f"fused{flag}.npz")
        env = dict(os.environ, MW_FUSED_PROLONG=flag)
        subprocess.run([sys.executable, "-c", _FUSED_SCRIPT, root, path], env=env, check=True, timeout=600)
        res[flag] = np.load(path)
    for k in res["1"].files:
        assert np.array_equal(res["1"][k], res["0"][k]), k
    assert res["1"]["it_f64"][0] < 100
