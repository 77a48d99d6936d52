"""Tensor-level wrappers over the C ABI (device tensors in, device tensors out).

Each function launches the CUDA kernels of ``libmeeuuw_b200.so`` on the current torch stream.
Outputs are allocated here when not supplied; the hot loop (``meeuuw_b200.timestep``) passes
preallocated buffers so that nothing is allocated per step.
"""
import ctypes
import threading

import torch

from . import _lib as L
from ._lib import call, ptr, stream_ptr

f64, i32, u8 = torch.float64, torch.int32, torch.uint8


class Workspace:
    """Grow-only device scratch owned by the caller (the library never allocates)."""

    def __init__(self, device="cuda"):
        self.device = device
        self.buf = torch.empty(0, dtype=torch.uint8, device=device)

    def get(self, nbytes):
        nbytes = int(nbytes)
        if self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=self.device)
        return ctypes.c_void_p(self.buf.data_ptr()), ctypes.c_size_t(self.buf.numel())


_ws = {}
_scope = threading.local()


class workspace_scope:
    """Within this context, workspace(tag) returns the scratch of `owner` (a model): the same
    buffers whichever stream the kernels go to, so a time step recorded into a CUDA graph on a
    capture stream uses the buffers of the model's eager steps."""

    def __init__(self, owner):
        self.key = id(owner)

    def __enter__(self):
        self.prev = getattr(_scope, "key", None)
        _scope.key = self.key
        return self

    def __exit__(self, *exc):
        _scope.key = self.prev


def workspace(tag="default"):
    """Scratch for `tag`: the current model's (inside workspace_scope) or the current stream's, so
    that models advanced concurrently on different streams never share scratch and reuse is
    ordered by one stream."""
    owner = getattr(_scope, "key", None)
    if owner is not None:
        key = (tag, "model", owner)
    else:
        key = (tag, torch.cuda.current_stream().cuda_stream if torch.cuda.is_available() else 0)
    if key not in _ws:
        _ws[key] = Workspace()
    return _ws[key]


def _empty(n, dtype=f64, like=None):
    dev = like.device if like is not None else "cuda"
    return torch.empty(n, dtype=dtype, device=dev)


def as_u8(active):
    if active.dtype == torch.bool:
        return active.view(torch.uint8)
    if active.dtype != torch.uint8:
        raise TypeError("active must be bool or uint8")
    return active


# ----------------------------------------------------------------------------- PIC
def locate(box, active, x, z, r=None, t=None, iel=None, err=None):
    n = x.numel()
    r = _empty(n, like=x) if r is None else r
    t = _empty(n, like=x) if t is None else t
    iel = _empty(n, i32, like=x) if iel is None else iel
    call("mw_locate_box", box, n, ptr(as_u8(active)), ptr(x), ptr(z), ptr(r), ptr(t), ptr(iel), ptr(err), stream_ptr())
    return r, t, iel


def interp(box, active, r, t, iel, fields, outs=None):
    n = r.numel()
    if outs is None:
        outs = [_empty(n, like=r) for _ in fields]
    for i in range(0, len(fields), L.MAX_FIELDS):
        fs, os_ = fields[i:i + L.MAX_FIELDS], outs[i:i + L.MAX_FIELDS]
        call("mw_interp_q2", box, n, ptr(as_u8(active)), ptr(r), ptr(t), ptr(iel), len(fs), L.ptr_array(fs),
             L.ptr_array(os_), stream_ptr())
    return outs


def material_struct(cfg):
    m = L.MwMaterial()
    if cfg.material == "two_material":
        m.kind = L.MATERIAL_TWO
        for i, v in enumerate(cfg.mat_rho):
            m.mat_rho[i] = v
        for i, v in enumerate(cfg.mat_eta):
            m.mat_eta[i] = v
    else:
        m.kind = L.MATERIAL_BOUSSINESQ
    m.rho0, m.alphaT, m.fk_gamma, m.eta0 = cfg.rho0, cfg.alphaT, cfg.fk_gamma, 1.0
    m.hcond, m.hcapa, m.hprod = cfg.hcond, cfg.hcapa, cfg.hprod
    return m


def interp_material(box, active, r, t, iel, mat, nodal, material, out):
    """nodal: dict exx, ezz, exz, q, T (tensors or None); out: dict of per-particle tensors."""
    nd = L.MwNodal5(*[ptr(nodal.get(k)) for k in ("exx", "ezz", "exz", "q", "T")])
    op = L.MwSwarmProps(*[ptr(out.get(k)) for k in ("exx", "ezz", "exz", "p", "T", "rho", "eta", "hcond", "hcapa",
                                                     "hprod", "alpha")])
    call("mw_interp_material", box, r.numel(), ptr(as_u8(active)), ptr(r), ptr(t), ptr(iel), ptr(mat), nd, material,
         op, stream_ptr())
    return out


def advect(box, rk, dt, x, z, active, u, w, up=None, wp=None, err=None, dt_dev=None):
    call("mw_advect_box", box, int(rk), float(dt), ptr(dt_dev), x.numel(), ptr(x), ptr(z), ptr(as_u8(active)),
         ptr(u), ptr(w), ptr(up), ptr(wp), ptr(err), stream_ptr())
    return x, z, up, wp, active


def bin_particles(nel, active, iel, counts=None, offsets=None, order=None, err=None):
    n = iel.numel()
    counts = _empty(nel, i32, like=iel) if counts is None else counts
    offsets = _empty(nel + 1, i32, like=iel) if offsets is None else offsets
    order = _empty(max(n, 1), i32, like=iel) if order is None else order
    wp, wb = workspace("bin").get(L.lib().mw_bin_workspace_bytes(nel))
    call("mw_bin_particles", nel, n, ptr(as_u8(active)), ptr(iel), ptr(counts), ptr(offsets), ptr(order), wp, wb,
         ptr(err), stream_ptr())
    return counts, offsets, order


def project_elements(nel, offsets, order, rho, eta, averaging, rho_e=None, eta_e=None, err=None):
    rho_e = _empty(nel, like=rho) if rho_e is None else rho_e
    eta_e = _empty(nel, like=rho) if eta_e is None else eta_e
    call("mw_project_elements", nel, ptr(offsets), ptr(order), ptr(rho), ptr(eta), L.AVG[averaging], ptr(rho_e),
         ptr(eta_e), ptr(err), stream_ptr())
    return rho_e, eta_e


def project_nodes(box, flavour, fields, offsets, order, r, t, outs=None, exact_order=False):
    """fields: list of (phi, averaging) -> list of nodal arrays (nn_V).  exact_order=True sums in
    the reference's particle-index order (per-node merge, slower)."""
    nn = (2 * box.nelx + 1) * (2 * box.nelz + 1)
    if outs is None:
        outs = [_empty(nn, like=r) for _ in fields]
    for i in range(0, len(fields), L.MAX_FIELDS):
        fs, os_ = fields[i:i + L.MAX_FIELDS], outs[i:i + L.MAX_FIELDS]
        avg = (ctypes.c_int32 * len(fs))(*[L.AVG[a] for _, a in fs])
        if exact_order:
            wp, wb = None, ctypes.c_size_t(0)
        else:
            wp, wb = workspace("proj").get(L.lib().mw_project_nodes_workspace_bytes(box, len(fs)))
        call("mw_project_nodes", box, int(flavour), len(fs), avg, ptr(offsets), ptr(order), ptr(r), ptr(t),
             L.ptr_array([p for p, _ in fs]), L.ptr_array(os_), wp, wb, stream_ptr())
    return outs


def nodal_to_qpoints(box, space, N, phi, out=None):
    nel = box.nelx * box.nelz
    out = _empty((nel, 9), like=phi) if out is None else out
    call("mw_nodal_to_qpoints", box, int(space), ptr(N), ptr(phi), ptr(out), stream_ptr())
    return out


# ----------------------------------------------------------------------------- assembly
def assemble_stokes(box, blocks, precision, q, tables, bc_fix_V, bc_val_V, eta_ref, L_ref, out=None):
    """q: dict rhoq, etaq, JxWq, jcbi**q, gxq, gzq (nel,9) and eta_e (nel)."""
    nel = box.nelx * box.nelz
    nv = 2 * (2 * box.nelx + 1) * (2 * box.nelz + 1)
    npp = (box.nelx + 1) * (box.nelz + 1)
    dt = torch.float32 if precision == 1 else f64
    dev = q["etaq"].device
    if out is None:
        if blocks:
            out = dict(VV_K=torch.empty(nel * 324, dtype=dt, device=dev), VV_G=torch.empty(nel * 72, dtype=dt, device=dev),
                       VV_GT=torch.empty(nel * 72, dtype=dt, device=dev), VV_M=torch.empty(nel * 16, dtype=dt, device=dev),
                       VV_M_eta=torch.empty(nel * 16, dtype=dt, device=dev), VV_H=torch.empty(nel * 72, dtype=dt, device=dev))
        else:
            out = dict(VV_Stokes=torch.empty(nel * 468, dtype=dt, device=dev))
        out["rhs_f"] = torch.empty(nv, dtype=f64, device=dev)
        out["rhs_h"] = torch.empty(npp, dtype=f64, device=dev)
    ins = L.MwStokesIn(*[ptr(q[k]) for k in ("rhoq", "etaq", "JxWq", "jcbi00q", "jcbi01q", "jcbi10q", "jcbi11q", "gxq",
                                             "gzq", "eta_e")],
                       *[ptr(tables[k]) for k in ("N_V", "N_P", "dNdr_V", "dNdt_V", "dNdr_P", "dNdt_P")],
                       ptr(as_u8(bc_fix_V)), ptr(bc_val_V), float(eta_ref), float(L_ref))
    outs = L.MwStokesOut(*[ptr(out.get(k)) for k in ("VV_Stokes", "VV_K", "VV_G", "VV_GT", "VV_M", "VV_M_eta", "VV_H",
                                                     "rhs_f", "rhs_h")])
    wp, wb = workspace("asm").get(L.lib().mw_assemble_stokes_workspace_bytes(box))
    call("mw_assemble_stokes", box, int(bool(blocks)), int(precision), ins, outs, wp, wb, stream_ptr())
    return out


def _energy_in(T, q, tables, bc_fix_T, bc_val_T, dt, rho0, formulation, dt_dev):
    keys = ("rhoq", "etaq", "Tq", "uq", "wq", "hcondq", "hcapaq", "alphaq", "hprodq", "exxq", "ezzq", "exzq", "JxWq",
            "jcbi00q", "jcbi01q", "jcbi10q", "jcbi11q")
    return L.MwEnergyIn(ptr(T), *[ptr(q.get(k)) for k in keys], ptr(tables["N_V"]), ptr(tables["dNdr_V"]),
                        ptr(tables["dNdt_V"]), ptr(as_u8(bc_fix_T)), ptr(bc_val_T), float(dt), float(rho0),
                        ptr(dt_dev), 1 if formulation == "EBA" else 0)


def assemble_energy(box, precision, T, q, tables, bc_fix_T, bc_val_T, dt, rho0, formulation, VV=None, rhs=None,
                    dt_dev=None):
    nel = box.nelx * box.nelz
    nn = (2 * box.nelx + 1) * (2 * box.nelz + 1)
    dty = torch.float32 if precision == 1 else f64
    VV = torch.empty(nel * 81, dtype=dty, device=T.device) if VV is None else VV
    rhs = torch.empty(nn, dtype=f64, device=T.device) if rhs is None else rhs
    ins = _energy_in(T, q, tables, bc_fix_T, bc_val_T, dt, rho0, formulation, dt_dev)
    wp, wb = workspace("asm").get(L.lib().mw_assemble_energy_workspace_bytes(box))
    call("mw_assemble_energy", box, int(precision), ins, ptr(VV), ptr(rhs), wp, wb, stream_ptr())
    return VV, rhs


# ----------------------------------------------------------------------------- sparse patterns
COO_KINDS = {"stokes": 0, "K": 1, "G": 2, "GT": 3, "MP": 4, "T": 5}


def coo_pattern(box, kind, device="cuda"):
    """The reference's (II, JJ) of matrix `kind` (meeuuw.py:874-1017), int32 device tensors."""
    k = COO_KINDS[kind]
    n = L.lib().mw_coo_length(box, k)
    II = torch.empty(n, dtype=torch.int32, device=device)
    JJ = torch.empty(n, dtype=torch.int32, device=device)
    call("mw_coo_pattern", box, k, ptr(II), ptr(JJ), stream_ptr())
    return II, JJ


class CsrPattern:
    """Row pointers and sorted column indices of the summed matrix `kind`, built once on the
    device; values(VV) sums an assembled VV of the same kind into them (coo_matrix((VV, (II, JJ)))
    .tocsr() of meeuuw.py:1784-1800, without leaving the device)."""

    def __init__(self, box, kind, device="cuda"):
        self.box, self.kind = box, COO_KINDS[kind]
        self.rows = L.lib().mw_csr_rows(box, self.kind)
        self.row_ptr = torch.empty(self.rows + 1, dtype=torch.int64, device=device)
        nnz = ctypes.c_int64()
        wp, wb = workspace("csr").get(L.lib().mw_csr_workspace_bytes(box, self.kind))
        call("mw_csr_pattern", box, self.kind, ptr(self.row_ptr), ctypes.byref(nnz), wp, wb, stream_ptr())
        self.nnz = nnz.value
        self.col = torch.empty(self.nnz, dtype=torch.int32, device=device)
        call("mw_csr_columns", box, self.kind, ptr(self.row_ptr), ptr(self.col), stream_ptr())

    def values(self, VV, out=None):
        out = torch.empty(self.nnz, dtype=f64, device=VV.device) if out is None else out
        call("mw_csr_values", self.box, self.kind, ptr(VV), ptr(self.row_ptr), ptr(self.col), ptr(out), stream_ptr())
        return out

    def tensor(self, VV, ncols):
        """torch.sparse_csr_tensor of the summed matrix (ncols columns)."""
        return torch.sparse_csr_tensor(self.row_ptr, self.col.to(torch.int64), self.values(VV),
                                       size=(self.rows, ncols), check_invariants=False)


def energy_op_setup(box, T, q, tables, bc_fix_T, bc_val_T, dt, rho0, formulation, op=None, rhs=None, dt_dev=None):
    """Matrix-free energy operator (Gauss-point coefficients, diagonal, Dirichlet flags) and the
    right-hand side of build_matrix_energy.  Returns (op, rhs); op is a uint8 device buffer."""
    nn = (2 * box.nelx + 1) * (2 * box.nelz + 1)
    nb = L.lib().mw_energy_op_bytes(box)
    op = torch.empty(nb, dtype=torch.uint8, device=T.device) if op is None else op
    rhs = torch.empty(nn, dtype=f64, device=T.device) if rhs is None else rhs
    ins = _energy_in(T, q, tables, bc_fix_T, bc_val_T, dt, rho0, formulation, dt_dev)
    call("mw_energy_op_setup", box, ins, ptr(op), op.numel(), ptr(rhs), stream_ptr())
    return op, rhs


def energy_op_apply(box, op, x, y=None):
    y = torch.empty_like(x) if y is None else y
    call("mw_energy_op_apply", box, ptr(op), ptr(x), ptr(y), stream_ptr())
    return y


# ----------------------------------------------------------------------------- post
PNORM = {"none": 0, "surface": 1, "volume": 2}


def pressure_offset(box, normalisation, p, N_P, JxWq, volume, out=None):
    out = torch.empty(1, dtype=f64, device=p.device) if out is None else out
    wp, wb = workspace("post").get(L.lib().mw_post_workspace_bytes())
    call("mw_pressure_offset", box, PNORM[normalisation], ptr(p), ptr(N_P), ptr(JxWq), float(volume), ptr(out), wp, wb,
         stream_ptr())
    return out


def nodal_pressure(box, p, offset, N_P_n, q=None, subtract=True):
    nn = (2 * box.nelx + 1) * (2 * box.nelz + 1)
    q = torch.empty(nn, dtype=f64, device=p.device) if q is None else q
    call("mw_nodal_pressure", box, ptr(p), ptr(offset), int(bool(subtract)), ptr(N_P_n), ptr(q), stream_ptr())
    return q


def nodal_strain_rate(box, u, w, tables, jcbi=None, out=None):
    nn = u.numel()
    out = [torch.empty(nn, dtype=f64, device=u.device) for _ in range(3)] if out is None else out
    j = jcbi if jcbi is not None else (None, None, None, None)
    call("mw_nodal_strain_rate", box, ptr(u), ptr(w), ptr(tables["dNdr_V_n"]), ptr(tables["dNdt_V_n"]),
         *[ptr(a) for a in j], *[ptr(o) for o in out], stream_ptr())
    return out


def nodal_heat_flux(box, T, hcond_n, tables, jcbi=None, out=None):
    nn = T.numel()
    out = [torch.empty(nn, dtype=f64, device=T.device) for _ in range(4)] if out is None else out
    j = jcbi if jcbi is not None else (None, None, None, None)
    call("mw_nodal_heat_flux", box, ptr(T), ptr(hcond_n), ptr(tables["dNdr_V_n"]), ptr(tables["dNdt_V_n"]),
         *[ptr(a) for a in j], *[ptr(o) for o in out], stream_ptr())
    return out


def gauss_struct():
    from .fe_tables import gauss3
    qc, qw = gauss3()
    g = L.MwGauss3()
    for i in range(3):
        g.c[i], g.w[i] = qc[i], qw[i]
    return g


def compute_nu(box, T, dTdx, dTdz, hcond_n, out=None):
    out = torch.empty(13, dtype=f64, device=T.device) if out is None else out
    wp, wb = workspace("nu").get(L.lib().mw_nu_workspace_bytes(box))
    call("mw_compute_nu", box, ptr(T), ptr(dTdx), ptr(dTdz), ptr(hcond_n), gauss_struct(), ptr(out), wp, wb,
         stream_ptr())
    return out


def global_quantities(uq, wq, Tq, rhoq, JxWq, volume, out=None):
    out = torch.empty(3, dtype=f64, device=uq.device) if out is None else out
    wp, wb = workspace("post").get(L.lib().mw_post_workspace_bytes())
    call("mw_global_quantities", uq.numel(), ptr(uq), ptr(wq), ptr(Tq), ptr(rhoq), ptr(JxWq), float(volume), ptr(out),
         wp, wb, stream_ptr())
    return out


def stokes_rhs_body(box, rhoq, gxq, gzq, JxWq, N_V, bc_fix_V, rhs_f, rhs_h):
    """Stokes right-hand side for all-zero Dirichlet values (body force only)."""
    wp, wb = workspace("asm").get(L.lib().mw_assemble_stokes_workspace_bytes(box))
    call("mw_stokes_rhs_body", box, ptr(rhoq), ptr(gxq), ptr(gzq), ptr(JxWq), ptr(N_V), ptr(as_u8(bc_fix_V)),
         ptr(rhs_f), ptr(rhs_h), wp, wb, stream_ptr())
    return rhs_f, rhs_h


def split_solution(solV, solP, scale, u, w, p):
    call("mw_split_solution", u.numel(), p.numel(), ptr(solV), ptr(solP), float(scale), ptr(u), ptr(w), ptr(p),
         stream_ptr())
    return u, w, p


def elemental_to_qpoints(a, b, aq, bq):
    call("mw_elemental_to_qpoints", a.numel(), ptr(a), ptr(b), ptr(aq), ptr(bq), stream_ptr())


def energy_matvec(box, VV, x, y=None):
    y = torch.empty_like(x) if y is None else y
    call("mw_energy_matvec", box, ptr(VV), ptr(x), ptr(y), stream_ptr())
    return y


def energy_solve(box, VV, rhs, T, rtol=1e-12, maxit=200):
    """Solves in place into T (T holds the initial guess).  Returns (iterations, relres)."""
    it = ctypes.c_int32()
    rr = ctypes.c_double()
    wp, wb = workspace("energy").get(L.lib().mw_energy_solve_workspace_bytes(box))
    rc = L.lib().mw_energy_solve(box, ptr(VV), ptr(rhs), ptr(T), float(rtol), int(maxit), ctypes.byref(it),
                                 ctypes.byref(rr), wp, wb, stream_ptr())
    if rc not in (0, 3):
        raise RuntimeError(f"mw_energy_solve returned {L.STATUS.get(rc, rc)}")
    return it.value, rr.value


def energy_op_solve(box, op, rhs, T, rtol=1e-12, maxit=200):
    """energy_solve on the matrix-free operator of energy_op_setup."""
    it = ctypes.c_int32()
    rr = ctypes.c_double()
    wp, wb = workspace("energy_op").get(L.lib().mw_energy_op_solve_workspace_bytes(box))
    rc = L.lib().mw_energy_op_solve(box, ptr(op), ptr(rhs), ptr(T), float(rtol), int(maxit), ctypes.byref(it),
                                    ctypes.byref(rr), wp, wb, stream_ptr())
    if rc not in (0, 3):
        raise RuntimeError(f"mw_energy_op_solve returned {L.STATUS.get(rc, rc)}")
    return it.value, rr.value


def energy_device_info(box, op=False):
    """(iterations, relative residual) of the last energy solve on this stream (op: of the
    matrix-free one), from the device."""
    it = ctypes.c_int32()
    rr = ctypes.c_double()
    if op:
        wp, wb = workspace("energy_op").get(L.lib().mw_energy_op_solve_workspace_bytes(box))
    else:
        wp, wb = workspace("energy").get(L.lib().mw_energy_solve_workspace_bytes(box))
    call("mw_energy_device_info", box, wp, ctypes.byref(it), ctypes.byref(rr), stream_ptr())
    return it.value, rr.value


def compute_dt(u, w, hcond, hcapa, rho, CFLnb, hx, hz, dt_max, solve_T, state, out=None):
    out = torch.empty(3, dtype=f64, device=u.device) if out is None else out
    prm = L.MwDtParams(float(CFLnb), float(hx), float(hz), float(dt_max), int(bool(solve_T)))
    wp, wb = workspace("post").get(L.lib().mw_post_workspace_bytes())
    n = rho.numel()
    call("mw_compute_dt", u.numel(), ptr(u), ptr(w), n, ptr(hcond), ptr(hcapa), ptr(rho), prm, ptr(state), ptr(out),
         wp, wb, stream_ptr())
    return out


# ----------------------------------------------------------------------------- tensor-core GEMM
class MwGemmEpilogue(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("relu", ctypes.c_int32), ("splits", ctypes.c_int32),
                ("bias", ctypes.c_void_p), ("out", ctypes.c_void_p), ("ldo", ctypes.c_int64)]


L.extra_protos({
    "mw_gemm_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "mw_gemm_bf16_tn": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                         ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, MwGemmEpilogue,
                                         ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]),
})

EPI_F32, EPI_BF16 = 0, 1


L.extra_protos({
    "mw_conv3x3_bf16": (ctypes.c_int32, [ctypes.c_int32] * 4 + [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                                               ctypes.c_int64, MwGemmEpilogue, ctypes.c_void_p,
                                                               ctypes.c_void_p]),
})


def conv3x3_ok(C, H, W):
    """Whether mw_conv3x3_bf16 takes this shape (else im2col + gemm_bf16_tn)."""
    return C % 32 == 0 and W <= 128 and 128 % W == 0 and (H * W) % 128 == 0


def conv3x3_bf16(X, B, H, W, C, Wt, out=None, bias=None, relu=False, out_bf16=False, err=None):
    """3x3 'same' convolution of NHWC BF16 X [B*H*W, C] with Wt [N, Kp] (K = tap*C + c) as an
    implicit GEMM on the tensor cores: out [B*H*W, N]."""
    N = Wt.shape[0]
    M = B * H * W
    if out is None:
        out = torch.empty(M, N, dtype=torch.bfloat16 if out_bf16 else torch.float32, device=X.device)
    ep = MwGemmEpilogue(EPI_BF16 if out_bf16 else EPI_F32, int(bool(relu)), 1, ptr(bias), ptr(out), out.stride(0))
    call("mw_conv3x3_bf16", B, H, W, C, ptr(X), N, ptr(Wt), Wt.stride(0), ep, ptr(err), stream_ptr())
    return out


def gemm_bf16_tn(A, B, out=None, bias=None, relu=False, splits=1, out_bf16=False, err=None):
    """out[M, N] = A[M, K] @ B[N, K]^T on the tensor cores (A, B bf16, K % 64 == 0)."""
    M, K = A.shape
    N = B.shape[0]
    if out is None:
        out = torch.empty(M, N, dtype=torch.bfloat16 if out_bf16 else torch.float32, device=A.device)
    ep = MwGemmEpilogue(EPI_BF16 if out_bf16 else EPI_F32, int(bool(relu)), int(splits), ptr(bias), ptr(out),
                        out.stride(0))
    if splits > 1:
        wp, wb = workspace("gemm").get(L.lib().mw_gemm_workspace_bytes(M, N, splits))
    else:
        wp, wb = None, ctypes.c_size_t(0)
    call("mw_gemm_bf16_tn", M, N, K, ptr(A), A.stride(0), ptr(B), B.stride(0), ep, wp, wb, ptr(err), stream_ptr())
    return out


# ---------------------------------------------------------------- least squares, population control
def ls_fit(box, ncoef, offsets, order, x, z, fields, limit_h=0.0, err=None):
    """compute_ls_coefficients_P1 (ncoef 3) / _Q1 (ncoef 4) for the particle fields `fields`, with
    the driver's slope limiter when limit_h > 0 (P1).  offsets/order: bins of every particle.
    Returns [(coef (nel, ncoef), fmin (nel), fmax (nel)) per field]."""
    nel = box.nelx * box.nelz
    outs = [(_empty(nel * ncoef, like=x).view(nel, ncoef), _empty(nel, like=x), _empty(nel, like=x))
            for _ in fields]
    for i in range(0, len(fields), L.MAX_FIELDS):
        fs = L.MwLsFields()
        chunk = list(range(i, min(len(fields), i + L.MAX_FIELDS)))
        for k, j in enumerate(chunk):
            fs.phi[k] = fields[j].data_ptr()
            fs.coef[k] = outs[j][0].data_ptr()
            fs.fmin[k] = outs[j][1].data_ptr()
            fs.fmax[k] = outs[j][2].data_ptr()
        fs.n = len(chunk)
        call("mw_ls_fit", box, int(ncoef), ptr(offsets), ptr(order), ptr(x), ptr(z), fs, float(limit_h), ptr(err),
             stream_ptr())
    return outs


def ls_to_qpoints(box, coef, xq, zq, out=None):
    """meeuuw.py:1517-1532: the fit evaluated at the quadrature points, (nel, 9)."""
    out = torch.empty_like(xq) if out is None else out
    call("mw_ls_to_qpoints", box, int(coef.shape[1]), ptr(coef), ptr(xq), ptr(zq), ptr(out), stream_ptr())
    return out


def population_control(box, nparticle_min, counts, offsets, order, active, iel, r, t, x, z, mat=None, avg=(),
                       source=None, draws=None, seed=0, added=None, err=None):
    """population_control (pic_functions.py:1621-1812).  avg: per-particle fields the new particles
    take as their element's mean.  Returns the device scalar holding the number of particles added."""
    n = x.numel()
    nel = box.nelx * box.nelz
    added = torch.zeros(1, dtype=i32, device=x.device) if added is None else added
    pf = L.MwPcFields()
    for k, f in enumerate(avg):
        pf.f[k] = f.data_ptr()
    pf.n = len(avg)
    wp, wb = workspace("population").get(L.lib().mw_population_workspace_bytes(nel, n))
    max_new = draws.numel() // 2 if draws is not None else n
    call("mw_population_control", box, int(nparticle_min), n, ptr(counts), ptr(offsets), ptr(order),
         ptr(as_u8(active)), ptr(iel), ptr(r), ptr(t), ptr(x), ptr(z), ptr(mat), ptr(source), pf, ptr(draws),
         int(max_new), ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), ptr(added), wp, wb, ptr(err), stream_ptr())
    return added
