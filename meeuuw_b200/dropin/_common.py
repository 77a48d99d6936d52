"""Argument handling shared by the drop-in functions.

The reference's functions take numpy arrays and return freshly allocated numpy arrays.  The
drop-ins accept numpy arrays or torch tensors: numpy (or CPU tensors) in -> numpy out, with the
host<->device copies done here; CUDA tensors in -> CUDA tensors out, no copies.  Every computation
runs in the library's CUDA kernels; a missing library or GPU raises, there is no host fallback.

Only the uniform box mesh of the reference (``build_velocity_mesh.py``, ``build_velocity_
connectivity.py``, x-fastest node numbering) is supported.  Its connectivity is recognised from
``icon_V`` once per array and checked in full against the arithmetic numbering the kernels use;
any other mesh raises ``NotImplementedError``.
"""
import numpy as np
import torch

from .. import _lib as L

f64, i32 = torch.float64, torch.int32


def is_device(a):
    return isinstance(a, torch.Tensor) and a.is_cuda


def host_mode(*arrays):
    """True when the caller works with host arrays (no CUDA tensor among `arrays`)."""
    return not any(is_device(a) for a in arrays)


def dev(a, dtype=None):
    """Contiguous CUDA tensor view/copy of a numpy array, list or tensor (None passes through)."""
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        t = a if a.is_cuda else a.cuda()
    else:
        arr = np.asarray(a)
        if arr.dtype == np.bool_:
            arr = arr.view(np.uint8)
        t = torch.from_numpy(np.ascontiguousarray(arr)).cuda()
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def dev_u8(a):
    """Boolean masks as uint8 on the device."""
    t = dev(a)
    if t.dtype == torch.bool:
        return t.view(torch.uint8)
    if t.dtype != torch.uint8:
        t = (t != 0).to(torch.uint8)
    return t


def back(t, host, dtype=None):
    """Result in the caller's world: numpy (synchronising copy) or the CUDA tensor itself."""
    if not host:
        return t
    a = t.cpu().numpy()
    return a.astype(dtype) if dtype is not None and a.dtype != dtype else a


def copy_into(dst, src):
    """Write a device result into the caller's array (in-place contracts)."""
    if isinstance(dst, torch.Tensor):
        if dst.data_ptr() != src.data_ptr():
            dst.copy_(src.view(dst.dtype) if dst.dtype == torch.bool and src.dtype == torch.uint8 else src)
    else:
        a = src.cpu().numpy()
        if dst.dtype == np.bool_:
            a = a.astype(np.bool_)
        dst[...] = a


def _arith_icon(nelx, nelz):
    nnx = 2 * nelx + 1
    ex = np.tile(np.arange(nelx), nelz)
    ez = np.repeat(np.arange(nelz), nelx)
    b = 2 * ex + 2 * ez * nnx
    return np.stack([b, b + 2, b + 2 + 2 * nnx, b + 2 * nnx, b + 1, b + 2 + nnx, b + 1 + 2 * nnx, b + nnx,
                     b + 1 + nnx]).astype(np.int64)


def _arith_icon_P(nelx, nelz):
    ex = np.tile(np.arange(nelx), nelz)
    ez = np.repeat(np.arange(nelz), nelx)
    b = ex + ez * (nelx + 1)
    return np.stack([b, b + 1, b + nelx + 2, b + nelx + 1]).astype(np.int64)


_checked = {}


def _key(a):
    if isinstance(a, torch.Tensor):
        return ("t", a.data_ptr(), tuple(a.shape))
    return ("n", a.__array_interface__["data"][0], a.shape)


def box_dims(icon_V, nel):
    """(nelx, nelz) of the uniform box mesh whose Q2 connectivity is icon_V (9, nel)."""
    key = _key(icon_V)
    hit = _checked.get(key)
    if hit is not None:
        return hit
    ic = icon_V.cpu().numpy() if isinstance(icon_V, torch.Tensor) else np.asarray(icon_V)
    if ic.ndim != 2 or ic.shape[0] != 9 or ic.shape[1] != nel or nel < 1:
        raise NotImplementedError("only the 9-node Q2 connectivity of a uniform box mesh is supported")
    nnx2 = int(ic[3, 0]) - int(ic[0, 0])
    if nnx2 <= 0 or nnx2 % 2:
        raise NotImplementedError("icon_V is not the box mesh's x-fastest Q2 numbering")
    nelx = (nnx2 // 2 - 1) // 2
    if nelx < 1 or nel % nelx:
        raise NotImplementedError("icon_V is not the box mesh's x-fastest Q2 numbering")
    nelz = nel // nelx
    if not np.array_equal(ic.astype(np.int64), _arith_icon(nelx, nelz)):
        raise NotImplementedError("icon_V is not the box mesh's x-fastest Q2 numbering")
    _checked[key] = (nelx, nelz)
    return nelx, nelz


def check_icon_P(icon_P, nelx, nelz):
    key = _key(icon_P)
    if key in _checked:
        return
    ic = icon_P.cpu().numpy() if isinstance(icon_P, torch.Tensor) else np.asarray(icon_P)
    if ic.shape != (4, nelx * nelz) or not np.array_equal(ic.astype(np.int64), _arith_icon_P(nelx, nelz)):
        raise NotImplementedError("icon_P is not the box mesh's Q1 numbering")
    _checked[key] = True


def box(nelx, nelz, hx=None, hz=None, Lx=None, Lz=None):
    """mw_box from the element counts and whichever of (h, L) the caller knows.  A caller's hx, hz
    are kept bit for bit (locate divides by them); unknown lengths default to 1 per element (the
    index-only kernels ignore them)."""
    if hx is None:
        hx = (Lx / nelx) if Lx is not None else 1.0
    if hz is None:
        hz = (Lz / nelz) if Lz is not None else 1.0
    Lx = hx * nelx if Lx is None else Lx
    Lz = hz * nelz if Lz is None else Lz
    return L.MwBox(int(nelx), int(nelz), float(Lx), float(Lz), float(hx), float(hz))


def check_coords(x_V, z_V, nelx, nelz, hx, hz):
    """The kernels place V node (ix, iz) at (ix*hx/2, iz*hz/2) as build_velocity_mesh.py:116-117
    does; other coordinates raise."""
    key = ("xz", _key(x_V), _key(z_V), hx, hz)
    if key in _checked:
        return
    xa = x_V.cpu().numpy() if isinstance(x_V, torch.Tensor) else np.asarray(x_V)
    za = z_V.cpu().numpy() if isinstance(z_V, torch.Tensor) else np.asarray(z_V)
    nnx, nnz = 2 * nelx + 1, 2 * nelz + 1
    ix = np.tile(np.arange(nnx), nnz)
    iz = np.repeat(np.arange(nnz), nnx)
    if xa.shape != (nnx * nnz,) or not (np.array_equal(xa, ix * hx / 2) and np.array_equal(za, iz * hz / 2)):
        raise NotImplementedError("x_V, z_V are not the uniform box lattice i*h/2")
    _checked[key] = True


def require_box(geometry="box", axisymmetric=False):
    if geometry != "box" or axisymmetric:
        raise NotImplementedError(f"the device path covers the plane-strain box geometry (got {geometry!r}, "
                                  f"axisymmetric={axisymmetric})")


def raise_flags(err, messages):
    """SystemExit with the reference's message for the first device flag that is set."""
    e = int(err.item())
    for flag, msg in messages:
        if e & flag:
            raise SystemExit(msg)
