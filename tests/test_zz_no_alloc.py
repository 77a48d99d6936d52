"""The allocation-free Nusselt entry point (mw_compute_nu_noalloc) against mw_compute_nu.

mw_compute_nu_noalloc serves callers that hold the solution on the device but cannot allocate
device memory (a monitoring hook given read-only device pointers by the host code); its scratch
is a fixed device array inside the library.  This file is collected last so that a run stopping
at the first failure has already run every other test; it also passes on its own in a fresh
process.  Tolerance: the same 1e-12 relative as the other FP64 reductions (both entry points run
the same kernels, so the values are in fact identical).
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _inputs(nelx, nelz, seed):
    rng = np.random.default_rng(seed)
    nn = (2 * nelx + 1) * (2 * nelz + 1)
    return [torch.as_tensor(rng.uniform(lo, hi, nn)).cuda()
            for lo, hi in ((0.0, 1.0), (-2.0, 2.0), (-2.0, 2.0), (0.5, 1.5))]


def _noalloc(lib, box, T, dTdx, dTdz, hc, g, out=None):
    from meeuuw_b200 import _lib
    fn = lib.mw_compute_nu_noalloc
    fn.restype = ctypes.c_int32
    fn.argtypes = [_lib.MwBox] + [ctypes.c_void_p] * 4 + [_lib.MwGauss3, ctypes.c_void_p, ctypes.c_void_p]
    if out is None:
        out = torch.full((13,), float("nan"), dtype=torch.float64, device="cuda")
    rc = fn(box, T.data_ptr(), dTdx.data_ptr(), dTdz.data_ptr(), hc.data_ptr(), g, out.data_ptr(),
            torch.cuda.current_stream().cuda_stream)
    return rc, out


def test_nu_noalloc_matches_workspace_entry_point_twice():
    from meeuuw_b200 import _lib, ops
    _lib.require_cuda()
    lib = _lib.lib()
    box = _lib.box_of(48, 32, 1.5, 1.0)
    g = ops.gauss_struct()
    for seed in (0, 1):                       # two calls in a row, different data
        T, dTdx, dTdz, hc = _inputs(48, 32, seed)
        ref = ops.compute_nu(box, T, dTdx, dTdz, hc).cpu().numpy()
        rc, out = _noalloc(lib, box, T, dTdx, dTdz, hc, g)
        assert rc == _lib.MW_OK
        out = out.cpu().numpy()
        assert np.all(np.isfinite(out))
        assert np.max(np.abs(out - ref) / np.maximum(np.abs(ref), 1e-300)) < 1e-12


def test_nu_noalloc_rejects_meshes_beyond_its_capacity():
    from meeuuw_b200 import _lib, ops
    _lib.require_cuda()
    box = _lib.box_of(16384, 4, 1.0, 1.0)     # 2*(nelx+nelz) > 32768 boundary elements
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc, _ = _noalloc(_lib.lib(), box, dummy, dummy, dummy, dummy, ops.gauss_struct())
    assert rc == 6                            # MW_ERR_TOO_LARGE, before any launch


def test_nu_noalloc_leaves_device_memory_unchanged():
    """After the set-up call, further calls leave the device's free memory exactly as it was."""
    from meeuuw_b200 import _lib, ops
    _lib.require_cuda()
    lib = _lib.lib()
    box = _lib.box_of(40, 24, 1.0, 1.0)
    g = ops.gauss_struct()
    T, dTdx, dTdz, hc = _inputs(40, 24, 2)
    ref = ops.compute_nu(box, T, dTdx, dTdz, hc).cpu().numpy()
    outs = [torch.full((13,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(5)]
    rc, _ = _noalloc(lib, box, T, dTdx, dTdz, hc, g, outs[0])          # set-up call
    assert rc == _lib.MW_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()                                # cudaMemGetInfo
    for o in outs:
        rc, _ = _noalloc(lib, box, T, dTdx, dTdz, hc, g, o)
        assert rc == _lib.MW_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    for o in outs:
        assert np.max(np.abs(o.cpu().numpy() - ref) / np.maximum(np.abs(ref), 1e-300)) < 1e-12


def test_nu_noalloc_at_exactly_its_capacity():
    """A mesh with exactly MW_NU_NOALLOC_MAX_BOUNDARY_ELEMENTS boundary elements is accepted."""
    from meeuuw_b200 import _lib, ops
    _lib.require_cuda()
    nelx, nelz = 16380, 4                     # 2*(nelx+nelz) = 32768
    box = _lib.box_of(nelx, nelz, 4.0, 1.0)
    T, dTdx, dTdz, hc = _inputs(nelx, nelz, 3)
    ref = ops.compute_nu(box, T, dTdx, dTdz, hc).cpu().numpy()
    rc, out = _noalloc(_lib.lib(), box, T, dTdx, dTdz, hc, ops.gauss_struct())
    assert rc == _lib.MW_OK
    out = out.cpu().numpy()
    assert np.max(np.abs(out - ref) / np.maximum(np.abs(ref), 1e-300)) < 1e-12
