"""The reference's sparse index arrays and summed CSR matrices, built on the device.

* II/JJ of every matrix kind equal the oracle's (``oracle/fe.py``, pinned to the driver's own loops
  of meeuuw.py:874-1017 by ``test_oracle_golden.py``) bit for bit, on the reference fixtures' 6x4
  mesh and on a 16x12 box;
* the CSR pattern (row pointers, sorted columns) equals SciPy's coo_matrix((VV, (II, JJ))).tocsr()
  with its duplicates summed; the values agree to 1e-14 relative to the largest entry -- with VV
  the reference's own assembled arrays (``tests/golden``).
"""
import numpy as np
import pytest
import scipy.sparse as sps
import torch

from conftest import golden

pytestmark = pytest.mark.gpu

KINDS = ("stokes", "K", "G", "GT", "MP", "T")


def _mesh(nelx, nelz, Lx):
    from oracle.fe import BoxMesh
    return BoxMesh(nelx, nelz, Lx, 1.0)


def _oracle_coo(m, kind):
    if kind == "stokes":
        return m.coo_stokes()
    if kind == "K":
        return m.coo_K()
    if kind in ("G", "GT"):
        IG, JG, IGT, JGT = m.coo_G()
        return (IG, JG) if kind == "G" else (IGT, JGT)
    if kind == "MP":
        return m.coo_MP()
    return m.coo_T()


def _shape(m, kind):
    nV, nP, nT = m.Nfem_V, m.Nfem_P, m.Nfem_V // 2
    return {"stokes": (nV + nP, nV + nP), "K": (nV, nV), "G": (nV, nP), "GT": (nP, nV), "MP": (nP, nP),
            "T": (nT, nT)}[kind]


@pytest.mark.parametrize("shape", [(6, 4, 1.5), (16, 12, 1.3)])
@pytest.mark.parametrize("kind", KINDS)
def test_coo_and_csr_patterns(shape, kind):
    from meeuuw_b200 import _lib, ops
    nelx, nelz, Lx = shape
    m = _mesh(nelx, nelz, Lx)
    box = _lib.box_of(nelx, nelz, Lx, 1.0)
    II, JJ = ops.coo_pattern(box, kind)
    I0, J0 = _oracle_coo(m, kind)
    assert np.array_equal(II.cpu().numpy(), I0) and np.array_equal(JJ.cpu().numpy(), J0)
    csr = ops.CsrPattern(box, kind)
    ref = sps.coo_matrix((np.ones(len(I0)), (I0, J0)), shape=_shape(m, kind)).tocsr()
    ref.sum_duplicates()
    ref.sort_indices()
    assert csr.rows == ref.shape[0] and csr.nnz == ref.nnz
    assert np.array_equal(csr.row_ptr.cpu().numpy(), ref.indptr)
    assert np.array_equal(csr.col.cpu().numpy(), ref.indices)
    # values: random VV, summed duplicates against SciPy's
    rng = np.random.default_rng(len(I0))
    vv = rng.standard_normal(len(I0))
    got = csr.values(torch.as_tensor(vv).cuda()).cpu().numpy()
    refv = sps.coo_matrix((vv, (I0, J0)), shape=_shape(m, kind)).tocsr()
    refv.sum_duplicates()
    refv.sort_indices()
    assert np.max(np.abs(got - refv.data)) <= 1e-14 * np.max(np.abs(refv.data))


@pytest.mark.parametrize("case,key,kind", [("stokes_full_bc", "out_VV_Stokes", "stokes"),
                                           ("stokes_blocks", "out_VV_K", "K"), ("stokes_blocks", "out_VV_G", "G"),
                                           ("stokes_blocks", "out_VV_GT", "GT"), ("stokes_blocks", "out_VV_M", "MP"),
                                           ("energy_BA", "out_VV_T", "T")])
def test_csr_of_reference_assembly(case, key, kind):
    """The summed matrices of the reference's own VV arrays (6x4 mesh, Dirichlet rows eliminated)."""
    from meeuuw_b200 import _lib, ops
    g = golden(case)
    vv = np.asarray(g[key], dtype=np.float64)
    if vv.size == 0:
        pytest.skip("fixture without this block")
    m = _mesh(6, 4, 1.5)
    box = _lib.box_of(6, 4, 1.5, 1.0)
    I0, J0 = _oracle_coo(m, kind)
    assert len(vv) == len(I0)
    csr = ops.CsrPattern(box, kind)
    A = csr.tensor(torch.as_tensor(vv).cuda(), _shape(m, kind)[1])
    ref = sps.coo_matrix((vv, (I0, J0)), shape=_shape(m, kind)).tocsr()
    ref.sum_duplicates()
    ref.sort_indices()
    assert np.array_equal(A.crow_indices().cpu().numpy(), ref.indptr)
    assert np.max(np.abs(A.values().cpu().numpy() - ref.data)) <= 1e-14 * np.max(np.abs(ref.data))
    x = np.random.default_rng(0).standard_normal(ref.shape[1])
    y = (A @ torch.as_tensor(x).cuda().unsqueeze(1)).squeeze(1).cpu().numpy()
    assert np.max(np.abs(y - ref @ x)) <= 1e-13 * np.max(np.abs(ref @ x))
