// The reference's sparse-matrix index arrays and their summed CSR form, on the device (sm_100a).
//
// Reference: meeuuw.py:874-1017 builds, once, the COO row/column arrays II/JJ of the Stokes
// matrix (full layout), its K, G, G^T blocks, the Q1 pressure mass matrix and the Q2 temperature
// matrix in element order; meeuuw.py:1784-1800 and :2232 convert (VV, (II, JJ)) to CSR/CSC with
// SciPy every step, summing duplicates.  Here both come from the uniform box's arithmetic
// connectivity (q2_node / q1_node, the reference's node numbering):
//   * mw_coo_pattern writes II/JJ, one thread per entry, in the reference's order;
//   * mw_csr_pattern writes the summed matrix's row pointers and sorted column indices -- the
//     columns of a row are the dofs of a contiguous lattice block (the closure of the row node's
//     incident elements), so each row's length and column list are arithmetic;
//   * mw_csr_values sums the VV entries of every (row, column) over the elements that hold both,
//     in ascending element order (the order the entries appear in VV), one thread per nonzero.
#include <algorithm>

#include "common.cuh"

namespace mw {

enum CooKind { CK_STOKES = 0, CK_K = 1, CK_G = 2, CK_GT = 3, CK_MP = 4, CK_T = 5 };
// dof spaces: velocity (2 dofs per Q2 node), temperature (1 per Q2 node), pressure (1 per Q1 node)
enum Space { SP_V = 0, SP_T = 1, SP_P = 2 };

MW_HD int per_element(int kind) {
  return kind == CK_STOKES ? 468 : kind == CK_K ? 324 : (kind == CK_G || kind == CK_GT) ? 72 : kind == CK_MP ? 16 : 81;
}

// global dof of element-local index a in space sp (velocity: a = 2 k + component)
MW_D int64_t local_dof(const mw_box& b, int sp, int ex, int ez, int a) {
  const int nnx = 2 * b.nelx + 1;
  if (sp == SP_V) return 2 * q2_node(ex, ez, a >> 1, nnx) + (a & 1);
  if (sp == SP_T) return q2_node(ex, ez, a, nnx);
  return q1_node(ex, ez, a, b.nelx);
}

// ---------------------------------------------------------------- COO (II, JJ)
__global__ void k_coo_pattern(mw_box b, int kind, int32_t* __restrict__ II, int32_t* __restrict__ JJ) {
  const int per = per_element(kind);
  const int64_t total = (int64_t)b.nelx * b.nelz * per;
  const int64_t nfemV = 2LL * (2 * b.nelx + 1) * (2 * b.nelz + 1);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i / per;
    const int l = (int)(i - e * per);
    const int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
    int64_t r = 0, c = 0;
    if (kind == CK_STOKES) {                    // per ikk: 18 (V, V), then 4 pairs (V, P), (P, V)
      const int ikk = l / 26, m = l % 26;
      const int64_t m1 = local_dof(b, SP_V, ex, ez, ikk);
      if (m < 18) { r = m1; c = local_dof(b, SP_V, ex, ez, m); }
      else {
        const int j = (m - 18) >> 1;
        const int64_t m2 = local_dof(b, SP_P, ex, ez, j) + nfemV;
        if (((m - 18) & 1) == 0) { r = m1; c = m2; } else { r = m2; c = m1; }
      }
    } else if (kind == CK_K) {
      r = local_dof(b, SP_V, ex, ez, l / 18); c = local_dof(b, SP_V, ex, ez, l % 18);
    } else if (kind == CK_G) {
      r = local_dof(b, SP_V, ex, ez, l / 4); c = local_dof(b, SP_P, ex, ez, l % 4);
    } else if (kind == CK_GT) {
      r = local_dof(b, SP_P, ex, ez, l / 18); c = local_dof(b, SP_V, ex, ez, l % 18);
    } else if (kind == CK_MP) {
      r = local_dof(b, SP_P, ex, ez, l / 4); c = local_dof(b, SP_P, ex, ez, l % 4);
    } else {
      r = local_dof(b, SP_T, ex, ez, l / 9); c = local_dof(b, SP_T, ex, ez, l % 9);
    }
    II[i] = (int32_t)r;
    JJ[i] = (int32_t)c;
  }
}

// ---------------------------------------------------------------- CSR of the summed matrix
// A row: its space, node (lattice or Q1 coordinates), dof component; its incident elements form
// the range [ex0, ex1] x [ez0, ez1].
struct RowInfo {
  int sp, ix, iz, comp;
  int ex0, ex1, ez0, ez1;
};

MW_HD int row_space(int kind, int64_t r, int64_t nfemV) {
  if (kind == CK_STOKES) return r < nfemV ? SP_V : SP_P;
  if (kind == CK_K || kind == CK_G) return SP_V;
  if (kind == CK_GT || kind == CK_MP) return SP_P;
  return SP_T;
}

MW_D RowInfo row_info(const mw_box& b, int kind, int64_t r) {
  const int nnx = 2 * b.nelx + 1;
  const int64_t nfemV = 2LL * nnx * (2 * b.nelz + 1);
  RowInfo R;
  R.sp = row_space(kind, r, nfemV);
  if (R.sp == SP_P) {
    const int64_t n = kind == CK_STOKES ? r - nfemV : r;
    R.ix = (int)(n % (b.nelx + 1)); R.iz = (int)(n / (b.nelx + 1)); R.comp = 0;
    R.ex0 = max(R.ix - 1, 0); R.ex1 = min(R.ix, b.nelx - 1);
    R.ez0 = max(R.iz - 1, 0); R.ez1 = min(R.iz, b.nelz - 1);
  } else {
    const int64_t n = R.sp == SP_V ? r >> 1 : r;
    R.comp = R.sp == SP_V ? (int)(r & 1) : 0;
    R.ix = (int)(n % nnx); R.iz = (int)(n / nnx);
    R.ex0 = (R.ix & 1) ? (R.ix >> 1) : max((R.ix >> 1) - 1, 0);
    R.ex1 = (R.ix & 1) ? (R.ix >> 1) : min(R.ix >> 1, b.nelx - 1);
    R.ez0 = (R.iz & 1) ? (R.iz >> 1) : max((R.iz >> 1) - 1, 0);
    R.ez1 = (R.iz & 1) ? (R.iz >> 1) : min(R.iz >> 1, b.nelz - 1);
  }
  return R;
}

// The column blocks of a row, in ascending column order: up to two (a velocity / temperature block
// of Q2 lattice nodes, then a pressure block of Q1 nodes for the Stokes matrix's velocity rows).
struct ColBlock {
  int sp;             // column space
  int x0, z0, nx, nz; // node block
  int64_t base;       // column offset of the space (Nfem_V for the Stokes matrix's pressure columns)
};

MW_D int col_blocks(const mw_box& b, int kind, const RowInfo& R, ColBlock* cb) {
  const int64_t nfemV = 2LL * (2 * b.nelx + 1) * (2 * b.nelz + 1);
  auto q2blk = [&](int sp) {
    ColBlock c;
    c.sp = sp; c.x0 = 2 * R.ex0; c.z0 = 2 * R.ez0; c.nx = 2 * (R.ex1 - R.ex0) + 3; c.nz = 2 * (R.ez1 - R.ez0) + 3;
    c.base = 0;
    return c;
  };
  auto q1blk = [&](int64_t base) {
    ColBlock c;
    c.sp = SP_P; c.x0 = R.ex0; c.z0 = R.ez0; c.nx = R.ex1 - R.ex0 + 2; c.nz = R.ez1 - R.ez0 + 2;
    c.base = base;
    return c;
  };
  if (kind == CK_STOKES) {
    if (R.sp == SP_V) { cb[0] = q2blk(SP_V); cb[1] = q1blk(nfemV); return 2; }
    cb[0] = q2blk(SP_V); return 1;
  }
  if (kind == CK_K || kind == CK_GT) { cb[0] = q2blk(SP_V); return 1; }
  if (kind == CK_G || kind == CK_MP) { cb[0] = q1blk(0); return 1; }
  cb[0] = q2blk(SP_T); return 1;
}

MW_D int dofs_per_node(int sp) { return sp == SP_V ? 2 : 1; }

__global__ void k_csr_rowlen(mw_box b, int kind, int64_t rows, int64_t* __restrict__ len) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const RowInfo R = row_info(b, kind, r);
    ColBlock cb[2];
    const int nb = col_blocks(b, kind, R, cb);
    int64_t n = 0;
    for (int k = 0; k < nb; ++k) n += (int64_t)cb[k].nx * cb[k].nz * dofs_per_node(cb[k].sp);
    len[r] = n;
  }
}

// Exclusive scan of n int64 values in place into out[0..n] (out[n] = total): a block-level pass
// that writes per-block totals, a single-block pass over the totals, and an add pass.
constexpr int SCAN_B = 1024;
__global__ void k_scan64_block(const int64_t* __restrict__ in, int64_t* __restrict__ out, int64_t* __restrict__ bsum,
                               int64_t n) {
  __shared__ int64_t sh[SCAN_B];
  const int64_t i = (int64_t)blockIdx.x * SCAN_B + threadIdx.x;
  sh[threadIdx.x] = i < n ? in[i] : 0;
  __syncthreads();
  for (int o = 1; o < SCAN_B; o <<= 1) {           // Hillis-Steele inclusive scan
    const int64_t v = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  if (i < n) out[i + 1] = sh[threadIdx.x];
  if (threadIdx.x == SCAN_B - 1) bsum[blockIdx.x] = sh[SCAN_B - 1];
}

__global__ void k_scan64_sums(int64_t* __restrict__ bsum, int nb) {   // one thread: exclusive prefix of the totals
  if (threadIdx.x || blockIdx.x) return;
  int64_t s = 0;
  for (int k = 0; k < nb; ++k) { const int64_t v = bsum[k]; bsum[k] = s; s += v; }
}

__global__ void k_scan64_add(int64_t* __restrict__ out, const int64_t* __restrict__ bsum, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * SCAN_B + threadIdx.x;
  if (i < n) out[i + 1] += bsum[blockIdx.x];
  if (i == 0) out[0] = 0;
}

__global__ void k_csr_cols(mw_box b, int kind, int64_t rows, const int64_t* __restrict__ row_ptr,
                           int32_t* __restrict__ col) {
  const int nnx = 2 * b.nelx + 1;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const RowInfo R = row_info(b, kind, r);
    ColBlock cb[2];
    const int nb = col_blocks(b, kind, R, cb);
    int64_t p = row_ptr[r];
    for (int k = 0; k < nb; ++k) {
      const ColBlock& c = cb[k];
      const int dn = dofs_per_node(c.sp);
      for (int z = 0; z < c.nz; ++z)
        for (int x = 0; x < c.nx; ++x) {
          const int64_t node = c.sp == SP_P ? (int64_t)(c.z0 + z) * (b.nelx + 1) + c.x0 + x
                                            : (int64_t)(c.z0 + z) * nnx + c.x0 + x;
          for (int d = 0; d < dn; ++d) col[p++] = (int32_t)(c.base + node * dn + d);
        }
    }
  }
}

// element-local index of a node of space sp in element (ex, ez), or -1 when the node is not in it
MW_D int local_node(const mw_box& b, int sp, int ex, int ez, int ix, int iz) {
  if (sp == SP_P) {
    const int dx = ix - ex, dz = iz - ez;
    if (dx < 0 || dx > 1 || dz < 0 || dz > 1) return -1;
    return dz == 0 ? dx : 3 - dx;                       // (0,0) 0, (1,0) 1, (1,1) 2, (0,1) 3
  }
  const int dx = ix - 2 * ex, dz = iz - 2 * ez;
  if (dx < 0 || dx > 2 || dz < 0 || dz > 2) return -1;
  if (dz == 0) return dx == 0 ? 0 : (dx == 1 ? 4 : 1);
  if (dz == 1) return dx == 0 ? 7 : (dx == 1 ? 8 : 5);
  return dx == 0 ? 3 : (dx == 1 ? 6 : 2);
}

// position of the entry (local row a, local column c) in an element's block of VV, or -1
MW_D int vv_pos(int kind, int rsp, int csp, int a, int c) {
  switch (kind) {
    case CK_STOKES:
      if (rsp == SP_V && csp == SP_V) return a * 26 + c;
      if (rsp == SP_V) return a * 26 + 18 + 2 * c;          // (V a, P c)
      if (csp == SP_V) return c * 26 + 18 + 2 * a + 1;      // (P a, V c)
      return -1;                                            // no (P, P) entries
    case CK_K: return a * 18 + c;
    case CK_G: return a * 4 + c;
    case CK_GT: return a * 18 + c;
    case CK_MP: return a * 4 + c;
    default: return a * 9 + c;
  }
}

__global__ void k_csr_values(mw_box b, int kind, int64_t rows, const double* __restrict__ vv,
                             const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                             double* __restrict__ val) {
  const int nnx = 2 * b.nelx + 1;
  const int64_t nfemV = 2LL * nnx * (2 * b.nelz + 1);
  const int per = per_element(kind);
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const RowInfo R = row_info(b, kind, r);
    for (int64_t p = row_ptr[r]; p < row_ptr[r + 1]; ++p) {
      const int64_t cg = col[p];
      // the column's space, node and component
      int csp, cx, cz, cc;
      if (kind == CK_STOKES && cg >= nfemV) {
        csp = SP_P; const int64_t n = cg - nfemV; cx = (int)(n % (b.nelx + 1)); cz = (int)(n / (b.nelx + 1)); cc = 0;
      } else if (kind == CK_G || kind == CK_MP) {
        csp = SP_P; cx = (int)(cg % (b.nelx + 1)); cz = (int)(cg / (b.nelx + 1)); cc = 0;
      } else if (kind == CK_T) {
        csp = SP_T; cx = (int)(cg % nnx); cz = (int)(cg / nnx); cc = 0;
      } else {
        csp = SP_V; const int64_t n = cg >> 1; cx = (int)(n % nnx); cz = (int)(n / nnx); cc = (int)(cg & 1);
      }
      double acc = 0.0;
      for (int ez = R.ez0; ez <= R.ez1; ++ez)             // ascending element order
        for (int ex = R.ex0; ex <= R.ex1; ++ex) {
          const int ar = local_node(b, R.sp, ex, ez, R.ix, R.iz);
          const int ac = local_node(b, csp, ex, ez, cx, cz);
          if (ar < 0 || ac < 0) continue;
          const int a = R.sp == SP_V ? 2 * ar + R.comp : ar, c = csp == SP_V ? 2 * ac + cc : ac;
          const int pos = vv_pos(kind, R.sp, csp, a, c);
          if (pos >= 0) acc += vv[((int64_t)ez * b.nelx + ex) * per + pos];
        }
      val[p] = acc;
    }
  }
}

static int64_t csr_rows(mw_box b, int kind) {
  const int64_t nV = 2LL * (2 * b.nelx + 1) * (2 * b.nelz + 1), nP = (int64_t)(b.nelx + 1) * (b.nelz + 1);
  const int64_t nT = (int64_t)(2 * b.nelx + 1) * (2 * b.nelz + 1);
  switch (kind) {
    case CK_STOKES: return nV + nP;
    case CK_K: case CK_G: return nV;
    case CK_GT: case CK_MP: return nP;
    default: return nT;
  }
}

}  // namespace mw

using namespace mw;

extern "C" {

int64_t mw_coo_length(mw_box box, int32_t kind) {
  if (box.nelx <= 0 || box.nelz <= 0 || kind < 0 || kind > CK_T) return -1;
  return (int64_t)box.nelx * box.nelz * per_element(kind);
}

int mw_coo_pattern(mw_box box, int32_t kind, int32_t* II, int32_t* JJ, void* stream) {
  const int64_t n = mw_coo_length(box, kind);
  if (n < 0 || !II || !JJ) return MW_ERR_BAD_ARG;
  k_coo_pattern<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(box, kind, II, JJ);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int64_t mw_csr_rows(mw_box box, int32_t kind) {
  if (box.nelx <= 0 || box.nelz <= 0 || kind < 0 || kind > CK_T) return -1;
  return csr_rows(box, kind);
}

size_t mw_csr_workspace_bytes(mw_box box, int32_t kind) {
  const int64_t rows = csr_rows(box, kind);
  return (size_t)(rows + (rows + SCAN_B - 1) / SCAN_B + 1) * sizeof(int64_t);
}

int mw_csr_pattern(mw_box box, int32_t kind, int64_t* row_ptr, int64_t* nnz, void* work, size_t work_bytes,
                   void* stream) {
  const int64_t rows = mw_csr_rows(box, kind);
  if (rows < 0 || !row_ptr || !nnz) return MW_ERR_BAD_ARG;
  if (!work || work_bytes < mw_csr_workspace_bytes(box, kind)) return MW_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  int64_t* len = (int64_t*)work;
  int64_t* bsum = len + rows;
  const int nb = (int)((rows + SCAN_B - 1) / SCAN_B);
  k_csr_rowlen<<<grid_for(rows, 256), 256, 0, s>>>(box, kind, rows, len);
  k_scan64_block<<<nb, SCAN_B, 0, s>>>(len, row_ptr, bsum, rows);
  k_scan64_sums<<<1, 32, 0, s>>>(bsum, nb);
  k_scan64_add<<<nb, SCAN_B, 0, s>>>(row_ptr, bsum, rows);
  MW_CHECK_LAUNCH();
  if (cudaMemcpyAsync(nnz, row_ptr + rows, sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return MW_ERR_CUDA;
  return MW_OK;
}

int mw_csr_columns(mw_box box, int32_t kind, const int64_t* row_ptr, int32_t* col, void* stream) {
  const int64_t rows = mw_csr_rows(box, kind);
  if (rows < 0 || !row_ptr || !col) return MW_ERR_BAD_ARG;
  k_csr_cols<<<grid_for(rows, 256), 256, 0, (cudaStream_t)stream>>>(box, kind, rows, row_ptr, col);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_csr_values(mw_box box, int32_t kind, const double* VV, const int64_t* row_ptr, const int32_t* col, double* val,
                  void* stream) {
  const int64_t rows = mw_csr_rows(box, kind);
  if (rows < 0 || !VV || !row_ptr || !col || !val) return MW_ERR_BAD_ARG;
  k_csr_values<<<grid_for(rows, 128), 128, 0, (cudaStream_t)stream>>>(box, kind, rows, VV, row_ptr, col, val);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

}  // extern "C"
