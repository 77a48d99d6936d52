// Device solve of the Crank-Nicolson energy system (sm_100a).
//
// Reference: meeuuw.py:2232-2235 converts (II_T, JJ_T, VV_T) to CSR (summing duplicates) and calls
// SuperLU's spsolve.  Here the element matrices VV_T written by build_matrix_energy
// (build_matrix_energy.py:133-137, nel*81 values) are used directly: y = A x is a node-centric
// gather over the (up to 4) incident elements in ascending element order -- the summed COO
// matrix applied without forming it -- and the system is solved by Jacobi-preconditioned
// BiCGSTAB in FP64 to a relative residual tolerance.  The solve first regroups the rows by node
// class (k_energy_rows) so that every matvec of the iteration reads them coalesced.
//
// The time stepper uses the matrix-free form of the same operator instead (mw_energy_op_*): the
// Gauss-point coefficients of the element matrices stored once per step, the element products
// formed on the fly in shared-memory tiles, the right-hand side and the Jacobi diagonal formed by
// the same kernel -- no element matrices are written or read.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "q2_ref.cuh"
#include "tma.cuh"

namespace mw {

MW_D int q2_local_e(int dx, int dz) {
  if (dz == 0) return dx == 0 ? 0 : (dx == 1 ? 4 : 1);
  if (dz == 1) return dx == 0 ? 7 : (dx == 1 ? 8 : 5);
  return dx == 0 ? 3 : (dx == 1 ? 6 : 2);
}

// y = A x  (mode 0), or r = b - A x (mode 1).  Also writes diag when diag != null.
__global__ void k_energy_matvec(mw_box b, const double* __restrict__ vv, const double* __restrict__ x,
                                const double* __restrict__ rhs, double* __restrict__ y, double* __restrict__ diag,
                                int mode) {
  pdl_entry();
  const int nnx = 2 * b.nelx + 1;
  const int64_t nn = (int64_t)nnx * (2 * b.nelz + 1);
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    int ix = (int)(n % nnx), iz = (int)(n / nnx);
    int exs[2], ezs[2], nxe = 0, nze = 0;
    if (ix & 1) exs[nxe++] = ix >> 1;
    else { if (ix / 2 - 1 >= 0) exs[nxe++] = ix / 2 - 1; if (ix / 2 < b.nelx) exs[nxe++] = ix / 2; }
    if (iz & 1) ezs[nze++] = iz >> 1;
    else { if (iz / 2 - 1 >= 0) ezs[nze++] = iz / 2 - 1; if (iz / 2 < b.nelz) ezs[nze++] = iz / 2; }
    double acc = 0.0, dg = 0.0;
    for (int a = 0; a < nze; ++a)
      for (int c = 0; c < nxe; ++c) {
        int ex = exs[c], ez = ezs[a];
        int kl = q2_local_e(ix - 2 * ex, iz - 2 * ez);
        const double* row = vv + (((int64_t)ez * b.nelx + ex) * 81 + kl * 9);
        for (int j = 0; j < 9; ++j) acc += row[j] * x[q2_node(ex, ez, j, nnx)];
        dg += row[kl];
      }
    y[n] = mode == 1 ? rhs[n] - acc : acc;
    if (diag) diag[n] = dg;
  }
}

// ---------------------------------------------------------------- row planes of the solver
// The solve keeps the element-matrix rows grouped by node class (the lattice parity of the node),
// each class's rows stored as coefficient planes coef[(slot * 9 + j) * M + m] (m the node's index
// in its class, M the class size), so one warp reads 32 consecutive nodes' coefficient j in one
// coalesced access.  Classes and their incident elements, in ascending element order (the order
// the node-centric sum above visits them):
//   0 centre (odd ix, odd iz):          (ez, ex) local 8
//   1 horizontal midpoint (odd, even):  (ez-1, ex) local 6, (ez, ex) local 4
//   2 vertical midpoint (even, odd):    (ez, ex-1) local 5, (ez, ex) local 7
//   3 corner (even, even):              (ez-1, ex-1) 2, (ez-1, ex) 3, (ez, ex-1) 1, (ez, ex) 0
// Slots of boundary nodes without the element hold zeros and are skipped.
struct RowPlanes {
  int mx[4], mz[4], slots[4];
  int64_t m0[5];          // first node of each class in the flat index (m0[4] = all nodes)
  int64_t off[4];         // first coefficient of each class
  int64_t total;          // coefficients
};

inline RowPlanes row_planes(mw_box b) {
  RowPlanes P;
  const int mx[4] = {b.nelx, b.nelx, b.nelx + 1, b.nelx + 1}, mz[4] = {b.nelz, b.nelz + 1, b.nelz, b.nelz + 1};
  const int sl[4] = {1, 2, 2, 4};
  int64_t m = 0, o = 0;
  for (int c = 0; c < 4; ++c) {
    P.mx[c] = mx[c]; P.mz[c] = mz[c]; P.slots[c] = sl[c];
    P.m0[c] = m;
    P.off[c] = o;
    m += (int64_t)mx[c] * mz[c];
    o += (int64_t)sl[c] * 9 * mx[c] * mz[c];
  }
  P.m0[4] = m;
  P.total = o;
  return P;
}

// entry c of a per-class table in the kernel parameters, without indexing them at run time
// (which would copy the parameter block to local memory)
template <typename T>
MW_D T pick(const T (&a)[4], int c) { return c == 0 ? a[0] : (c == 1 ? a[1] : (c == 2 ? a[2] : a[3])); }

// element (ex, ez) and the node's local index kl in it for slot s of class c's node (i, k);
// false when the mesh has no such element
MW_D bool slot_element(int c, int s, int i, int k, const mw_box& b, int* ex, int* ez, int* kl) {
  int dx = 0, dz = 0;          // element offset from (i, k)
  if (c == 0) { *kl = 8; }
  else if (c == 1) { dz = s == 0 ? -1 : 0; *kl = s == 0 ? 6 : 4; }
  else if (c == 2) { dx = s == 0 ? -1 : 0; *kl = s == 0 ? 5 : 7; }
  else { dz = s < 2 ? -1 : 0; dx = (s & 1) ? 0 : -1; *kl = s == 0 ? 2 : (s == 1 ? 3 : (s == 2 ? 1 : 0)); }
  *ex = i + dx;
  *ez = k + dz;
  return *ex >= 0 && *ex < b.nelx && *ez >= 0 && *ez < b.nelz;
}

// class of flat node index t and its index m in the class
MW_D int class_of(const RowPlanes& P, int64_t t, int64_t* m) {
  const int c = t >= P.m0[1] ? (t >= P.m0[2] ? (t >= P.m0[3] ? 3 : 2) : 1) : 0;
  *m = t - (c == 0 ? P.m0[0] : (c == 1 ? P.m0[1] : (c == 2 ? P.m0[2] : P.m0[3])));
  return c;
}

// coefficient planes from VV_T (nel*81, build_matrix_energy.py:133-137): one thread per (node, slot)
__global__ void k_energy_rows(mw_box b, RowPlanes P, const double* __restrict__ vv, double* __restrict__ coef) {
  pdl_entry();
  const int64_t nrow = P.total / 9;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrow; r += (int64_t)gridDim.x * blockDim.x) {
    const int c = r >= P.off[3] / 9 ? 3 : (r >= P.off[2] / 9 ? 2 : (r >= P.off[1] / 9 ? 1 : 0));
    const int mxc = pick(P.mx, c);
    const int64_t off = pick(P.off, c);
    const int64_t M = (int64_t)mxc * pick(P.mz, c);
    const int64_t q = r - off / 9;
    const int s = (int)(q / M);
    const int64_t m = q - s * M;
    const int i = (int)(m % mxc), k = (int)(m / mxc);
    int ex, ez, kl;
    double* dst = coef + off + (int64_t)s * 9 * M + m;
    if (slot_element(c, s, i, k, b, &ex, &ez, &kl)) {
      const double* row = vv + (((int64_t)ez * b.nelx + ex) * 81 + kl * 9);
#pragma unroll
      for (int j = 0; j < 9; ++j) dst[j * M] = row[j];
    } else {
#pragma unroll
      for (int j = 0; j < 9; ++j) dst[j * M] = 0.0;
    }
  }
}

__global__ void k_edot_partial(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                               double* __restrict__ part) {
  pdl_entry();
  __shared__ double sh[32];
  double v = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v += a[i] * b[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) part[blockIdx.x] = v;
  }
}

__global__ void k_edot_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  pdl_entry();
  __shared__ double sh[32];
  double v = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) v += part[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) out[0] = v;
  }
}

// BiCGSTAB vector updates with device scalars s[]: see the host loop for the slot meaning.
// Deterministic grid-wide sums of K values per thread: block sums go to part[k * gridDim.x + block],
// the last block to arrive adds them in block order, writes *out[k] and resets the counter.  Called
// once, by every thread, at the end of a kernel.
template <int K>
MW_D void grid_sums(double (&v)[K], double* part, unsigned* counter, double* const (&out)[K]) {
  __shared__ double sh[K][32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double t = v[k];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sh[k][wid] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double t = 0;
      for (int w = 0; w < nw; ++w) t += sh[k][w];
      part[k * gridDim.x + blockIdx.x] = t;
    }
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double t = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) t += ((volatile double*)part)[k * gridDim.x + i];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    __syncthreads();
    if (lane == 0) sh[k][wid] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double u = 0;
      for (int w = 0; w < nw; ++w) u += sh[k][w];
      *out[k] = u;
    }
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// k_energy_matvec on the coefficient planes: the same products summed in the same order.  ND = 1
// also sums (a0, y) (the iteration's (r0, v)), ND = 2 sums (y, a0) and (y, y) ((t, s), (t, t)).
template <int ND>
__global__ void k_energy_matvec_rows(mw_box b, RowPlanes P, const double* __restrict__ coef,
                                     const double* __restrict__ x, const double* __restrict__ rhs,
                                     double* __restrict__ y, double* __restrict__ diag, int mode,
                                     const double* __restrict__ a0, double* __restrict__ part,
                                     unsigned* __restrict__ counter, double* o0, double* o1) {
  pdl_entry();
  const int nnx = 2 * b.nelx + 1;
  double v[ND > 0 ? ND : 1] = {};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < P.m0[4]; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t m;
    const int c = class_of(P, t, &m);
    const int mxc = pick(P.mx, c);
    const int64_t M = (int64_t)mxc * pick(P.mz, c);
    const int i = (int)(m % mxc), k = (int)(m / mxc);
    const int ix = 2 * i + ((c == 0 || c == 1) ? 1 : 0), iz = 2 * k + ((c == 0 || c == 2) ? 1 : 0);
    const double* cf = coef + pick(P.off, c) + m;
    const int nslot = pick(P.slots, c);
    double acc = 0.0, dg = 0.0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {                   // unrolled and predicated: the slots' loads overlap
      int ex, ez, kl;
      if (s < nslot && slot_element(c, s, i, k, b, &ex, &ez, &kl)) {
        const double* row = cf + (int64_t)s * 9 * M;
#pragma unroll
        for (int j = 0; j < 9; ++j) acc += row[j * M] * x[q2_node(ex, ez, j, nnx)];
        dg += row[kl * M];
      }
    }
    const int64_t n = (int64_t)iz * nnx + ix;
    y[n] = mode == 1 ? rhs[n] - acc : acc;
    if (diag) diag[n] = dg;
    if (ND == 1) v[0] += a0[n] * acc;
    if (ND == 2) {
      v[0] += acc * a0[n];
      v[ND - 1] += acc * acc;
    }
  }
  if (ND == 1) {
    double* const out[1] = {o0};
    grid_sums<1>(*reinterpret_cast<double(*)[1]>(v), part, counter, out);
  } else if (ND == 2) {
    double* const out[2] = {o0, o1};
    grid_sums<2>(*reinterpret_cast<double(*)[2]>(v), part, counter, out);
  }
}

// ---------------------------------------------------------------- matrix-free operator
// A = M + (dt/2)(Ka + Kd) of build_matrix_energy.py:69-114 from its Gauss-point coefficients: per
// element and Gauss point q, with xv, gr, gs the value and reference-coordinate derivatives of x,
//   P = cM xv + au gr + aw gs,  Qr = dr gr,  Qs = ds gs,   y_k += N_qk P + dN/dr_qk Qr + dN/ds_qk Qs
// and the five coefficient planes
//   cM = rho0 hcapa JxW                                                    (mass, :77)
//   au = (dt/2) cM u jcbi00,        aw = (dt/2) cM w jcbi11                (advection, :81)
//   dr = (dt/2) hcond JxW jcbi00^2, ds = (dt/2) hcond JxW jcbi11^2         (diffusion, :79)
// (the box's Jacobian is diagonal; jcbi01q and jcbi10q are not read).  Dirichlet rows and columns
// as the reference's elimination (:118-130): fixed entries of x are zeroed before the element
// products and fixed rows return diag_i x_i, diag the summed element diagonals.  A CTA owns the
// nodes of an ETX x ETZ tile of elements, recomputes a one-element halo on the left and bottom,
// and sums every owned node's incident elements in ascending element order from shared memory.
constexpr int ETX = 16, ETZ = 8;
constexpr int EEX = ETX + 1, EEZ = ETZ + 1, ENEL = EEX * EEZ;   // 153 element computations
constexpr int ELX = 2 * ETX + 3, ELZ = 2 * ETZ + 3;           // 35 x 19 staged nodes
constexpr int E_THREADS = 160;
constexpr int E_PLANES = 5;

__constant__ RefTables c_eref;

struct EnergyOp {
  const double* planes;   // [(c * 9 + q) * nel + e], c = cM, au, aw, dr, ds
  const double* diag;     // summed element diagonals (nn)
  const uint8_t* fix;     // Dirichlet flags (nn)
  int32_t* flag;          // flag word of standalone applies (after the flags, 16-byte aligned)
};

inline int64_t eop_plane_doubles(mw_box b) { return (int64_t)E_PLANES * 9 * b.nelx * b.nelz; }
inline int64_t eop_nodes(mw_box b) { return (int64_t)(2 * b.nelx + 1) * (2 * b.nelz + 1); }
inline EnergyOp eop_view(mw_box b, const void* op) {
  EnergyOp o;
  o.planes = (const double*)op;
  o.diag = o.planes + eop_plane_doubles(b);
  o.fix = reinterpret_cast<const uint8_t*>(o.diag + eop_nodes(b));
  o.flag = reinterpret_cast<int32_t*>(const_cast<uint8_t*>(o.fix) + (eop_nodes(b) + 15) / 16 * 16);
  return o;
}

MW_D double eN(int q, int k) { return c_eref.NV[q * 9 + k]; }
MW_D double eR(int q, int k) { return c_eref.dr[q * 9 + k]; }
MW_D double eS(int q, int k) { return c_eref.dt[q * 9 + k]; }

// Gauss point q's contribution to y_k (k = 0..8) of one element from the staged node values: xa
// feeds the mass term, xb the advection and diffusion terms (the same array for the operator
// itself); c: the point's five coefficients.  Terms whose basis value vanishes at a Gauss point are
// dropped at compile time.
MW_D void energy_point(int q, const double (&c)[E_PLANES], const double* xa, const double* xb, double* y) {
  double xv = 0.0, gr = 0.0, gs = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    if (ref_nv(q, k) != 0.0) xv += eN(q, k) * xa[k];
    if (ref_dr(q, k) != 0.0) gr += eR(q, k) * xb[k];
    if (ref_dt(q, k) != 0.0) gs += eS(q, k) * xb[k];
  }
  const double P = c[0] * xv + c[1] * gr + c[2] * gs;
  const double Qr = c[3] * gr, Qs = c[4] * gs;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    if (ref_nv(q, k) != 0.0) y[k] += eN(q, k) * P;
    if (ref_dr(q, k) != 0.0) y[k] += eR(q, k) * Qr;
    if (ref_dt(q, k) != 0.0) y[k] += eS(q, k) * Qs;
  }
}

// tile geometry of tile t: first owned element (ex0, ez0), owned node ranges [ix0, ix1) x [iz0, iz1)
struct ETile {
  int ex0, ez0, ix0, ix1, iz0, iz1, lx0, lz0;
};
MW_D ETile etile(const mw_box& b, int64_t t) {
  const int ntx = (b.nelx + ETX - 1) / ETX;
  ETile T;
  T.ex0 = (int)(t % ntx) * ETX;
  T.ez0 = (int)(t / ntx) * ETZ;
  T.ix0 = 2 * T.ex0;
  T.iz0 = 2 * T.ez0;
  T.ix1 = T.ex0 + ETX >= b.nelx ? 2 * b.nelx + 1 : 2 * (T.ex0 + ETX);
  T.iz1 = T.ez0 + ETZ >= b.nelz ? 2 * b.nelz + 1 : 2 * (T.ez0 + ETZ);
  T.lx0 = 2 * T.ex0 - 2;        // staged lattice origin
  T.lz0 = 2 * T.ez0 - 2;
  return T;
}

// sum over the incident elements of node (ix, iz), ascending element order, of the element-local
// values ye[element][9] of the tile
MW_D double enode_sum(const mw_box& b, const ETile& T, int ix, int iz, const double* ye) {
  const bool xo = ix & 1, zo = iz & 1;
  const int xa = xo ? (ix >> 1) : (ix >> 1) - 1, xb = ix >> 1;
  const int za = zo ? (iz >> 1) : (iz >> 1) - 1, zb = iz >> 1;
  const bool vxa = xa >= 0, vxb = !xo && xb < b.nelx;
  const bool vza = za >= 0, vzb = !zo && zb < b.nelz;
  double acc = 0.0;
  if (vza) {
    const int lez = za - (T.ez0 - 1);
    if (vxa) acc += ye[(lez * EEX + xa - (T.ex0 - 1)) * 9 + q2_local_e(ix - 2 * xa, iz - 2 * za)];
    if (vxb) acc += ye[(lez * EEX + xb - (T.ex0 - 1)) * 9 + q2_local_e(ix - 2 * xb, iz - 2 * za)];
  }
  if (vzb) {
    const int lez = zb - (T.ez0 - 1);
    if (vxa) acc += ye[(lez * EEX + xa - (T.ex0 - 1)) * 9 + q2_local_e(ix - 2 * xa, iz - 2 * zb)];
    if (vxb) acc += ye[(lez * EEX + xb - (T.ex0 - 1)) * 9 + q2_local_e(ix - 2 * xb, iz - 2 * zb)];
  }
  return acc;
}

// Set-up: the coefficient planes, the summed element diagonals, the Dirichlet flags and the
// right-hand side of build_matrix_energy.py:112-130, assembled per node:
//   rhs_i = dt (heat sources)_i + (M - (dt/2) K) T_old - A x_bc   (free rows; x_bc = bc_val on fixed
//           nodes, 0 elsewhere: the lifting of the fixed columns)
//   rhs_i = diag_i bc_val_i                                        (fixed rows)
// i.e. the element products of mass input T_old - x_bc and stiffness input -(T_old + x_bc).
__global__ void __launch_bounds__(E_THREADS) k_energy_op_setup(mw_box b, mw_energy_in in, double* __restrict__ planes,
                                                                double* __restrict__ diag, uint8_t* __restrict__ fix,
                                                                double* __restrict__ rhs) {
  pdl_entry();
  __shared__ double sa[ELZ * ELX], sb[ELZ * ELX];
  __shared__ double sy[ENEL * 9], sd[ENEL * 9];
  const int tid = threadIdx.x;
  const int nnx = 2 * b.nelx + 1, nnz = 2 * b.nelz + 1;
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  const int64_t ntile = (int64_t)((b.nelx + ETX - 1) / ETX) * ((b.nelz + ETZ - 1) / ETZ);
  const double dt = in.dt_dev ? *in.dt_dev : in.dt;
  const double h = dt * 0.5;
  for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const ETile T = etile(b, t);
    for (int i = tid; i < ELZ * ELX; i += E_THREADS) {
      const int ix = T.lx0 + i % ELX, iz = T.lz0 + i / ELX;
      double a = 0.0, c = 0.0;
      if (ix >= 0 && ix < nnx && iz >= 0 && iz < nnz) {
        const int64_t n = (int64_t)iz * nnx + ix;
        const double xbc = in.bc_fix_T[n] ? in.bc_val_T[n] : 0.0;
        a = in.T[n] - xbc;
        c = -(in.T[n] + xbc);
      }
      sa[i] = a;
      sb[i] = c;
    }
    __syncthreads();
    if (tid < ENEL) {
      const int lex = tid % EEX, lez = tid / EEX;
      const int ex = T.ex0 - 1 + lex, ez = T.ez0 - 1 + lez;
      if (ex >= 0 && ex < b.nelx && ez >= 0 && ez < b.nelz) {
        const int64_t e = (int64_t)ez * b.nelx + ex;
        const bool own = lex > 0 && lez > 0;
        double xa[9], xb[9], y[9], sk[9], dk[9];
        const int bx = 2 * lex, bz = 2 * lez;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          const int li = (bz + q2_dz(k)) * ELX + bx + q2_dx(k);
          xa[k] = sa[li];
          xb[k] = sb[li];
          y[k] = 0.0; sk[k] = 0.0; dk[k] = 0.0;
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) {
          const int64_t g = e * 9 + q;
          const double jxw = in.JxWq[g], j00 = in.jcbi00q[g], j11 = in.jcbi11q[g];
          const double cM = in.rho0 * in.hcapaq[g] * jxw, cK = h * in.hcondq[g] * jxw;
          const double c[E_PLANES] = {cM, h * cM * in.uq[g] * j00, h * cM * in.wq[g] * j11, cK * j00 * j00,
                                      cK * j11 * j11};
          double sq = in.hprodq[g] * jxw;                                       // :83
          if (in.formulation == 1) {                                            // :85-110 (EBA)
            const double exx = in.exxq[g], ezz = in.ezzq[g], exz = in.exzq[g];
            sq += 2 * in.etaq[g] *
                  (2.0 / 3.0 * exx * exx + 2.0 / 3.0 * ezz * ezz - 2.0 / 3.0 * exx * ezz + 2 * exz * exz) * jxw;
            sq += in.alphaq[g] * in.Tq[g] * (-in.wq[g] * in.rho0 * 10) * jxw;
          }
          if (own)
#pragma unroll
            for (int cc = 0; cc < E_PLANES; ++cc) planes[(int64_t)(cc * 9 + q) * nel + e] = c[cc];
          energy_point(q, c, xa, xb, y);
#pragma unroll
          for (int k = 0; k < 9; ++k) {                 // element diagonal A_kk and heat source
            if (ref_nv(q, k) != 0.0) {
              sk[k] += eN(q, k) * sq;
              double a = c[0] * eN(q, k);
              if (ref_dr(q, k) != 0.0) a += c[1] * eR(q, k);
              if (ref_dt(q, k) != 0.0) a += c[2] * eS(q, k);
              dk[k] += eN(q, k) * a;
            }
            if (ref_dr(q, k) != 0.0) dk[k] += c[3] * eR(q, k) * eR(q, k);
            if (ref_dt(q, k) != 0.0) dk[k] += c[4] * eS(q, k) * eS(q, k);
          }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          sy[tid * 9 + k] = dt * sk[k] + y[k];
          sd[tid * 9 + k] = dk[k];
        }
      }
    }
    __syncthreads();
    const int nox = T.ix1 - T.ix0, noz = T.iz1 - T.iz0;
    for (int i = tid; i < nox * noz; i += E_THREADS) {
      const int ix = T.ix0 + i % nox, iz = T.iz0 + i / nox;
      const int64_t n = (int64_t)iz * nnx + ix;
      const double d = enode_sum(b, T, ix, iz, sd);
      const uint8_t f = in.bc_fix_T[n] ? 1 : 0;
      diag[n] = d;
      fix[n] = f;
      rhs[n] = f ? d * in.bc_val_T[n] : enode_sum(b, T, ix, iz, sy);
    }
    __syncthreads();
  }
}

// Coefficients of one tile for the TMA path: planes [45][nelz][nelx] read as a 3D box of 18 x 9 x
// 45 starting at element (ex0 - 2, ez0 - 1) -- x even, so the box starts on a 16-byte boundary --
// into shared memory [45][9][18]; elements off the mesh read as zero.
constexpr int EBX = ETX + 2, EBZ = EEZ;                 // 18 x 9 elements per box
constexpr int EP_TILE = E_PLANES * 9 * EBZ * EBX;       // doubles
constexpr long long E_SPIN = 1LL << 22;                 // mbarrier polls before a tile load is given up
constexpr size_t E_SMEM_TMA = (size_t)(EP_TILE + ELZ * ELX + ENEL * 9) * sizeof(double) + 16;
constexpr size_t E_SMEM = (size_t)(ELZ * ELX + ENEL * 9) * sizeof(double);

// y = A x (MODE 0) or y = rhs - A x (MODE 1) on the owned nodes of each tile; ND = 1 also sums
// (a0, Ax), ND = 2 sums (Ax, a0) and (Ax, Ax), as k_energy_matvec_rows.  TMA: each tile's
// coefficients arrive in shared memory by one TMA box (one thread issues it, all wait on an
// mbarrier while the staging of x runs), so a CTA has its 58 KB of coefficients in flight at once
// instead of one element's 45 loads at a time; a load not complete after E_SPIN polls sets
// MW_FLAG_ITER_LIMIT in *flag (when given), waits for it once more (bounded) and stops computing.
// Without TMA (odd nelx: the planes' rows are not 16-byte multiples) the coefficients are read
// from global memory.
template <int MODE, int ND, bool TMA>
__global__ void __launch_bounds__(E_THREADS) k_energy_op_apply(const __grid_constant__ CUtensorMap tmP, mw_box b,
                                                                EnergyOp op, const double* __restrict__ x,
                                                                const double* __restrict__ rhs, double* __restrict__ y,
                                                                const double* __restrict__ a0, double* __restrict__ part,
                                                                unsigned* __restrict__ counter, double* o0, double* o1,
                                                                int32_t* flag) {
  pdl_entry();
  extern __shared__ __align__(128) double esm[];
  double* sc = esm;                                     // TMA: the tile's coefficients
  double* sx = esm + (TMA ? EP_TILE : 0);
  double* sy = sx + ELZ * ELX;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sy + ENEL * 9);
  const int tid = threadIdx.x;
  const int nnx = 2 * b.nelx + 1, nnz = 2 * b.nelz + 1;
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  const int64_t ntile = (int64_t)((b.nelx + ETX - 1) / ETX) * ((b.nelz + ETZ - 1) / ETZ);
  double v[ND > 0 ? ND : 1] = {};
  if (TMA) {
    if (tid == 0) {
      mbar_init(bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  uint32_t parity = 0;
  for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const ETile T = etile(b, t);
    if (TMA && tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier reads of sc before the copy
      mbar_expect_tx(bar, (uint32_t)(EP_TILE * sizeof(double)));
      tma_load_3d(sc, &tmP, bar, T.ex0 - 2, T.ez0 - 1, 0);
    }
    {  // stage x (fixed entries zeroed): every load issued before any store, one round trip
      constexpr int NS = (ELZ * ELX + E_THREADS - 1) / E_THREADS;
      double xv[NS];
      uint8_t fv[NS];
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const int i = tid + k * E_THREADS;
        const int ix = T.lx0 + i % ELX, iz = T.lz0 + i / ELX;
        xv[k] = 0.0;
        fv[k] = 1;
        if (i < ELZ * ELX && ix >= 0 && ix < nnx && iz >= 0 && iz < nnz) {
          const int64_t n = (int64_t)iz * nnx + ix;
          fv[k] = op.fix[n];
          xv[k] = x[n];
        }
      }
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const int i = tid + k * E_THREADS;
        if (i < ELZ * ELX) sx[i] = fv[k] ? 0.0 : xv[k];
      }
    }
    if (TMA) {
      const bool ok = mbar_wait_bounded(bar, parity, E_SPIN);
      parity ^= 1u;
      if (__syncthreads_or(!ok)) {                     // give up: flag, drain the copy, stop
        if (tid == 0) {
          if (flag) atomicOr(flag, MW_FLAG_ITER_LIMIT);
          mbar_wait_bounded(bar, parity ^ 1u, E_SPIN);
        }
        __syncthreads();
        break;
      }
    } else {
      __syncthreads();
    }
    if (tid < ENEL) {
      const int lex = tid % EEX, lez = tid / EEX;
      const int ex = T.ex0 - 1 + lex, ez = T.ez0 - 1 + lez;
      if (ex >= 0 && ex < b.nelx && ez >= 0 && ez < b.nelz) {
        const int64_t e = (int64_t)ez * b.nelx + ex;
        double xe[9], ye[9];
        const int bx = 2 * lex, bz = 2 * lez;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          xe[k] = sx[(bz + q2_dz(k)) * ELX + bx + q2_dx(k)];
          ye[k] = 0.0;
        }
        const double* pl = op.planes + e;
        const double* ps = sc + lez * EBX + lex + 1;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
          double c[E_PLANES];
#pragma unroll
          for (int cc = 0; cc < E_PLANES; ++cc)
            c[cc] = TMA ? ps[(cc * 9 + q) * EBZ * EBX] : __ldg(pl + (int64_t)(cc * 9 + q) * nel);
          energy_point(q, c, xe, xe, ye);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) sy[tid * 9 + k] = ye[k];
      }
    }
    __syncthreads();
    {  // owned nodes: the loads of every node first, then the (rare) fixed rows, then the stores
      const int nox = T.ix1 - T.ix0, noz = T.iz1 - T.iz0;
      constexpr int NO = ((2 * ETX + 1) * (2 * ETZ + 1) + E_THREADS - 1) / E_THREADS;
      int64_t nk[NO];
      uint8_t fk[NO];
      double acc[NO], bk[NO], ak[NO];
#pragma unroll
      for (int k = 0; k < NO; ++k) {
        const int i = tid + k * E_THREADS;
        nk[k] = -1;
        fk[k] = 0;
        acc[k] = bk[k] = ak[k] = 0.0;
        if (i < nox * noz) {
          const int ix = T.ix0 + i % nox, iz = T.iz0 + i / nox;
          const int64_t n = (int64_t)iz * nnx + ix;
          nk[k] = n;
          fk[k] = op.fix[n];
          if (MODE == 1) bk[k] = rhs[n];
          if (ND > 0) ak[k] = a0[n];
          acc[k] = enode_sum(b, T, ix, iz, sy);
        }
      }
#pragma unroll
      for (int k = 0; k < NO; ++k)
        if (nk[k] >= 0 && fk[k]) acc[k] = op.diag[nk[k]] * x[nk[k]];
#pragma unroll
      for (int k = 0; k < NO; ++k) {
        if (nk[k] < 0) continue;
        y[nk[k]] = MODE == 1 ? bk[k] - acc[k] : acc[k];
        if (ND == 1) v[0] += ak[k] * acc[k];
        if (ND == 2) {
          v[0] += acc[k] * ak[k];
          v[ND - 1] += acc[k] * acc[k];
        }
      }
    }
    __syncthreads();
  }
  if (ND == 1) {
    double* const out[1] = {o0};
    grid_sums<1>(*reinterpret_cast<double(*)[1]>(v), part, counter, out);
  } else if (ND == 2) {
    double* const out[2] = {o0, o1};
    grid_sums<2>(*reinterpret_cast<double(*)[2]>(v), part, counter, out);
  }
}

// The coefficient-plane map of the TMA path; false when the planes cannot be described (odd nelx).
static bool eop_plane_map(CUtensorMap* m, mw_box b, const void* op) {
  auto enc = get_encode();
  if (!enc || (b.nelx & 1) || ((uintptr_t)op & 15)) return false;
  cuuint64_t dims[3] = {(cuuint64_t)b.nelx, (cuuint64_t)b.nelz, (cuuint64_t)(E_PLANES * 9)};
  cuuint64_t strides[2] = {(cuuint64_t)b.nelx * 8, (cuuint64_t)b.nelx * b.nelz * 8};
  cuuint32_t box[3] = {(cuuint32_t)EBX, (cuuint32_t)EBZ, (cuuint32_t)(E_PLANES * 9)};
  cuuint32_t estr[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(op), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Launches k_energy_op_apply<MODE, ND> on the TMA path when the map could be made.
template <int MODE, int ND>
static void launch_eop_apply(bool tma, const CUtensorMap& tm, int grid, cudaStream_t s, mw_box b, const EnergyOp& op,
                             const double* x, const double* rhs, double* y, const double* a0, double* part,
                             unsigned* counter, double* o0, double* o1, int32_t* flag) {
  if (tma) {
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(k_energy_op_apply<MODE, ND, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)E_SMEM_TMA);
      attr = true;
    }
    pdl_launch(k_energy_op_apply<MODE, ND, true>, grid, E_THREADS, E_SMEM_TMA, s, tm, b, op, x, rhs, y, a0, part, counter,
               o0, o1, flag);
  } else {
    pdl_launch(k_energy_op_apply<MODE, ND, false>, grid, E_THREADS, E_SMEM, s, tm, b, op, x, rhs, y, a0, part, counter,
               o0, o1, flag);
  }
}

// Scalar slots of the iteration (sc): 0 rho = (r0, r), 1 rho of the previous iteration, 2 alpha,
// 3 omega, 4 (r0, v), 5 (t, s), 6 (t, t), 7 (r0, r) of the new residual, 10 (b, b), 11 (r, r),
// 12 iteration count.  Each iteration is six launches: the direction update, A p^ with (r0, v),
// the s update, A s^ with (t, s) and (t, t), the x / r update with (r, r) and (r0, r), the scalar
// roll with the loop test.

// p = r + beta (p - omega v), beta = (rho/rho_old) (alpha/omega) (p = r on the first iteration);
// p^ = D^-1 p
__global__ void k_bicg_p(int64_t n, const double* __restrict__ sc, const double* __restrict__ r,
                         const double* __restrict__ v, double* __restrict__ p, const double* __restrict__ dg,
                         double* __restrict__ ph) {
  pdl_entry();
  const bool first = sc[12] == 0.0;
  const double beta = first ? 0.0 : (sc[0] / sc[1]) * (sc[2] / sc[3]);
  const double om = first ? 0.0 : sc[3];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double pi = first ? r[i] : r[i] + beta * (p[i] - om * v[i]);   // the first pass never reads p, v
    p[i] = pi;
    ph[i] = pi / dg[i];
  }
}

// s = r - alpha v, alpha = rho / (r0, v); s^ = D^-1 s
__global__ void k_bicg_s(int64_t n, const double* __restrict__ sc, const double* __restrict__ r,
                         const double* __restrict__ v, double* __restrict__ sv, const double* __restrict__ dg,
                         double* __restrict__ sh) {
  pdl_entry();
  const double alpha = sc[0] / sc[4];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double si = r[i] - alpha * v[i];
    sv[i] = si;
    sh[i] = si / dg[i];
  }
}

// x += alpha p^ + omega s^ ; r = s - omega t ; omega = (t, s) / (t, t); then (r, r) -> sc[11] and
// (r0, r) -> sc[7]
__global__ void k_bicg_x(int64_t n, double* __restrict__ sc, const double* __restrict__ ph,
                         const double* __restrict__ sh, const double* __restrict__ sv, const double* __restrict__ t,
                         const double* __restrict__ r0, double* __restrict__ x, double* __restrict__ r,
                         double* __restrict__ part, unsigned* __restrict__ counter) {
  pdl_entry();
  const double alpha = sc[0] / sc[4];
  const double omega = sc[6] != 0.0 ? sc[5] / sc[6] : 0.0;
  double v[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += alpha * ph[i] + omega * sh[i];
    const double ri = sv[i] - omega * t[i];
    r[i] = ri;
    v[0] += ri * ri;
    v[1] += r0[i] * ri;
  }
  double* const out[2] = {sc + 11, sc + 7};
  grid_sums<2>(v, part, counter, out);
}

// keep alpha (slot 2) and omega (slot 3) of this iteration, rho_old <- rho, rho <- (r0, r);
// count the iteration and, inside a recorded graph (use_h), set the loop condition: continue while
// the residual is finite, above rtol * ||b|| and the count is below maxit
__global__ void k_bicg_roll(double* sc, double rtol, int maxit, cudaGraphConditionalHandle h, int use_h) {
  pdl_entry();
  if (threadIdx.x || blockIdx.x) return;
  sc[2] = sc[0] / sc[4];
  sc[3] = sc[6] != 0.0 ? sc[5] / sc[6] : 0.0;
  sc[1] = sc[0];
  sc[0] = sc[7];
  const double it = sc[12] + 1;
  sc[12] = it;
  const double rr = sc[11];
  if (use_h) cudaGraphSetConditional(h, (isfinite(rr) && rr > rtol * rtol * sc[10] && it < (double)maxit) ? 1u : 0u);
}

// ---- the iteration as a recorded CUDA graph with a device WHILE loop ----
// sc[12] = iteration count; rho = (r0, r) = (r, r) to start with (r0 = r)
__global__ void k_bicg_init(double* sc, double rtol, int maxit, cudaGraphConditionalHandle h, int use_h) {
  pdl_entry();
  if (!(sc[10] > 0)) sc[10] = 1.0;
  sc[12] = 0;
  sc[0] = sc[11];
  const double rr = sc[11];
  if (use_h) cudaGraphSetConditional(h, (isfinite(rr) && rr > rtol * rtol * sc[10] && maxit > 0) ? 1u : 0u);
}

// Workspace of the solve (doubles): nine node vectors, then the dot-product partials, the device
// scalars and the row planes.
constexpr int E_NB = 1184;                 // dot-product CTAs (8 per SM); two partials per CTA
constexpr int64_t E_SC = 2 * E_NB + 16;    // scalars, after the partials (slot 200: the arrival counter)
constexpr int64_t E_COEF = E_SC + 256;     // row planes, after the scalars

// The operator of a solve: the element matrices VV_T (row planes built from them in the
// workspace), or a matrix-free operator from mw_energy_op_setup.
struct EnergyA {
  const double* VV;
  const void* op;
};

struct EnergyGraph {
  int dev;
  const void *VV, *rhs, *T, *work;   // VV: the operator (VV_T or the matrix-free operator)
  int nelx, nelz, maxit;
  double rtol;
  cudaGraphExec_t exec;
};
static std::vector<EnergyGraph> g_energy_graphs;
static std::mutex g_energy_mutex;
static cudaStream_t g_energy_stream[64], g_energy_body[64];   // library stream, body-capture stream
static cudaEvent_t g_energy_ev[64][2];
static uint64_t g_eref_ready = 0;   // devices whose c_eref is loaded

// The reference-element tables of the matrix-free operator in this device's constant bank (once
// per device; synchronous, so the first call on a device precedes any stream capture).
static int ensure_energy_tables() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MW_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_energy_mutex);
  if (g_eref_ready >> dev & 1u) return MW_OK;
  RefTables T;
  host_ref_tables(&T);
  if (cudaMemcpyToSymbol(c_eref, &T, sizeof(T)) != cudaSuccess) return MW_ERR_CUDA;
  g_eref_ready |= uint64_t(1) << dev;
  return MW_OK;
}

}  // namespace mw

using namespace mw;

extern "C" {

size_t mw_energy_solve_workspace_bytes(mw_box box) {
  int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  return (size_t)(9 * nn + E_COEF + row_planes(box).total) * sizeof(double);
}

int mw_energy_device_info(mw_box box, const void* work, int32_t* iters, double* relres, void* stream) {
  const int64_t n = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  const double* sc = (const double*)work + 9 * n + E_SC;
  double q[3];
  int32_t flag = 0;
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemcpyAsync(q, sc + 10, sizeof(q), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&flag, sc + 202, sizeof(flag), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return MW_ERR_CUDA;
  if (iters) *iters = (int32_t)q[2];
  if (relres) *relres = flag ? NAN : std::sqrt(q[1] / q[0]);     // a tile load given up: no result
  return MW_OK;
}

int mw_energy_matvec(mw_box box, const double* VV_T, const double* x, double* y, void* stream) {
  int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  pdl_launch(k_energy_matvec, grid_for(nn, 256), 256, 0, (cudaStream_t)stream, box, VV_T, x, nullptr, y, nullptr, 0);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

// The buffers of the solve in its workspace (doubles): r, r0, p, v, s, t, p^, s^, diag, the
// dot-product partials, the scalar slots (the arrival counter of the fused dot products in slot
// 200) and the row planes.
struct EnergyBufs {
  int64_t n;
  double *r, *r0, *p, *v, *sv, *t, *ph, *sh, *dg, *part, *sc, *coef;
  unsigned* counter;
  RowPlanes RP;
  int grid;               // CTAs of the node kernels (at most E_NB: one partial slot each)
  EnergyA A;
  EnergyOp op;            // the matrix-free operator's view (A.op set)
  int grid_op;            // CTAs of the matrix-free apply (tile loop; at most E_NB)
  bool tma;               // coefficient tiles by TMA (the plane map could be made)
  CUtensorMap tm;
  int32_t* flag;          // device flag word of the solve (a tile load given up)
};

static EnergyBufs energy_bufs(mw_box box, void* work, EnergyA A) {
  EnergyBufs E;
  E.A = A;
  E.n = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  double* w = (double*)work;
  const int64_t n = E.n;
  E.r = w; E.r0 = w + n; E.p = w + 2 * n; E.v = w + 3 * n; E.sv = w + 4 * n; E.t = w + 5 * n;
  E.ph = w + 6 * n; E.sh = w + 7 * n; E.dg = w + 8 * n;
  E.part = w + 9 * n;
  E.sc = w + 9 * n + E_SC;
  E.counter = reinterpret_cast<unsigned*>(E.sc + 200);
  E.coef = w + 9 * n + E_COEF;
  E.RP = row_planes(box);
  E.grid = std::min(grid_for(n, 256), E_NB);
  E.flag = reinterpret_cast<int32_t*>(E.sc + 202);
  E.tma = false;
  memset(&E.tm, 0, sizeof(E.tm));
  if (A.op) {
    E.op = eop_view(box, A.op);
    E.dg = const_cast<double*>(E.op.diag);
    const int64_t ntile = (int64_t)((box.nelx + ETX - 1) / ETX) * ((box.nelz + ETZ - 1) / ETZ);
    E.grid_op = (int)std::min<int64_t>(ntile, E_NB);
    E.tma = eop_plane_map(&E.tm, box, A.op);
  }
  return E;
}

// Row planes from VV_T, r = b - A T (T holds the initial guess) with diag(A), r0 = r, (b, b) and
// (r, r) into sc[10], sc[11].
static void energy_start(const EnergyBufs& E, mw_box box, const double* rhs, double* T, cudaStream_t s) {
  cudaMemsetAsync(E.counter, 0, 4 * sizeof(double), s);        // arrival counter and flag word (slots 200-203)
  if (E.A.op) {
    launch_eop_apply<1, 0>(E.tma, E.tm, E.grid_op, s, box, E.op, T, rhs, E.r, nullptr, nullptr, nullptr, nullptr,
                           nullptr, E.flag);
  } else {
    pdl_launch(k_energy_rows, grid_for(E.RP.total / 9, 256), 256, 0, s, box, E.RP, E.A.VV, E.coef);
    pdl_launch(k_energy_matvec_rows<0>, E.grid, 256, 0, s, box, E.RP, E.coef, T, rhs, E.r, E.dg, 1, nullptr,
               nullptr, nullptr, nullptr, nullptr);
  }
  cudaMemcpyAsync(E.r0, E.r, sizeof(double) * E.n, cudaMemcpyDeviceToDevice, s);
  const double* a[2] = {rhs, E.r};
  for (int k = 0; k < 2; ++k) {
    pdl_launch(k_edot_partial, E_NB, 256, 0, s, E.n, a[k], a[k], E.part);
    pdl_launch(k_edot_final, 1, 256, 0, s, E.part, E_NB, E.sc + 10 + k);
  }
}

// One BiCGSTAB iteration (Jacobi-preconditioned), six launches; with use_h the last one sets the
// WHILE condition of the recorded loop.
static void energy_iteration(const EnergyBufs& E, mw_box box, double* T, double rtol, int maxit,
                             cudaGraphConditionalHandle h, int use_h, cudaStream_t s) {
  pdl_launch(k_bicg_p, E.grid, 256, 0, s, E.n, E.sc, E.r, E.v, E.p, E.dg, E.ph);
  if (E.A.op)
    launch_eop_apply<0, 1>(E.tma, E.tm, E.grid_op, s, box, E.op, E.ph, nullptr, E.v, E.r0, E.part, E.counter, E.sc + 4,
                           nullptr, E.flag);
  else
    pdl_launch(k_energy_matvec_rows<1>, E.grid, 256, 0, s, box, E.RP, E.coef, E.ph, nullptr, E.v, nullptr, 0, E.r0,
               E.part, E.counter, E.sc + 4, nullptr);
  pdl_launch(k_bicg_s, E.grid, 256, 0, s, E.n, E.sc, E.r, E.v, E.sv, E.dg, E.sh);
  if (E.A.op)
    launch_eop_apply<0, 2>(E.tma, E.tm, E.grid_op, s, box, E.op, E.sh, nullptr, E.t, E.sv, E.part, E.counter, E.sc + 5,
                           E.sc + 6, E.flag);
  else
    pdl_launch(k_energy_matvec_rows<2>, E.grid, 256, 0, s, box, E.RP, E.coef, E.sh, nullptr, E.t, nullptr, 0, E.sv,
               E.part, E.counter, E.sc + 5, E.sc + 6);
  pdl_launch(k_bicg_x, E.grid, 256, 0, s, E.n, E.sc, E.ph, E.sh, E.sv, E.t, E.r0, T, E.r, E.part, E.counter);
  pdl_launch(k_bicg_roll, 1, 32, 0, s, E.sc, rtol, maxit, h, use_h);
}

// Records the BiCGSTAB solve on the capturing stream s (body captured on b); false on failure.
static bool energy_record(mw_box box, EnergyA A, const double* rhs, double* T, double rtol, int maxit, void* work,
                          cudaStream_t s, cudaStream_t b);

// The solve from a graph recorded once per (device, buffers, sizes, rtol, maxit).  A caller's own
// (non-default) stream is captured and launched on directly, so solves of models on different
// streams run concurrently; the legacy default stream, which cannot be captured, is served through
// a library stream ordered after / before it by events.  Returns false when no graph can be used.
static bool energy_solve_graph(mw_box box, EnergyA A, const double* rhs, double* T, double rtol, int32_t maxit,
                               int32_t* iters, double* relres, void* work, cudaStream_t caller) {
  const void* key = A.op ? A.op : (const void*)A.VV;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  const bool legacy = caller == nullptr || caller == cudaStreamLegacy || caller == cudaStreamPerThread;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t s = caller;
  {
    std::lock_guard<std::mutex> lock(g_energy_mutex);
    if (!g_energy_body[dev]) {
      if (cudaStreamCreateWithFlags(&g_energy_stream[dev], cudaStreamNonBlocking) != cudaSuccess ||
          cudaStreamCreateWithFlags(&g_energy_body[dev], cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&g_energy_ev[dev][0], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&g_energy_ev[dev][1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
    }
    if (legacy) s = g_energy_stream[dev];
    for (auto& e : g_energy_graphs)
      if (e.dev == dev && e.VV == key && e.rhs == rhs && e.T == T && e.work == work && e.nelx == box.nelx &&
          e.nelz == box.nelz && e.maxit == maxit && e.rtol == rtol) { exec = e.exec; break; }
    if (!exec) {
      if (g_energy_graphs.size() >= 512) return false;
      cudaStream_t rec = g_energy_stream[dev];   // recording only records: any capturable stream will do
      if (cudaStreamBeginCapture(rec, cudaStreamCaptureModeThreadLocal) != cudaSuccess) { cudaGetLastError(); return false; }
      bool ok = energy_record(box, A, rhs, T, rtol, maxit, work, rec, g_energy_body[dev]);
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(g_energy_body[dev], &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t gb = nullptr;
        cudaStreamEndCapture(g_energy_body[dev], &gb);
        ok = false;
      }
      cudaGraph_t g = nullptr;
      ok = cudaStreamEndCapture(rec, &g) == cudaSuccess && g && ok && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
      if (!ok) { cudaGetLastError(); return false; }
      g_energy_graphs.push_back({dev, key, rhs, T, work, box.nelx, box.nelz, maxit, rtol, exec});
    }
    if (legacy) {   // the library stream is shared: keep this path serialised
      cudaEventRecord(g_energy_ev[dev][0], caller);
      cudaStreamWaitEvent(s, g_energy_ev[dev][0], 0);
      if (cudaGraphLaunch(exec, s) != cudaSuccess) { cudaGetLastError(); return false; }
      cudaEventRecord(g_energy_ev[dev][1], s);
      cudaStreamWaitEvent(caller, g_energy_ev[dev][1], 0);
    }
  }
  if (!legacy && cudaGraphLaunch(exec, s) != cudaSuccess) { cudaGetLastError(); return false; }
  const int64_t n = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  const double* sc = (const double*)work + 9 * n + E_SC;
  double q[3];
  int32_t flag = 0;
  cudaMemcpyAsync(q, sc + 10, sizeof(q), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&flag, sc + 202, sizeof(flag), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return false;
  if (iters) *iters = (int32_t)q[2];
  if (relres) *relres = flag ? NAN : std::sqrt(q[1] / q[0]);
  return true;
}

}  // extern "C"

static int energy_solve(mw_box box, EnergyA A, const double* rhs, double* T, double rtol, int32_t maxit,
                        int32_t* iters, double* relres, void* work, void* stream) {
  {  // the caller is recording a graph: record the solve into it, results stay on the device
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStream_t cs_stream = (cudaStream_t)stream;
    if (cs_stream != nullptr && cudaStreamIsCapturing(cs_stream, &cs) == cudaSuccess &&
        cs == cudaStreamCaptureStatusActive) {
      int dev = 0;
      if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MW_ERR_CUDA;
      std::lock_guard<std::mutex> lock(g_energy_mutex);
      if (!g_energy_body[dev] && cudaStreamCreateWithFlags(&g_energy_body[dev], cudaStreamNonBlocking) != cudaSuccess)
        return MW_ERR_CUDA;
      if (!energy_record(box, A, rhs, T, rtol, maxit, work, cs_stream, g_energy_body[dev])) return MW_ERR_CUDA;
      if (iters) *iters = 0;
      if (relres) *relres = 0;
      return MW_OK;
    }
    cudaGetLastError();
  }
  {
    int32_t it = 0;
    double rel = 0;
    if (energy_solve_graph(box, A, rhs, T, rtol, maxit, &it, &rel, work, (cudaStream_t)stream)) {
      if (iters) *iters = it;
      if (relres) *relres = rel;
      if (cudaGetLastError() != cudaSuccess) return MW_ERR_CUDA;
      return rel <= rtol ? MW_OK : MW_ERR_NOT_CONVERGED;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  const EnergyBufs E = energy_bufs(box, work, A);
  auto rd = [&](const double* d) {
    double h = 0;
    cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return h;
  };
  energy_start(E, box, rhs, T, s);
  pdl_launch(k_bicg_init, 1, 1, 0, s, E.sc, rtol, maxit, cudaGraphConditionalHandle(0), 0);
  double bb = rd(E.sc + 10);
  double rr = rd(E.sc + 11);
  int it = 0;
  for (it = 1; it <= maxit && rr > rtol * rtol * bb; ++it) {
    energy_iteration(E, box, T, rtol, maxit, cudaGraphConditionalHandle(0), 0, s);
    rr = rd(E.sc + 11);
    if (!std::isfinite(rr)) break;
  }
  int32_t flag = 0;
  cudaMemcpyAsync(&flag, E.flag, sizeof(flag), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  const double rel = flag ? NAN : std::sqrt(rr / bb);   // a tile load given up: no result
  if (iters) *iters = it - 1;
  if (relres) *relres = rel;
  if (cudaGetLastError() != cudaSuccess) return MW_ERR_CUDA;
  return rel <= rtol ? MW_OK : MW_ERR_NOT_CONVERGED;
}

extern "C" {

int mw_energy_solve(mw_box box, const double* VV_T, const double* rhs, double* T, double rtol, int32_t maxit,
                    int32_t* iters, double* relres, void* work, size_t work_bytes, void* stream) {
  if (!VV_T || work_bytes < mw_energy_solve_workspace_bytes(box) || maxit < 1) return MW_ERR_BAD_ARG;
  return energy_solve(box, EnergyA{VV_T, nullptr}, rhs, T, rtol, maxit, iters, relres, work, stream);
}

size_t mw_energy_op_bytes(mw_box box) {
  if (box.nelx <= 0 || box.nelz <= 0) return 0;
  return (size_t)(eop_plane_doubles(box) + eop_nodes(box)) * sizeof(double) + (size_t)((eop_nodes(box) + 15) / 16) * 16 +
         16;
}

int mw_energy_op_setup(mw_box box, mw_energy_in in, void* op, size_t op_bytes, double* rhs, void* stream) {
  if (box.nelx <= 0 || box.nelz <= 0 || !op || !rhs || op_bytes < mw_energy_op_bytes(box)) return MW_ERR_BAD_ARG;
  if (!in.T || !in.uq || !in.wq || !in.hcondq || !in.hcapaq || !in.hprodq || !in.JxWq || !in.jcbi00q || !in.jcbi11q ||
      !in.bc_fix_T || !in.bc_val_T)
    return MW_ERR_BAD_ARG;
  if (in.formulation == 1 && (!in.etaq || !in.exxq || !in.ezzq || !in.exzq || !in.alphaq || !in.Tq))
    return MW_ERR_BAD_ARG;
  if (ensure_energy_tables() != MW_OK) return MW_ERR_CUDA;
  double* planes = (double*)op;
  double* diag = planes + eop_plane_doubles(box);
  uint8_t* fix = reinterpret_cast<uint8_t*>(diag + eop_nodes(box));
  const int64_t ntile = (int64_t)((box.nelx + ETX - 1) / ETX) * ((box.nelz + ETZ - 1) / ETZ);
  if (cudaMemsetAsync(eop_view(box, op).flag, 0, 16, (cudaStream_t)stream) != cudaSuccess) return MW_ERR_CUDA;
  pdl_launch(k_energy_op_setup, (int)std::min<int64_t>(ntile, 8 * num_sms()), E_THREADS, 0, (cudaStream_t)stream, box,
             in, planes, diag, fix, rhs);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_energy_op_apply(mw_box box, const void* op, const double* x, double* y, void* stream) {
  if (box.nelx <= 0 || box.nelz <= 0 || !op || !x || !y) return MW_ERR_BAD_ARG;
  if (ensure_energy_tables() != MW_OK) return MW_ERR_CUDA;
  const int64_t ntile = (int64_t)((box.nelx + ETX - 1) / ETX) * ((box.nelz + ETZ - 1) / ETZ);
  CUtensorMap tm;
  memset(&tm, 0, sizeof(tm));
  const bool tma = eop_plane_map(&tm, box, op);
  const EnergyOp o = eop_view(box, op);
  launch_eop_apply<0, 0>(tma, tm, (int)std::min<int64_t>(ntile, E_NB), (cudaStream_t)stream, box, o, x, nullptr, y,
                         nullptr, nullptr, nullptr, nullptr, nullptr, o.flag);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

size_t mw_energy_op_solve_workspace_bytes(mw_box box) {
  int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  return (size_t)(9 * nn + E_COEF) * sizeof(double);
}

int mw_energy_op_solve(mw_box box, const void* op, const double* rhs, double* T, double rtol, int32_t maxit,
                       int32_t* iters, double* relres, void* work, size_t work_bytes, void* stream) {
  if (!op || work_bytes < mw_energy_op_solve_workspace_bytes(box) || maxit < 1) return MW_ERR_BAD_ARG;
  if (ensure_energy_tables() != MW_OK) return MW_ERR_CUDA;
  return energy_solve(box, EnergyA{nullptr, op}, rhs, T, rtol, maxit, iters, relres, work, stream);
}

}  // extern "C"

static bool energy_record(mw_box box, EnergyA A, const double* rhs, double* T, double rtol, int maxit, void* work,
                          cudaStream_t s, cudaStream_t b) {
  const EnergyBufs E = energy_bufs(box, work, A);
  energy_start(E, box, rhs, T, s);
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  if (cudaStreamGetCaptureInfo(s, &st, nullptr, &g, nullptr, nullptr) != cudaSuccess) return false;
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) return false;
  pdl_launch(k_bicg_init, 1, 1, 0, s, E.sc, rtol, maxit, h, 1);
  if (cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd) != cudaSuccess) return false;
  cudaGraphNodeParams prm = {cudaGraphNodeTypeConditional};
  prm.conditional.handle = h;
  prm.conditional.type = cudaGraphCondTypeWhile;
  prm.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, g, deps, nd, &prm) != cudaSuccess) return false;
  if (cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) return false;
  if (cudaStreamBeginCaptureToGraph(b, prm.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return false;
  energy_iteration(E, box, T, rtol, maxit, h, 1, b);         // the body: one iteration and the loop test
  cudaGraph_t gb = nullptr;
  return cudaStreamEndCapture(b, &gb) == cudaSuccess;
}
