// Device solve of the Crank-Nicolson energy system (sm_100a).
//
// Reference: meeuuw.py:2232-2235 converts (II_T, JJ_T, VV_T) to CSR (summing duplicates) and calls
// SuperLU's spsolve.  Here the element matrices VV_T written by build_matrix_energy
// (build_matrix_energy.py:133-137, nel*81 values) are used directly: y = A x is a node-centric
// gather over the (up to 4) incident elements in ascending element order -- the summed COO
// matrix applied without forming it -- and the system is solved by Jacobi-preconditioned
// BiCGSTAB in FP64 to a relative residual tolerance.  The solve first regroups the rows by node
// class (k_energy_rows) so that every matvec of the iteration reads them coalesced.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"

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

struct EnergyGraph {
  int dev;
  const void *VV, *rhs, *T, *work;
  int nelx, nelz, maxit;
  double rtol;
  cudaGraphExec_t exec;
};
static std::vector<EnergyGraph> g_energy_graphs;
static std::mutex g_energy_mutex;
static cudaStream_t g_energy_stream[64], g_energy_body[64];   // library stream, body-capture stream
static cudaEvent_t g_energy_ev[64][2];

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
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemcpyAsync(q, sc + 10, sizeof(q), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return MW_ERR_CUDA;
  if (iters) *iters = (int32_t)q[2];
  if (relres) *relres = std::sqrt(q[1] / q[0]);
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
};

static EnergyBufs energy_bufs(mw_box box, void* work) {
  EnergyBufs E;
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
  return E;
}

// Row planes from VV_T, r = b - A T (T holds the initial guess) with diag(A), r0 = r, (b, b) and
// (r, r) into sc[10], sc[11].
static void energy_start(const EnergyBufs& E, mw_box box, const double* VV_T, const double* rhs, double* T,
                         cudaStream_t s) {
  cudaMemsetAsync(E.counter, 0, sizeof(unsigned), s);
  pdl_launch(k_energy_rows, grid_for(E.RP.total / 9, 256), 256, 0, s, box, E.RP, VV_T, E.coef);
  pdl_launch(k_energy_matvec_rows<0>, E.grid, 256, 0, s, box, E.RP, E.coef, T, rhs, E.r, E.dg, 1, nullptr,
             nullptr, nullptr, nullptr, nullptr);
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
  pdl_launch(k_energy_matvec_rows<1>, E.grid, 256, 0, s, box, E.RP, E.coef, E.ph, nullptr, E.v, nullptr, 0, E.r0,
             E.part, E.counter, E.sc + 4, nullptr);
  pdl_launch(k_bicg_s, E.grid, 256, 0, s, E.n, E.sc, E.r, E.v, E.sv, E.dg, E.sh);
  pdl_launch(k_energy_matvec_rows<2>, E.grid, 256, 0, s, box, E.RP, E.coef, E.sh, nullptr, E.t, nullptr, 0, E.sv,
             E.part, E.counter, E.sc + 5, E.sc + 6);
  pdl_launch(k_bicg_x, E.grid, 256, 0, s, E.n, E.sc, E.ph, E.sh, E.sv, E.t, E.r0, T, E.r, E.part, E.counter);
  pdl_launch(k_bicg_roll, 1, 32, 0, s, E.sc, rtol, maxit, h, use_h);
}

// Records the BiCGSTAB solve on the capturing stream s (body captured on b); false on failure.
static bool energy_record(mw_box box, const double* VV_T, const double* rhs, double* T, double rtol, int maxit,
                          void* work, cudaStream_t s, cudaStream_t b);

// The solve from a graph recorded once per (device, buffers, sizes, rtol, maxit).  A caller's own
// (non-default) stream is captured and launched on directly, so solves of models on different
// streams run concurrently; the legacy default stream, which cannot be captured, is served through
// a library stream ordered after / before it by events.  Returns false when no graph can be used.
static bool energy_solve_graph(mw_box box, const double* VV_T, const double* rhs, double* T, double rtol,
                               int32_t maxit, int32_t* iters, double* relres, void* work, cudaStream_t caller) {
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
      if (e.dev == dev && e.VV == VV_T && e.rhs == rhs && e.T == T && e.work == work && e.nelx == box.nelx &&
          e.nelz == box.nelz && e.maxit == maxit && e.rtol == rtol) { exec = e.exec; break; }
    if (!exec) {
      if (g_energy_graphs.size() >= 512) return false;
      cudaStream_t rec = g_energy_stream[dev];   // recording only records: any capturable stream will do
      if (cudaStreamBeginCapture(rec, cudaStreamCaptureModeThreadLocal) != cudaSuccess) { cudaGetLastError(); return false; }
      bool ok = energy_record(box, VV_T, rhs, T, rtol, maxit, work, rec, g_energy_body[dev]);
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
      g_energy_graphs.push_back({dev, VV_T, rhs, T, work, box.nelx, box.nelz, maxit, rtol, exec});
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
  cudaMemcpyAsync(q, sc + 10, sizeof(q), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return false;
  if (iters) *iters = (int32_t)q[2];
  if (relres) *relres = std::sqrt(q[1] / q[0]);
  return true;
}

int mw_energy_solve(mw_box box, const double* VV_T, const double* rhs, double* T, double rtol, int32_t maxit,
                    int32_t* iters, double* relres, void* work, size_t work_bytes, void* stream) {
  if (work_bytes < mw_energy_solve_workspace_bytes(box) || maxit < 1) return MW_ERR_BAD_ARG;
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
      if (!energy_record(box, VV_T, rhs, T, rtol, maxit, work, cs_stream, g_energy_body[dev])) return MW_ERR_CUDA;
      if (iters) *iters = 0;
      if (relres) *relres = 0;
      return MW_OK;
    }
    cudaGetLastError();
  }
  {
    int32_t it = 0;
    double rel = 0;
    if (energy_solve_graph(box, VV_T, rhs, T, rtol, maxit, &it, &rel, work, (cudaStream_t)stream)) {
      if (iters) *iters = it;
      if (relres) *relres = rel;
      if (cudaGetLastError() != cudaSuccess) return MW_ERR_CUDA;
      return rel <= rtol ? MW_OK : MW_ERR_NOT_CONVERGED;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  const EnergyBufs E = energy_bufs(box, work);
  auto rd = [&](const double* d) {
    double h = 0;
    cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return h;
  };
  energy_start(E, box, VV_T, rhs, T, s);
  pdl_launch(k_bicg_init, 1, 1, 0, s, E.sc, rtol, maxit, cudaGraphConditionalHandle(0), 0);
  double bb = rd(E.sc + 10);
  double rr = rd(E.sc + 11);
  int it = 0;
  for (it = 1; it <= maxit && rr > rtol * rtol * bb; ++it) {
    energy_iteration(E, box, T, rtol, maxit, cudaGraphConditionalHandle(0), 0, s);
    rr = rd(E.sc + 11);
    if (!std::isfinite(rr)) break;
  }
  if (iters) *iters = it - 1;
  if (relres) *relres = std::sqrt(rr / bb);
  if (cudaGetLastError() != cudaSuccess) return MW_ERR_CUDA;
  return std::sqrt(rr / bb) <= rtol ? MW_OK : MW_ERR_NOT_CONVERGED;
}

}  // extern "C"

static bool energy_record(mw_box box, const double* VV_T, const double* rhs, double* T, double rtol, int maxit,
                          void* work, cudaStream_t s, cudaStream_t b) {
  const EnergyBufs E = energy_bufs(box, work);
  energy_start(E, box, VV_T, rhs, T, s);
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
