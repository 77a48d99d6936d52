// FP64 derived fields and reductions (sm_100a).
//
// Reference: compute_pressure_offset.py:12-66, compute_nodal_pressure.py:8-21,
// compute_strain_rate.py:51-73, compute_nodal_heat_flux.py:12-40, postprocessors.py:14-83 and
// :114-248, and the time-step rule of meeuuw.py:2112-2139.
//
// Node fields that the reference accumulates element by element are computed node-centrically:
// each node sums its (up to 4) incident elements in ascending element order, then divides by the
// count -- the reference's order, without atomics.  Global sums use a fixed two-level tree
// (deterministic, not the reference's sequential order).  The surface pressure offset's boundary
// sum runs sequentially in the reference's element order; the four boundary sums of Nu use one
// warp per side, lane-strided partial sums then a fixed warp-shuffle tree (deterministic, but not
// the reference's sequential order: values agree to round-off).
#include <cuda.h>

#include <mutex>

#include "common.cuh"

namespace mw {

// Scratch of mw_compute_nu_noalloc: 3 doubles per boundary (element, Gauss point) pair for at most
// MW_NU_NOALLOC_MAX_BOUNDARY_ELEMENTS boundary elements (2.25 MiB).  Every GPU that loads the
// library holds this array until the process exits.
static __device__ __align__(256) double g_nu_scratch[(size_t)MW_NU_NOALLOC_MAX_BOUNDARY_ELEMENTS * 3 * 3];

constexpr int RT = 256;   // reduction block size
constexpr int RB = 296;   // reduction blocks (2 x 148 SMs)

MW_D double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  v = 0.0;
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    v = lane < nw ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

MW_D double block_max(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  v = -1e308;
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    v = lane < nw ? sh[lane] : -1e308;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  }
  return v;
}

// ---- incident elements of Q2 lattice node (ix, iz), ascending, with the local node index ----
MW_D int q2_incident(const mw_box& b, int ix, int iz, int* ex, int* ez, int* kl) {
  int exs[2], ezs[2], nx = 0, nz = 0;
  if (ix & 1) exs[nx++] = ix >> 1;
  else { if (ix / 2 - 1 >= 0) exs[nx++] = ix / 2 - 1; if (ix / 2 < b.nelx) exs[nx++] = ix / 2; }
  if (iz & 1) ezs[nz++] = iz >> 1;
  else { if (iz / 2 - 1 >= 0) ezs[nz++] = iz / 2 - 1; if (iz / 2 < b.nelz) ezs[nz++] = iz / 2; }
  int n = 0;
  for (int a = 0; a < nz; ++a)
    for (int c = 0; c < nx; ++c) {
      int dx = ix - 2 * exs[c], dz = iz - 2 * ezs[a];
      int k;
      if (dz == 0) k = dx == 0 ? 0 : (dx == 1 ? 4 : 1);
      else if (dz == 1) k = dx == 0 ? 7 : (dx == 1 ? 8 : 5);
      else k = dx == 0 ? 3 : (dx == 1 ? 6 : 2);
      ex[n] = exs[c]; ez[n] = ezs[a]; kl[n] = k; ++n;
    }
  return n;
}

// Surface / volume pressure offset (compute_pressure_offset.py:206-238).
__global__ void k_poff_surface(mw_box b, const double* __restrict__ p, double* out) {
  if (threadIdx.x || blockIdx.x) return;
  double s = 0.0;
  const int ez = b.nelz - 1;                                   // top elements in element order
  for (int ex = 0; ex < b.nelx; ++ex)
    s += 0.5 * (p[q1_node(ex, ez, 2, b.nelx)] + p[q1_node(ex, ez, 3, b.nelx)]);
  out[0] = s / b.nelx;
}

__global__ void k_poff_volume_partial(mw_box b, const double* __restrict__ p, const double* __restrict__ NP,
                                      const double* __restrict__ JxWq, double* __restrict__ partial) {
  __shared__ double sh[32];
  __shared__ double N[36];
  for (int i = threadIdx.x; i < 36; i += blockDim.x) N[i] = NP[i];
  __syncthreads();
  const int64_t nq = (int64_t)b.nelx * b.nelz * 9;
  double acc = 0.0;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nq; g += (int64_t)gridDim.x * blockDim.x) {
    int64_t e = g / 9;
    int q = (int)(g % 9);
    int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
    double pq = N[q * 4] * p[q1_node(ex, ez, 0, b.nelx)];
    for (int k = 1; k < 4; ++k) pq += N[q * 4 + k] * p[q1_node(ex, ez, k, b.nelx)];
    acc += pq * JxWq[g];
  }
  double s = block_sum(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void k_final_sum(const double* __restrict__ partial, int n, double scale, double* out) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) out[0] = v * scale;
}

// q on V nodes from Q1 pressure, with the pressure offset removed first (meeuuw.py:1977, 2051).
__global__ void k_nodal_pressure(mw_box b, double* __restrict__ p, int64_t np, const double* __restrict__ offset,
                                 const double* __restrict__ NPn, double* __restrict__ q) {
  __shared__ double N[36];
  for (int i = threadIdx.x; i < 36; i += blockDim.x) N[i] = NPn[i];
  __syncthreads();
  const double off = offset ? offset[0] : 0.0;
  const int nnx = 2 * b.nelx + 1;
  const int64_t nn = (int64_t)nnx * (2 * b.nelz + 1);
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    int ex[4], ez[4], kl[4];
    int ne = q2_incident(b, (int)(n % nnx), (int)(n / nnx), ex, ez, kl);
    double acc = 0.0;
    for (int s = 0; s < ne; ++s) {
      double v = N[kl[s] * 4] * (p[q1_node(ex[s], ez[s], 0, b.nelx)] - off);
      for (int k = 1; k < 4; ++k) v += N[kl[s] * 4 + k] * (p[q1_node(ex[s], ez[s], k, b.nelx)] - off);
      acc += v;
    }
    q[n] = acc / ne;
  }
}

__global__ void k_sub_scalar(double* __restrict__ p, int64_t n, const double* __restrict__ offset) {
  const double off = offset[0];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] -= off;
}

// Gradients at a node of element e: jcbi arrays (nel, 9) may be NULL for a uniform box.
struct NodeJac { const double *j00, *j01, *j10, *j11; };

MW_D void node_grad(const mw_box& b, const NodeJac& J, const double* dNdr, const double* dNdt, int64_t e, int kl,
                    double* dx, double* dz) {
  double j00, j01, j10, j11;
  if (J.j00) { int64_t g = e * 9 + kl; j00 = J.j00[g]; j01 = J.j01[g]; j10 = J.j10[g]; j11 = J.j11[g]; }
  else { j00 = 2.0 / b.hx; j01 = 0.0; j10 = 0.0; j11 = 2.0 / b.hz; }
  for (int k = 0; k < 9; ++k) {
    dx[k] = j00 * dNdr[kl * 9 + k] + j01 * dNdt[kl * 9 + k];
    dz[k] = j10 * dNdr[kl * 9 + k] + j11 * dNdt[kl * 9 + k];
  }
}

// compute_nodal_strain_rate (compute_strain_rate.py:51-73) and compute_nodal_heat_flux
// (compute_nodal_heat_flux.py:12-40) share this node-centric loop.
__global__ void k_nodal_grad(mw_box b, int mode, const double* __restrict__ u, const double* __restrict__ w,
                             const double* __restrict__ hcond, const double* __restrict__ dNdr_n,
                             const double* __restrict__ dNdt_n, NodeJac J, double* __restrict__ o0,
                             double* __restrict__ o1, double* __restrict__ o2, double* __restrict__ o3) {
  __shared__ double R[81], T[81];
  for (int i = threadIdx.x; i < 81; i += blockDim.x) { R[i] = dNdr_n[i]; T[i] = dNdt_n[i]; }
  __syncthreads();
  const int nnx = 2 * b.nelx + 1;
  const int64_t nn = (int64_t)nnx * (2 * b.nelz + 1);
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    int ex[4], ez[4], kl[4];
    int ne = q2_incident(b, (int)(n % nnx), (int)(n / nnx), ex, ez, kl);
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (int s = 0; s < ne; ++s) {
      int64_t e = (int64_t)ez[s] * b.nelx + ex[s];
      double dx[9], dz[9];
      node_grad(b, J, R, T, e, kl[s], dx, dz);
      double xu = 0, zw = 0, xw = 0, zu = 0;
      for (int k = 0; k < 9; ++k) {
        int64_t m = q2_node(ex[s], ez[s], k, nnx);
        double uk = u[m];
        xu += dx[k] * uk; zu += dz[k] * uk;
        if (mode == 0) { double wk = w[m]; zw += dz[k] * wk; xw += dx[k] * wk; }
      }
      if (mode == 0) {                     // exx, ezz, exz
        a0 += xu; a1 += zw; a2 += 0.5 * xw + 0.5 * zu;
      } else {                             // -dT/dx, -dT/dz, -k dT/dx, -k dT/dz
        double hk = hcond[n];
        a0 -= xu; a1 -= zu; a2 -= hk * xu; a3 -= hk * zu;
      }
    }
    double c = (double)ne;
    o0[n] = a0 / c; o1[n] = a1 / c; o2[n] = a2 / c;
    if (mode == 1) o3[n] = a3 / c;
  }
}

// compute_Nu (postprocessors.py:114-248): per boundary element and Gauss point terms in parallel,
// then each side summed by one warp (lane-strided partials, fixed warp-shuffle tree).
__global__ void k_nu_terms(mw_box b, const double* __restrict__ T, const double* __restrict__ dTdx,
                           const double* __restrict__ dTdz, const double* __restrict__ hc, mw_gauss3 g,
                           double* __restrict__ terms) {
  // terms layout: side s (0 left, 1 right, 2 top, 3 bottom), element index along the side, qpoint,
  // 3 quantities (T, grad*n, -k*grad*n)
  const int nside[4] = {b.nelz, b.nelz, b.nelx, b.nelx};
  const int nnx = 2 * b.nelx + 1;
  const int64_t total = (int64_t)(2 * b.nelz + 2 * b.nelx) * 3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    int s = 0;
    while (r >= (int64_t)nside[s] * 3) { r -= (int64_t)nside[s] * 3; ++s; }
    int idx = (int)(r / 3), iq = (int)(r % 3);
    int ex, ez;
    double rq, tq, jcob, nsgn;
    const double* grad;
    if (s == 0) { ex = 0; ez = idx; rq = -1; tq = g.c[iq]; jcob = b.hz / 2; nsgn = -1; grad = dTdx; }
    else if (s == 1) { ex = b.nelx - 1; ez = idx; rq = +1; tq = g.c[iq]; jcob = b.hz / 2; nsgn = +1; grad = dTdx; }
    else if (s == 2) { ex = idx; ez = b.nelz - 1; rq = g.c[iq]; tq = +1; jcob = b.hx / 2; nsgn = +1; grad = dTdz; }
    else { ex = idx; ez = 0; rq = g.c[iq]; tq = -1; jcob = b.hx / 2; nsgn = -1; grad = dTdz; }
    // element side lengths exactly as the reference takes them from node coordinates (:154, 171, 188, 205)
    if (s == 0 || s == 1) jcob = ((double)(2 * ez + 2) * b.hz / 2 - (double)(2 * ez) * b.hz / 2) / 2;
    else jcob = ((double)(2 * ex + 2) * b.hx / 2 - (double)(2 * ex) * b.hx / 2) / 2;
    double N[9];
    q2_basis<double>(rq, tq, N);
    double Tq = 0, hq = 0, gq = 0;
    for (int k = 0; k < 9; ++k) {
      int64_t m = q2_node(ex, ez, k, nnx);
      Tq += N[k] * T[m]; hq += N[k] * hc[m]; gq += N[k] * grad[m];
    }
    double* o = terms + t * 3;
    o[0] = Tq * jcob * g.w[iq];
    o[1] = gq * jcob * g.w[iq] * nsgn;
    o[2] = hq * gq * jcob * g.w[iq] * nsgn;
  }
}

__global__ void k_nu_final(mw_box b, const double* __restrict__ terms, double* __restrict__ out) {
  // out: avrg_T_left, right, bottom, top, avrg_dTdx_left, right, avrg_dTdz_bottom, top,
  //      qx_left, qx_right, qz_bottom, qz_top, Nu     (postprocessors.py:234-248)
  // one warp per side: lane-strided partial sums, then a fixed-order warp reduction (deterministic)
  __shared__ double res[4][3];
  const int nside[4] = {b.nelz, b.nelz, b.nelx, b.nelx};
  const int s = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (s < 4) {
    int64_t off = 0;
    for (int k = 0; k < s; ++k) off += (int64_t)nside[k] * 3;
    double aT = 0, ag = 0, q = 0;
    for (int64_t t = off + lane; t < off + (int64_t)nside[s] * 3; t += 32) {
      aT += terms[t * 3]; ag += terms[t * 3 + 1]; q -= terms[t * 3 + 2];
    }
    for (int o = 16; o > 0; o >>= 1) {
      aT += __shfl_down_sync(0xffffffffu, aT, o);
      ag += __shfl_down_sync(0xffffffffu, ag, o);
      q += __shfl_down_sync(0xffffffffu, q, o);
    }
    if (lane == 0) { res[s][0] = aT; res[s][1] = ag; res[s][2] = q; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double aTl = res[0][0] / b.Lz, aTr = res[1][0] / b.Lz, aTt = res[2][0] / b.Lx, aTb = res[3][0] / b.Lx;
    double agl = res[0][1] / b.Lz, agr = res[1][1] / b.Lz, agt = res[2][1] / b.Lx, agb = res[3][1] / b.Lx;
    out[0] = aTl; out[1] = aTr; out[2] = aTb; out[3] = aTt;
    out[4] = agl; out[5] = agr; out[6] = agb; out[7] = agt;
    out[8] = res[0][2]; out[9] = res[1][2]; out[10] = res[3][2]; out[11] = res[2][2];
    out[12] = fabs(agt) / (aTb - aTt) * b.Lz;                                  // :232
  }
}

// vrms, Tavrg, total mass (postprocessors.py:53-78): two-level deterministic sums.
__global__ void k_global_partial(int64_t nq, const double* __restrict__ uq, const double* __restrict__ wq,
                                 const double* __restrict__ Tq, const double* __restrict__ rhoq,
                                 const double* __restrict__ JxWq, double* __restrict__ partial) {
  __shared__ double sh[32];
  double a = 0, t = 0, m = 0;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nq; g += (int64_t)gridDim.x * blockDim.x) {
    double jxw = JxWq[g];
    double u = uq[g], w = wq[g];
    a += (u * u + w * w) * jxw;
    if (Tq) t += Tq[g] * jxw;
    if (rhoq) m += rhoq[g] * jxw;
  }
  a = block_sum(a, sh);
  t = block_sum(t, sh);
  m = block_sum(m, sh);
  if (threadIdx.x == 0) { partial[blockIdx.x] = a; partial[gridDim.x + blockIdx.x] = t; partial[2 * gridDim.x + blockIdx.x] = m; }
}

__global__ void k_global_final(const double* __restrict__ partial, int nb, double volume, double* __restrict__ out) {
  __shared__ double sh[32];
  double a = 0, t = 0, m = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) { a += partial[i]; t += partial[nb + i]; m += partial[2 * nb + i]; }
  a = block_sum(a, sh);
  t = block_sum(t, sh);
  m = block_sum(m, sh);
  if (threadIdx.x == 0) { out[0] = sqrt(a / volume); out[1] = t / volume; out[2] = m; }
}

// The whole compute_global_quantities tuple (postprocessors.py:42-83): nine per-qpoint sums
// {TM, EK, WAG, TVD, ITE, vrms, Tavrg, num, denom} in two deterministic levels.  GPE stays 0 as
// in the reference (its line is commented out, :69).
struct GlobalFullIn {
  const double *uq, *wq, *Tq, *rhoq, *hcapaq, *etaq, *exxq, *ezzq, *exzq, *gxq, *gzq, *JxWq;
};

__global__ void k_global_full_partial(int64_t nq, GlobalFullIn in, double* __restrict__ partial) {
  __shared__ double sh[32];
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nq; g += (int64_t)gridDim.x * blockDim.x) {
    const double jxw = in.JxWq[g], u = in.uq[g], w = in.wq[g], rho = in.rhoq[g], T = in.Tq[g];
    const double exx = in.exxq[g], ezz = in.ezzq[g], exz = in.exzq[g], eta = in.etaq[g];
    const double eII = exx * exx + ezz * ezz + 2 * exz * exz;
    acc[0] += rho * jxw;
    acc[1] += 0.5 * rho * (u * u + w * w) * jxw;
    acc[2] -= rho * (u * in.gxq[g] + w * in.gzq[g]) * jxw;
    acc[3] += 2 * eta * (2 * exx * exx / 3 + 2 * ezz * ezz / 3 - 2 * exx * ezz / 3 + 2 * exz * exz) * jxw;
    acc[4] += rho * in.hcapaq[g] * T * jxw;
    acc[5] += (u * u + w * w) * jxw;
    acc[6] += T * jxw;
    acc[7] += eta * eII * jxw;
    acc[8] += eII * jxw;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double v = block_sum(acc[k], sh);
    if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = v;
  }
}

// out9 = {vrms, EK, WAG, TVD, GPE, ITE, TM, Tavrg, eta_avrg}; eta_avrg is NaN when the strain-rate
// sum is zero (the reference leaves it unassigned then)
__global__ void k_global_full_final(const double* __restrict__ partial, int nb, double volume, double* __restrict__ out) {
  __shared__ double sh[32];
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double a = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) a += partial[k * nb + i];
    acc[k] = block_sum(a, sh);
  }
  if (threadIdx.x == 0) {
    out[0] = sqrt(acc[5] / volume);
    out[1] = acc[1];
    out[2] = acc[2];
    out[3] = acc[3];
    out[4] = 0.0;
    out[5] = acc[4];
    out[6] = acc[0];
    out[7] = acc[6] / volume;
    out[8] = acc[8] > 0 ? acc[7] / acc[8] : __longlong_as_double(0x7ff8000000000000LL);
  }
}

// Time step (meeuuw.py:2112-2139): max |v| over V nodes and the particle means of hcond,
// hcapa, rho.  state = {dt1_mem, dt2_mem}; out = {dt, dt1, dt2}.
__global__ void k_dt_partial(int64_t nn, const double* __restrict__ u, const double* __restrict__ w, int64_t np,
                             const double* __restrict__ hk, const double* __restrict__ hc,
                             const double* __restrict__ rho, double* __restrict__ partial) {
  __shared__ double sh[32];
  double vmax = 0.0, a = 0, bsum = 0, c = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x)
    vmax = fmax(vmax, sqrt(u[i] * u[i] + w[i] * w[i]));
  if (hk)
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
      a += hk[i]; bsum += hc[i]; c += rho[i];
    }
  vmax = block_max(vmax, sh);
  a = block_sum(a, sh);
  bsum = block_sum(bsum, sh);
  c = block_sum(c, sh);
  if (threadIdx.x == 0) {
    int B = gridDim.x;
    partial[blockIdx.x] = vmax; partial[B + blockIdx.x] = a; partial[2 * B + blockIdx.x] = bsum;
    partial[3 * B + blockIdx.x] = c;
  }
}

__global__ void k_dt_final(const double* __restrict__ partial, int nb, int64_t np, mw_dt_params prm, double* state,
                           double* __restrict__ out) {
  __shared__ double sh[32];
  double vmax = 0.0, a = 0, bsum = 0, c = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    vmax = fmax(vmax, partial[i]); a += partial[nb + i]; bsum += partial[2 * nb + i]; c += partial[3 * nb + i];
  }
  vmax = block_max(vmax, sh);
  a = block_sum(a, sh);
  bsum = block_sum(bsum, sh);
  c = block_sum(c, sh);
  if (threadIdx.x == 0) {
    double h = fmin(prm.hx, prm.hz);
    double dt1 = prm.CFLnb * h / vmax;
    double dt2 = 1e50;
    if (prm.solve_T) {
      double kappa = (a / np) / (bsum / np) / (c / np);
      dt2 = prm.CFLnb * h * h / kappa;
    }
    dt1 = fmin(dt1, 1.25 * state[0]);
    dt2 = fmin(dt2, 1.25 * state[1]);
    double dt = fmin(fmin(dt1, dt2), prm.dt_max);
    state[0] = dt1; state[1] = dt2;
    out[0] = dt; out[1] = dt1; out[2] = dt2;
  }
}

// Split the Stokes solution: u, w from interleaved solV and p = solP * eta_ref/L_ref
// (meeuuw.py:1846-1851).
__global__ void k_split(int64_t nn, int64_t np, const double* __restrict__ solV, const double* __restrict__ solP,
                        double scale, double* __restrict__ u, double* __restrict__ w, double* __restrict__ p) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
    u[i] = solV[2 * i];
    w[i] = solV[2 * i + 1];
    if (i < np) p[i] = solP[i] * scale;
  }
}

// rhoq / etaq of the "elemental" projection (meeuuw.py:1512-1514, 1545-1547): phiq[e, :] = phi_e[e]
__global__ void k_broadcast_q(int64_t nel, const double* __restrict__ a, const double* __restrict__ b,
                              double* __restrict__ aq, double* __restrict__ bq) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nel * 9; g += (int64_t)gridDim.x * blockDim.x) {
    aq[g] = a[g / 9];
    if (b) bq[g] = b[g / 9];
  }
}

}  // namespace mw

using namespace mw;

extern "C" {

int mw_split_solution(int64_t nn_V, int64_t nn_P, const double* solV, const double* solP, double scale, double* u,
                      double* w, double* p, void* stream) {
  int64_t n = nn_V > nn_P ? nn_V : nn_P;
  k_split<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(nn_V, nn_P, solV, solP, scale, u, w, p);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_elemental_to_qpoints(int64_t nel, const double* a, const double* b, double* aq, double* bq, void* stream) {
  k_broadcast_q<<<grid_for(nel * 9, 256), 256, 0, (cudaStream_t)stream>>>(nel, a, b, aq, bq);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

size_t mw_post_workspace_bytes(void) { return (size_t)9 * RB * sizeof(double) + 64; }

int mw_pressure_offset(mw_box box, int32_t normalisation, const double* p, const double* N_P, const double* JxWq,
                       double volume, double* offset, void* work, size_t work_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (normalisation == MW_PNORM_NONE) {
    return cudaMemsetAsync(offset, 0, sizeof(double), s) == cudaSuccess ? MW_OK : MW_ERR_CUDA;
  }
  if (normalisation == MW_PNORM_SURFACE) {
    k_poff_surface<<<1, 32, 0, s>>>(box, p, offset);
    MW_CHECK_LAUNCH();
    return MW_OK;
  }
  if (normalisation != MW_PNORM_VOLUME || !N_P || !JxWq) return MW_ERR_BAD_ARG;
  if (work_bytes < mw_post_workspace_bytes()) return MW_ERR_WORKSPACE;
  double* part = (double*)work;
  k_poff_volume_partial<<<RB, RT, 0, s>>>(box, p, N_P, JxWq, part);
  MW_CHECK_LAUNCH();
  k_final_sum<<<1, RT, 0, s>>>(part, RB, 1.0 / volume, offset);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_nodal_pressure(mw_box box, double* p, const double* offset, int32_t subtract_in_place, const double* N_P_n,
                      double* q, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  int64_t np = (int64_t)(box.nelx + 1) * (box.nelz + 1);
  if (q) {
    k_nodal_pressure<<<grid_for(nn, 256), 256, 0, s>>>(box, p, np, offset, N_P_n, q);
    MW_CHECK_LAUNCH();
  }
  if (subtract_in_place && offset) {
    k_sub_scalar<<<grid_for(np, 256), 256, 0, s>>>(p, np, offset);
    MW_CHECK_LAUNCH();
  }
  return MW_OK;
}

int mw_nodal_strain_rate(mw_box box, const double* u, const double* w, const double* dNdr_V_n,
                         const double* dNdt_V_n, const double* jcbi00n, const double* jcbi01n, const double* jcbi10n,
                         const double* jcbi11n, double* exx_n, double* ezz_n, double* exz_n, void* stream) {
  int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  NodeJac J{jcbi00n, jcbi01n, jcbi10n, jcbi11n};
  k_nodal_grad<<<grid_for(nn, 128), 128, 0, (cudaStream_t)stream>>>(box, 0, u, w, nullptr, dNdr_V_n, dNdt_V_n, J,
                                                                       exx_n, ezz_n, exz_n, nullptr);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_nodal_heat_flux(mw_box box, const double* T, const double* hcond_n, const double* dNdr_T_n,
                       const double* dNdt_T_n, const double* jcbi00, const double* jcbi01, const double* jcbi10,
                       const double* jcbi11, double* dTdx_n, double* dTdz_n, double* qx_n, double* qz_n,
                       void* stream) {
  int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  NodeJac J{jcbi00, jcbi01, jcbi10, jcbi11};
  k_nodal_grad<<<grid_for(nn, 128), 128, 0, (cudaStream_t)stream>>>(box, 1, T, nullptr, hcond_n, dNdr_T_n, dNdt_T_n,
                                                                       J, dTdx_n, dTdz_n, qx_n, qz_n);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

size_t mw_nu_workspace_bytes(mw_box box) { return (size_t)(2 * box.nelx + 2 * box.nelz) * 9 * sizeof(double); }

int mw_compute_nu(mw_box box, const double* T, const double* dTdx_n, const double* dTdz_n, const double* hcond_n,
                  mw_gauss3 g, double* out13, void* work, size_t work_bytes, void* stream) {
  if (work_bytes < mw_nu_workspace_bytes(box)) return MW_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  int64_t total = (int64_t)(2 * box.nelz + 2 * box.nelx) * 3;
  k_nu_terms<<<grid_for(total, 128), 128, 0, s>>>(box, T, dTdx_n, dTdz_n, hcond_n, g, (double*)work);
  MW_CHECK_LAUNCH();
  k_nu_final<<<1, 128, 0, s>>>(box, (const double*)work, out13);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

// Device address of g_nu_scratch for the calling thread's current context (host code cannot use the
// symbol itself as a device pointer).  The address belongs to the context the module was loaded
// into, so it is cached per context, keyed by the context's process-unique id (cuCtxGetId): after a
// cudaDeviceReset, or under another context on the same device, the address is looked up again.
// The two driver calls are resolved through the runtime (no link-time dependency on libcuda).
typedef CUresult (*PFN_ctx_get_current)(CUcontext*);
typedef CUresult (*PFN_ctx_get_id)(CUcontext, unsigned long long*);

static void* driver_fn(const char* name) {
  cudaDriverEntryPointQueryResult q;
  void* p = nullptr;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return nullptr;
  return p;
}

static double* nu_scratch_for_current_context(int* status) {
  static std::mutex mtx;
  struct Entry { unsigned long long id; double* addr; };
  static Entry cache[64] = {};
  static int used = 0, next = 0;
  static PFN_ctx_get_current ctx_get_current = nullptr;
  static PFN_ctx_get_id ctx_get_id = nullptr;
  *status = MW_ERR_CUDA;
  std::lock_guard<std::mutex> lock(mtx);
  if (!ctx_get_current || !ctx_get_id) {
    ctx_get_current = (PFN_ctx_get_current)driver_fn("cuCtxGetCurrent");
    ctx_get_id = (PFN_ctx_get_id)driver_fn("cuCtxGetId");
    if (!ctx_get_current || !ctx_get_id) return nullptr;
  }
  CUcontext ctx = nullptr;
  CUresult cr = ctx_get_current(&ctx);
  if (cr != CUDA_SUCCESS && cr != CUDA_ERROR_NOT_INITIALIZED) return nullptr;
  unsigned long long id = 0;
  if (ctx) {
    if (ctx_get_id(ctx, &id) != CUDA_SUCCESS) return nullptr;
    for (int i = 0; i < used; ++i)
      if (cache[i].id == id) { *status = MW_OK; return cache[i].addr; }
  }
  // set-up: the runtime makes the current device's primary context current if none is, and loads
  // this file's module (with g_nu_scratch) if it is not loaded yet
  double* p = nullptr;
  if (cudaGetSymbolAddress((void**)&p, g_nu_scratch) != cudaSuccess || !p) return nullptr;
  if (!ctx) {
    if (ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx || ctx_get_id(ctx, &id) != CUDA_SUCCESS) return nullptr;
  }
  cache[next] = Entry{id, p};
  next = (next + 1) % 64;
  if (used < 64) ++used;
  *status = MW_OK;
  return p;
}

int mw_compute_nu_noalloc(mw_box box, const double* T, const double* dTdx_n, const double* dTdz_n,
                          const double* hcond_n, mw_gauss3 g, double* out13, void* stream) {
  if (box.nelx <= 0 || box.nelz <= 0 || !T || !dTdx_n || !dTdz_n || !hcond_n || !out13) return MW_ERR_BAD_ARG;
  const int64_t nbound = 2LL * box.nelx + 2LL * box.nelz;
  if (nbound > MW_NU_NOALLOC_MAX_BOUNDARY_ELEMENTS) return MW_ERR_TOO_LARGE;
  int st = MW_OK;
  double* scratch = nu_scratch_for_current_context(&st);
  if (st != MW_OK) return st;
  // every scratch slot the final sum reads is written by k_nu_terms first: nothing to clear
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t total = nbound * 3;
  k_nu_terms<<<grid_for(total, 128), 128, 0, s>>>(box, T, dTdx_n, dTdz_n, hcond_n, g, scratch);
  MW_CHECK_LAUNCH();
  k_nu_final<<<1, 128, 0, s>>>(box, scratch, out13);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_global_quantities(int64_t nq, const double* uq, const double* wq, const double* Tq, const double* rhoq,
                         const double* JxWq, double volume, double* out3, void* work, size_t work_bytes,
                         void* stream) {
  if (work_bytes < mw_post_workspace_bytes()) return MW_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  double* part = (double*)work;
  k_global_partial<<<RB, RT, 0, s>>>(nq, uq, wq, Tq, rhoq, JxWq, part);
  MW_CHECK_LAUNCH();
  k_global_final<<<1, RT, 0, s>>>(part, RB, volume, out3);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_global_quantities_full(int64_t nq, const double* uq, const double* wq, const double* Tq, const double* rhoq,
                              const double* hcapaq, const double* etaq, const double* exxq, const double* ezzq,
                              const double* exzq, const double* gxq, const double* gzq, const double* JxWq,
                              double volume, double* out9, void* work, size_t work_bytes, void* stream) {
  if (work_bytes < mw_post_workspace_bytes()) return MW_ERR_WORKSPACE;
  if (!uq || !wq || !Tq || !rhoq || !hcapaq || !etaq || !exxq || !ezzq || !exzq || !gxq || !gzq || !JxWq)
    return MW_ERR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  double* part = (double*)work;
  GlobalFullIn in{uq, wq, Tq, rhoq, hcapaq, etaq, exxq, ezzq, exzq, gxq, gzq, JxWq};
  k_global_full_partial<<<RB, RT, 0, s>>>(nq, in, part);
  MW_CHECK_LAUNCH();
  k_global_full_final<<<1, RT, 0, s>>>(part, RB, volume, out9);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_compute_dt(int64_t nn_V, const double* u, const double* w, int64_t nparticle, const double* swarm_hcond,
                  const double* swarm_hcapa, const double* swarm_rho, mw_dt_params prm, double* state2,
                  double* out3, void* work, size_t work_bytes, void* stream) {
  if (work_bytes < mw_post_workspace_bytes()) return MW_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  double* part = (double*)work;
  const double* hk = prm.solve_T ? swarm_hcond : nullptr;
  k_dt_partial<<<RB, RT, 0, s>>>(nn_V, u, w, nparticle, hk, swarm_hcapa, swarm_rho, part);
  MW_CHECK_LAUNCH();
  k_dt_final<<<1, RT, 0, s>>>(part, RB, nparticle, prm, state2, out3);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

}  // extern "C"
