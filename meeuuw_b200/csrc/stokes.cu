// Matrix-free Q2xQ1 Stokes operator, geometric-multigrid PCG for the velocity block, and the
// Uzawa (Schur-complement PCG) outer solver -- all on the device (sm_100a).
//
// Reference: the operator is the one assembled by build_matrix_stokes.py:18-278 (K, G with the
// Dirichlet elimination of :206-217); the outer scheme is uzawa3_solver_L2.py:21-99 and its
// M_eta-preconditioned form cd_u_eta.py:13-99; the reference solves K with SuperLU (splu), here
// K^-1 is a multigrid-preconditioned conjugate gradient run on the device.
//
// Operator tiles: a CTA owns a TX x TZ tile of elements' nodes; it recomputes a one-element halo
// on its left/bottom so that every owned node sums all its incident elements itself, in
// ascending element order, from shared memory.  No atomics, deterministic results.  The element
// kernel evaluates K u, G p, G^T u at the 3x3 Gauss points from the viscosity at the qpoints and
// the uniform-box Jacobian (no stored element matrices).
//
// Dirichlet semantics (identical to SpMV with the reference's eliminated COO): fixed velocity
// dofs are zeroed before the element products; fixed rows return diag(K)_i * u_i; G rows of
// fixed dofs are zero.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "q2_ref.cuh"

namespace mw {

// ---------------------------------------------------------------- reference-element tables
__constant__ RefTables c_ref;
static bool g_ref_ready = false;

// FP32 kernels take the values as immediates; FP64 ones read them from the constant bank (an FP64
// immediate would be materialised in registers for every use).  Which terms vanish is decided at
// compile time in both cases (ref_dr / ref_dt of q2_ref.cuh).
template <typename R> struct CT {
  MW_D static constexpr R dr(int q, int k) { return (R)ref_dr(q, k); }
  MW_D static constexpr R dt(int q, int k) { return (R)ref_dt(q, k); }
  MW_D static constexpr R np(int q, int k) { return (R)ref_np(q, k); }
  MW_D static constexpr R wq(int q) { return (R)ref_wq(q); }
};
template <> struct CT<double> {
  MW_D static double dr(int q, int k) { return c_ref.dr[q * 9 + k]; }
  MW_D static double dt(int q, int k) { return c_ref.dt[q * 9 + k]; }
  MW_D static double np(int q, int k) { return c_ref.NP[q * 4 + k]; }
  MW_D static double wq(int q) { return c_ref.wq[q]; }
};

static int ensure_ref_tables() {
  if (g_ref_ready) return MW_OK;
  RefTables T;
  host_ref_tables(&T);
  if (cudaMemcpyToSymbol(c_ref, &T, sizeof(T)) != cudaSuccess) return MW_ERR_CUDA;
  g_ref_ready = true;
  return MW_OK;
}

// ---------------------------------------------------------------- level geometry
struct LevelGeo {
  int nx, nz;        // elements
  int nnx, nnz;      // Q2 lattice nodes
  double hx, hz;
  double s;          // G scaling eta_ref / L_ref (build_matrix_stokes.py:157)
};

constexpr int TX = 16, TZ = 8;                 // owned element tile
constexpr int EX = TX + 1, EZ = TZ + 1;        // with the left/bottom halo
constexpr int NEL_T = EX * EZ;                 // 153 element computations per CTA
constexpr int LX = 2 * TX + 3, LZ = 2 * TZ + 3;// staged lattice nodes (35 x 19)
constexpr int PX = TX + 2, PZ = TZ + 2;        // staged pressure nodes (18 x 10)
constexpr int APPLY_THREADS = 160;

// AM_CHEB_Z: the second Chebyshev step of a sweep from a zero guess with the first one folded in:
// the velocity staged is x0 = (1/theta) D^-1 b (the first step's x and d), computed on the fly
// AM_CHEB_P: the first Chebyshev step after the coarse-grid correction with the prolongation folded
// in: the velocity staged is x + P x_c (free dofs), computed from a staged tile of the coarse
// correction with the taps and rounding of k_prolong_add, so the V-cycle needs no prolongation launch.
enum ApplyMode { AM_APPLY = 0, AM_RESID = 1, AM_CHEB = 2, AM_CHEB_Z = 3, AM_CHEB_P = 4 };

template <typename R> struct Vec2;
template <> struct Vec2<float> { typedef float2 T; };
template <> struct Vec2<double> { typedef double2 T; };

template <typename R>
struct ApplyArgs {
  const R* u;        // velocity (interleaved u,w), may be null
  const R* p;        // pressure, may be null
  const R* eta;      // (nel, 9)
  const uint8_t* fix;// (2*nn)
  const R* diag;     // (2*nn) assembled diag(K)
  R* yV;             // output velocity part (AM_APPLY: K u + G p; AM_RESID: b - (...))
  R* yP;             // output pressure part: G^T u (AM_RESID: h - G^T u); may be null
  const R* bV;       // rhs for residual / Chebyshev
  const R* bP;
  // Chebyshev: d = c1*d + c2*Dinv*r; xo = x + d   (x = u)
  R* d;
  R* xo;
  const double* cheb; // device coefficients {c1, c2}
  const double* cheb0;// AM_CHEB_Z: the first step's pair {0, 1/theta}
  const R* xc;        // AM_CHEB_P: the coarse correction (interleaved u, w) ...
  LevelGeo gc;        // ... on this coarse level
};

// Element contribution of K u_el + G p_el and G^T u_el at the 9 Gauss points: strain rate B u
// at each point, stress 2 eta (exx, ezz) and eta (du/dz + dw/dx) with the pressure term, then B^T
// back onto the nodes (build_matrix_stokes.py:130-157 applied to a vector).  The reference-element
// tables are __constant__ and every loop is unrolled, so each table value is an immediate
// constant-bank operand of the FMA; the uniform-box Jacobian enters as sx = 2/hx, sz = 2/hz.
// HAS_U = false: no velocity (G p only; the strain-rate terms vanish).  NEED_V = false: only the
// pressure rows are wanted (G^T u), so the B^T scatter and the shear gradients are skipped.
template <typename R, bool HAS_U = true, bool NEED_V = true>
MW_D void element_apply(R sx, R sz, R jac, R s, const R* ue, const R* pe, const R* eq, R* ye, R* ype, bool use_p) {
#pragma unroll
  for (int k = 0; k < 18; ++k) ye[k] = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) ype[k] = 0;
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    R dxu = 0, dzw = 0, dzu = 0, dxw = 0;
    if (HAS_U) {
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const R r = CT<R>::dr(q, k), t = CT<R>::dt(q, k);
        if (ref_dr(q, k) != 0.0) { dxu += r * ue[2 * k]; if (NEED_V) dxw += r * ue[2 * k + 1]; }
        if (ref_dt(q, k) != 0.0) { dzw += t * ue[2 * k + 1]; if (NEED_V) dzu += t * ue[2 * k]; }
      }
    }
    const R exx = sx * dxu, ezz = sz * dzw, gg = sz * dzu + sx * dxw;   // gg = du/dz + dw/dx
    const R jw = jac * CT<R>::wq(q);
    if (NEED_V) {
      const R e = eq[q] * jw;
      R pq = 0;
      if (use_p) {
#pragma unroll
        for (int k = 0; k < 4; ++k) pq += CT<R>::np(q, k) * pe[k];
      }
      const R sp = s * jw * pq;
      const R A = (R(2) * e * exx - sp) * sx, B = (R(2) * e * ezz - sp) * sz;
      const R Cx = e * gg * sx, Cz = e * gg * sz;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const R r = CT<R>::dr(q, k), t = CT<R>::dt(q, k);
        if (ref_dr(q, k) != 0.0) { ye[2 * k] += r * A; if (HAS_U) ye[2 * k + 1] += r * Cx; }
        if (ref_dt(q, k) != 0.0) { if (HAS_U) ye[2 * k] += t * Cz; ye[2 * k + 1] += t * B; }
      }
    }
    if (HAS_U) {
      const R dv = -s * jw * (exx + ezz);
#pragma unroll
      for (int k = 0; k < 4; ++k) ype[k] += CT<R>::np(q, k) * dv;
    }
  }
}

// FP32 variant on the packed two-lane FMA of sm_100 (__ffma2_rn): a node's (u, w) pair is one
// operand, so each nonzero basis value costs one instruction for both velocity components, in the
// gradients and in the B^T scatter.
template <>
MW_D void element_apply<float, true, true>(float sx, float sz, float jac, float s, const float* ue, const float* pe,
                                           const float* eq, float* ye, float* ype, bool use_p) {
  const float2* u2 = reinterpret_cast<const float2*>(ue);
  float2 y2[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) y2[k] = make_float2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 4; ++k) ype[k] = 0.f;
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    float2 gx = make_float2(0.f, 0.f), gz = make_float2(0.f, 0.f);   // (du/dr, dw/dr), (du/dt, dw/dt)
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float r = CT<float>::dr(q, k), t = CT<float>::dt(q, k);
      if (r != 0.f) gx = __ffma2_rn(make_float2(r, r), u2[k], gx);
      if (t != 0.f) gz = __ffma2_rn(make_float2(t, t), u2[k], gz);
    }
    const float exx = sx * gx.x, ezz = sz * gz.y, gg = sz * gz.x + sx * gx.y;
    const float jw = jac * CT<float>::wq(q);
    const float e = eq[q] * jw;
    float pq = 0.f;
    if (use_p) {
#pragma unroll
      for (int k = 0; k < 4; ++k) pq += CT<float>::np(q, k) * pe[k];
    }
    const float sp = s * jw * pq;
    const float2 ar = make_float2((2.f * e * exx - sp) * sx, e * gg * sx);   // coefficients of dN/dr
    const float2 at = make_float2(e * gg * sz, (2.f * e * ezz - sp) * sz);   // coefficients of dN/dt
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float r = CT<float>::dr(q, k), t = CT<float>::dt(q, k);
      if (r != 0.f) y2[k] = __ffma2_rn(make_float2(r, r), ar, y2[k]);
      if (t != 0.f) y2[k] = __ffma2_rn(make_float2(t, t), at, y2[k]);
    }
    const float dv = -s * jw * (exx + ezz);
#pragma unroll
    for (int k = 0; k < 4; ++k) ype[k] += CT<float>::np(q, k) * dv;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    ye[2 * k] = y2[k].x;
    ye[2 * k + 1] = y2[k].y;
  }
}

// local Q2 node index of lattice offset (dx, dz)
MW_D int q2_local_idx(int dx, int dz) {
  if (dz == 0) return dx == 0 ? 0 : (dx == 1 ? 4 : 1);
  if (dz == 1) return dx == 0 ? 7 : (dx == 1 ? 8 : 5);
  return dx == 0 ? 3 : (dx == 1 ? 6 : 2);
}

// ---------------------------------------------------------------- G and G^T as node stencils
// On the uniform box every element's G block is the same 18 x 4 matrix, G_el[2k][j] = cx GX[k][j],
// G_el[2k+1][j] = cz GZ[k][j] with cx = -s (hx hz / 4)(2 / hx), cz likewise (the pressure terms
// of build_matrix_stokes.py:130-157: -s B^T N_P JxW summed over the Gauss points), so the
// Schur-complement iteration's G p and G^T u need no element products: each node gathers its
// incident elements' entries in ascending element order.  Fixed velocity dofs: zero rows of G,
// zeroed entries of u for G^T (the reference's Dirichlet elimination).
// G p at velocity node (ix, iz) (f - G p with b): gx, gz are the GX, GZ tables, cx, cz the scalings.
MW_D void grad_node(const LevelGeo& g, const double* p, const uint8_t* fix, const double* b, double* y, int ix,
                    int iz, const double* gx, const double* gz, double cx, double cz) {
  const int64_t n = (int64_t)iz * g.nnx + ix;
  const bool xo = ix & 1, zo = iz & 1;
  const int xa = xo ? (ix >> 1) : (ix >> 1) - 1, xb = ix >> 1;
  const int za = zo ? (iz >> 1) : (iz >> 1) - 1, zb = iz >> 1;
  const int exs[2] = {xa, xb}, ezs[2] = {za, zb};
  const bool vx[2] = {xa >= 0, !xo && xb < g.nx}, vz[2] = {za >= 0, !zo && zb < g.nz};
  double ax = 0.0, az = 0.0;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      if (!vz[a] || !vx[c]) continue;
      const int ex = exs[c], ez = ezs[a];
      const int k = q2_local_idx(ix - 2 * ex, iz - 2 * ez);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double pv = p[q1_node(ex, ez, j, g.nx)];
        ax += gx[k * 4 + j] * pv;
        az += gz[k * 4 + j] * pv;
      }
    }
  const uchar2 ff = reinterpret_cast<const uchar2*>(fix)[n];
  double2 r{ff.x ? 0.0 : cx * ax, ff.y ? 0.0 : cz * az};
  if (b) {
    const double2 bb = reinterpret_cast<const double2*>(b)[n];
    r = double2{bb.x - r.x, bb.y - r.y};
  }
  reinterpret_cast<double2*>(y)[n] = r;
}

// G^T u at pressure node (px, pz)
MW_D double div_node(const LevelGeo& g, const double* u, const uint8_t* fix, int px, int pz, const double* gx,
                     const double* gz, double cx, double cz) {
  const double2* u2 = reinterpret_cast<const double2*>(u);
  const uchar2* f2 = reinterpret_cast<const uchar2*>(fix);
  // incident elements in ascending order and this node's Q1 index in each
  const int exs[4] = {px - 1, px, px - 1, px}, ezs[4] = {pz - 1, pz - 1, pz, pz}, js[4] = {2, 3, 1, 0};
  double acc = 0.0;
#pragma unroll 1
  for (int e = 0; e < 4; ++e) {
    const int ex = exs[e], ez = ezs[e], j = js[e];
    if (ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
    double sx = 0.0, sz = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const int64_t m = q2_node(ex, ez, k, g.nnx);
      const double2 uu = u2[m];
      const uchar2 ff = f2[m];
      sx += gx[k * 4 + j] * (ff.x ? 0.0 : uu.x);
      sz += gz[k * 4 + j] * (ff.y ? 0.0 : uu.y);
    }
    acc += cx * sx + cz * sz;
  }
  return acc;
}

// the element scalings of G: cx = -s (hx hz / 4)(2 / hx), cz = -s (hx hz / 4)(2 / hz)
MW_D void grad_scales(const LevelGeo& g, double* cx, double* cz) {
  const double jac = g.hx * g.hz / 4.0;
  *cx = -g.s * jac * (2.0 / g.hx);
  *cz = -g.s * jac * (2.0 / g.hz);
}

__global__ void k_grad_p(LevelGeo g, const double* __restrict__ p, const uint8_t* __restrict__ fix,
                         const double* __restrict__ b, double* __restrict__ y) {
  pdl_entry();
  __shared__ double gx[36], gz[36];
  if (threadIdx.x < 36) {
    gx[threadIdx.x] = c_ref.GX[threadIdx.x];
    gz[threadIdx.x] = c_ref.GZ[threadIdx.x];
  }
  __syncthreads();
  double cx, cz;
  grad_scales(g, &cx, &cz);
  // one lattice row per blockIdx.y: no index division
  for (int iz = blockIdx.y; iz < g.nnz; iz += gridDim.y)
    for (int ix = blockIdx.x * blockDim.x + threadIdx.x; ix < g.nnx; ix += gridDim.x * blockDim.x)
      grad_node(g, p, fix, b, y, ix, iz, gx, gz, cx, cz);
}

__global__ void k_div_u(LevelGeo g, const double* __restrict__ u, const uint8_t* __restrict__ fix,
                        double* __restrict__ y) {
  pdl_entry();
  __shared__ double gx[36], gz[36];
  if (threadIdx.x < 36) {
    gx[threadIdx.x] = c_ref.GX[threadIdx.x];
    gz[threadIdx.x] = c_ref.GZ[threadIdx.x];
  }
  __syncthreads();
  double cx, cz;
  grad_scales(g, &cx, &cz);
  const int ncx = g.nx + 1;
  // one pressure-node row per blockIdx.y: no index division
  for (int pz = blockIdx.y; pz <= g.nz; pz += gridDim.y)
    for (int px = blockIdx.x * blockDim.x + threadIdx.x; px < ncx; px += gridDim.x * blockDim.x)
      y[(int64_t)pz * ncx + px] = div_node(g, u, fix, px, pz, gx, gz, cx, cz);
}

// 1D Q2 prolongation: fine node i from coarse nodes
MW_D int pw(int i, int* J, double* w) {
  if (!(i & 1)) { J[0] = i / 2; w[0] = 1.0; return 1; }
  int E = i / 4;
  J[0] = 2 * E; J[1] = 2 * E + 1; J[2] = 2 * E + 2;
  if ((i & 3) == 1) { w[0] = 0.375; w[1] = 0.75; w[2] = -0.125; }
  else { w[0] = -0.125; w[1] = 0.75; w[2] = 0.375; }
  return 3;
}

// (P x_c) at fine lattice node (ix, iz): the taps summed in double in a fixed order (z outer, x
// inner) with explicit fused multiply-adds, so every path that prolongs (the prolongation kernel,
// the cluster tail, the Chebyshev step with the prolongation folded in) rounds alike.
// coarse(Jz, Jx) returns the coarse node's (u, w) pair.
template <typename V>
MW_D void prolong_taps(int ix, int iz, const V& coarse, double* s0, double* s1) {
  int Jx[3] = {0, 0, 0}, Jz[3] = {0, 0, 0};
  double wx[3] = {0, 0, 0}, wz[3] = {0, 0, 0};
  const int nxw = pw(ix, Jx, wx), nzw = pw(iz, Jz, wz);
  double a0 = 0, a1 = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
      if (a < nzw && b < nxw) {
        const auto v = coarse(Jz[a], Jx[b]);
        const double w = wz[a] * wx[b];
        a0 = fma(w, (double)v.x, a0);
        a1 = fma(w, (double)v.y, a1);
      }
  *s0 = a0;
  *s1 = a1;
}

// Levels whose element count is odd coarsen onto a uniform grid of ceil(n/2) elements over the same
// box (element size n h / ceil(n/2)), which is not nested in the fine one.  The prolongation
// there evaluates the coarse Q2 function at each fine node: fine lattice node i (position
// i L / (2 nf)) lies in coarse element E = floor(i nc / (2 nf)) (the last one at the far end) at
// local coordinate xi = (i nc - 2 nf E - nf) / nf, and takes the 1D Q2 basis values
// xi (xi - 1) / 2, (1 - xi)(1 + xi), xi (xi + 1) / 2 of coarse nodes 2E, 2E + 1, 2E + 2; the
// restriction is its exact transpose.  Nested dimensions (nf = 2 nc) keep the taps above.
MW_HD bool nested_1d(int nf, int nc) { return nf == 2 * nc; }
MW_HD bool nested_levels(const LevelGeo& gf, const LevelGeo& gc) {
  return nested_1d(gf.nx, gc.nx) && nested_1d(gf.nz, gc.nz);
}

MW_D int q2_weights_1d(int i, int nf, int nc, double* w) {
  int E = (int)(((int64_t)i * nc) / (2LL * nf));
  if (E > nc - 1) E = nc - 1;
  const double xi = (double)((int64_t)i * nc - 2LL * nf * E - nf) / (double)nf;
  w[0] = 0.5 * xi * (xi - 1.0);
  w[1] = (1.0 - xi) * (1.0 + xi);
  w[2] = 0.5 * xi * (xi + 1.0);
  return E;
}

// 1D prolongation taps of fine node i: count, coarse nodes J, weights w (nested or not)
MW_D int pw_g(int i, int nf, int nc, int* J, double* w) {
  if (nested_1d(nf, nc)) return pw(i, J, w);
  const int E = q2_weights_1d(i, nf, nc, w);
  J[0] = 2 * E; J[1] = 2 * E + 1; J[2] = 2 * E + 2;
  return 3;
}

// (P x_c) at fine node (ix, iz) between levels gf and gc: prolong_taps when both dimensions are
// nested, else the same sums over the general taps
template <typename G, typename V>
MW_D void prolong_taps_g(const G& gf, const G& gc, int ix, int iz, const V& coarse, double* s0, double* s1) {
  if (nested_1d(gf.nx, gc.nx) && nested_1d(gf.nz, gc.nz)) {
    prolong_taps(ix, iz, coarse, s0, s1);
    return;
  }
  int Jx[3] = {0, 0, 0}, Jz[3] = {0, 0, 0};
  double wx[3] = {0, 0, 0}, wz[3] = {0, 0, 0};
  const int nxw = pw_g(ix, gf.nx, gc.nx, Jx, wx), nzw = pw_g(iz, gf.nz, gc.nz, Jz, wz);
  double a0 = 0, a1 = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
      if (a < nzw && b < nxw) {
        const auto v = coarse(Jz[a], Jx[b]);
        const double w = wz[a] * wx[b];
        a0 = fma(w, (double)v.x, a0);
        a1 = fma(w, (double)v.y, a1);
      }
  *s0 = a0;
  *s1 = a1;
}

// the coarse-correction tile the AM_CHEB_P staging reads: coarse lattice nodes [ex0 - 2, ex0 + 17]
// x [ez0 - 2, ez0 + 9] cover every tap of the staged fine nodes [2 ex0 - 2, 2 ex0 + 32] x
// [2 ez0 - 2, 2 ez0 + 16]
constexpr int CLX = 20, CLZ = 12;

#ifndef MW_APPLY_MINB
#define MW_APPLY_MINB 5      // resident FP32 apply CTAs per SM the register budget is sized for
#endif

// Asynchronous copy (LDGSTS) of one node's component pair from global to shared memory.
template <typename R>
MW_D void cp_async_pair(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (sizeof(R) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
MW_D void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Shared memory of one operator-apply tile (the arrays of apply_tile).  Node vectors the epilogue
// reads for the four nodes each owned element emits (b; b, diag, d) are fetched asynchronously
// while the element products run (FP32 only: the FP64 tile's shared memory stays under the 48 KB
// static limit without them).
template <typename R, int MODE>
struct ApplySmem {
  typedef typename Vec2<R>::T R2;
  static constexpr bool CHEB = MODE == AM_CHEB || MODE == AM_CHEB_Z || MODE == AM_CHEB_P;
  static constexpr bool PRO = MODE == AM_CHEB_P;
  static constexpr int NPRE = sizeof(R) == 8 ? 0 : (CHEB ? 3 : (MODE == AM_RESID ? 1 : 0));
  static constexpr int NJ = APPLY_THREADS - TX * TZ;  // spare threads: right column and top row nodes
  __align__(16) R su[LZ * LX * 2];
  __align__(16) R2 spre[NPRE ? NPRE * 4 * TX * TZ : 1];
  __align__(16) R2 sspare[NPRE ? NPRE * 2 * NJ : 1];
  R sp[PZ * PX];
  R sye[NEL_T * 22];
  uchar2 sfix[LZ * LX];                              // Dirichlet flags of the staged nodes
  __align__(16) R2 scx[PRO ? CLZ * CLX : 1];         // AM_CHEB_P: the coarse correction tile
};

// Where one tile's shared arrays are: the static arrays of k_apply, or an ApplySmem carved from
// the dynamic shared memory of a kernel that runs several layouts.
template <typename R>
struct ApplyPtrs {
  typedef typename Vec2<R>::T R2;
  R* su;
  R2 *spre, *sspare;
  R *sp, *sye;
  uchar2* sfix;
  R2* scx;
};

template <typename R, int MODE>
MW_D ApplyPtrs<R> apply_ptrs(ApplySmem<R, MODE>& sm) {
  return ApplyPtrs<R>{sm.su, sm.spre, sm.sspare, sm.sp, sm.sye, sm.sfix, sm.scx};
}

// One operator apply over element tile (bx, bz) by the APPLY_THREADS threads of a CTA, in the
// shared arrays sm.  A CTA that runs several tiles one after another separates them with a
// __syncthreads() (the next tile's staging overwrites what this one's epilogue reads).
template <typename R, int MODE>
MW_D void apply_tile(const LevelGeo& g, const ApplyArgs<R>& a, int bx, int bz, const ApplyPtrs<R>& sm) {
  typedef typename Vec2<R>::T R2;
  constexpr bool CHEB = ApplySmem<R, MODE>::CHEB;
  constexpr bool PRO = ApplySmem<R, MODE>::PRO;
  constexpr int NPRE = ApplySmem<R, MODE>::NPRE;
  constexpr int NJ = ApplySmem<R, MODE>::NJ;
  static_assert(2 * TZ + 1 + 2 * TX <= 2 * NJ, "the spare threads take at most two boundary nodes each");
  R* const su = sm.su;
  R2* const spre = sm.spre;
  R2* const sspare = sm.sspare;
  R* const sp = sm.sp;
  R* const sye = sm.sye;
  uchar2* const sfix = sm.sfix;
  R2* const scx = sm.scx;
  const int ex0 = bx * TX, ez0 = bz * TZ;
  const int lx0 = 2 * ex0 - 2, lz0 = 2 * ez0 - 2;      // lattice origin of the staged nodes
  const int tid = threadIdx.x;
  const bool use_u = a.u != nullptr, use_p = a.p != nullptr;
  // Chebyshev coefficients, read now so that no epilogue load waits on them
  const double c1 = CHEB ? a.cheb[0] : 0.0;
  const R c2 = CHEB ? R(a.cheb[1]) : R(0);
  const R cz = MODE == AM_CHEB_Z ? R(a.cheb0[1]) : R(0);
  // ---- prefetch: the epilogue's node vectors (owned elements), the element viscosities ----
  // slot j of an owned element: 0 centre (2ex+1, 2ez+1), 1 bottom midpoint (2ex+1, 2ez),
  // 2 left midpoint (2ex, 2ez+1), 3 corner (2ex, 2ez)
  if (NPRE && a.yV && tid < TX * TZ) {
    const int ex = ex0 + tid % TX, ez = ez0 + tid / TX;
    if (ex < g.nx && ez < g.nz) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int ix = 2 * ex + (j < 2 ? 1 : 0), iz = 2 * ez + ((j & 1) ? 0 : 1);
        const int64_t n = (int64_t)iz * g.nnx + ix;
        cp_async_pair<R>(&spre[j * TX * TZ + tid], a.bV + 2 * n);
        if (NPRE == 3) {
          cp_async_pair<R>(&spre[(4 + j) * TX * TZ + tid], a.diag + 2 * n);
          if (MODE == AM_CHEB) cp_async_pair<R>(&spre[(8 + j) * TX * TZ + tid], a.d + 2 * n);
        }
      }
    }
  }
  // the spare threads' boundary nodes (at most 2 TZ + 1 + 2 TX = 49, two per spare thread)
  const bool lastx = ex0 + TX >= g.nx, lastz = ez0 + TZ >= g.nz;
  const int oz1 = lastz ? 2 * g.nz + 1 : 2 * (ez0 + TZ);
  const int ncol_v = lastx ? oz1 - 2 * ez0 : 0;
  const int nrow_v = lastz ? (lastx ? 2 * (g.nx - ex0) : 2 * TX) : 0;
  if (NPRE && a.yV && tid >= TX * TZ && (lastx || lastz)) {
#pragma unroll
    for (int it = 0; it < 2; ++it) {
      const int j = tid - TX * TZ + it * NJ;
      if (j < ncol_v + nrow_v) {
        const int ix = j < ncol_v ? 2 * g.nx : 2 * ex0 + (j - ncol_v);
        const int iz = j < ncol_v ? 2 * ez0 + j : 2 * g.nz;
        const int64_t n = (int64_t)iz * g.nnx + ix;
        const int q = tid - TX * TZ;
        cp_async_pair<R>(&sspare[it * NJ + q], a.bV + 2 * n);
        if (NPRE == 3) {
          cp_async_pair<R>(&sspare[(2 + it) * NJ + q], a.diag + 2 * n);
          if (MODE == AM_CHEB) cp_async_pair<R>(&sspare[(4 + it) * NJ + q], a.d + 2 * n);
        }
      }
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  R eq[9];
  if (tid < NEL_T) {
    const int ex = ex0 - 1 + tid % EX, ez = ez0 - 1 + tid / EX;
    if (ex >= 0 && ex < g.nx && ez >= 0 && ez < g.nz) {
      const R* eg = a.eta + ((int64_t)ez * g.nx + ex) * 9;
#pragma unroll
      for (int q = 0; q < 9; ++q) eq[q] = eg[q];
    }
  }
  // ---- AM_CHEB_P: the coarse correction tile (loaded now, stored after the fine loads) ----
  constexpr int NCT = PRO ? (CLZ * CLX + APPLY_THREADS - 1) / APPLY_THREADS : 1;
  R2 cv[NCT];
  const int cx0 = ex0 - 2, cz0 = ez0 - 2;
  if constexpr (PRO) {
#pragma unroll
    for (int k = 0; k < NCT; ++k) {
      const int i = tid + k * APPLY_THREADS;
      const int jz = i / CLX, jx = i - jz * CLX;
      const int cx = cx0 + jx, cz = cz0 + jz;
      cv[k].x = 0; cv[k].y = 0;
      if (i < CLZ * CLX && cx >= 0 && cx < a.gc.nnx && cz >= 0 && cz < a.gc.nnz)
        cv[k] = reinterpret_cast<const R2*>(a.xc)[(int64_t)cz * a.gc.nnx + cx];
    }
  }
  // x + P x_c on the free dofs of fine node (ix, iz) (the arithmetic of k_prolong_add)
  auto corrected = [&](int ix, int iz, R2 x, uchar2 ff) -> R2 {
    double s0, s1;
    prolong_taps(ix, iz, [&](int jz, int jx) { return scx[(jz - cz0) * CLX + (jx - cx0)]; }, &s0, &s1);
    if (!ff.x) x.x += (R)s0;
    if (!ff.y) x.y += (R)s1;
    return x;
  };
  // ---- stage velocity (masked; one vector load per node), pressure ----
  // A fixed number of nodes per thread, all loads issued before any shared-memory store, so the
  // staging costs one memory round trip rather than one per node.
  const R2* u2 = reinterpret_cast<const R2*>(a.u);
  const uchar2* f2 = reinterpret_cast<const uchar2*>(a.fix);
  R2* su2 = reinterpret_cast<R2*>(su);
  constexpr int NST = (LZ * LX + APPLY_THREADS - 1) / APPLY_THREADS;
  constexpr int NSP = (PZ * PX + APPLY_THREADS - 1) / APPLY_THREADS;
  R2 sv[NST];
  uchar2 sf[NST];
  R spv[NSP];
  if constexpr (sizeof(R) == 8) {                    // FP64: one node at a time (fewer live registers)
    if constexpr (PRO) {
#pragma unroll
      for (int k = 0; k < NCT; ++k)
        if (tid + k * APPLY_THREADS < CLZ * CLX) scx[tid + k * APPLY_THREADS] = cv[k];
      __syncthreads();
    }
    for (int i = tid; i < LZ * LX; i += APPLY_THREADS) {
      const int lz = i / LX, lx = i - lz * LX;
      const int ix = lx0 + lx, iz = lz0 + lz;
      R2 v;
      v.x = 0; v.y = 0;
      uchar2 ff = make_uchar2(0, 0);
      if (ix >= 0 && ix < g.nnx && iz >= 0 && iz < g.nnz) {
        const int64_t n = (int64_t)iz * g.nnx + ix;
        ff = f2[n];
        if (use_u) {
          R2 uu = u2[n];
          if constexpr (PRO) uu = corrected(ix, iz, uu, ff);
          v.x = ff.x ? R(0) : uu.x;
          v.y = ff.y ? R(0) : uu.y;
        }
      }
      su2[i] = v;
      sfix[i] = ff;
    }
    if (use_p)
      for (int i = tid; i < PZ * PX; i += APPLY_THREADS) {
        int jz = i / PX, jx = i % PX;
        int px = ex0 - 1 + jx, pz = ez0 - 1 + jz;
        sp[i] = (px >= 0 && px <= g.nx && pz >= 0 && pz <= g.nz) ? a.p[(int64_t)pz * (g.nx + 1) + px] : R(0);
      }
  } else {
#pragma unroll
  for (int k = 0; k < NST; ++k) {
    const int i = tid + k * APPLY_THREADS;
    const int lz = i / LX, lx = i - lz * LX;
    const int ix = lx0 + lx, iz = lz0 + lz;
    sv[k].x = 0; sv[k].y = 0;
    sf[k] = make_uchar2(0, 0);
    if (i < LZ * LX && ix >= 0 && ix < g.nnx && iz >= 0 && iz < g.nnz) {
      const int64_t n = (int64_t)iz * g.nnx + ix;
      sf[k] = f2[n];
      if (MODE == AM_CHEB_Z) {                       // x0 = (1/theta) D^-1 b
        const R2 bb = reinterpret_cast<const R2*>(a.bV)[n], dg = reinterpret_cast<const R2*>(a.diag)[n];
        sv[k].x = cz * bb.x / dg.x;
        sv[k].y = cz * bb.y / dg.y;
      } else if (use_u) {
        sv[k] = u2[n];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < NSP; ++k) {
    const int i = tid + k * APPLY_THREADS;
    const int jz = i / PX, jx = i % PX;
    const int px = ex0 - 1 + jx, pz = ez0 - 1 + jz;
    spv[k] = (use_p && i < PZ * PX && px >= 0 && px <= g.nx && pz >= 0 && pz <= g.nz)
                 ? a.p[(int64_t)pz * (g.nx + 1) + px] : R(0);
  }
  if constexpr (PRO) {
#pragma unroll
    for (int k = 0; k < NCT; ++k)
      if (tid + k * APPLY_THREADS < CLZ * CLX) scx[tid + k * APPLY_THREADS] = cv[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NST; ++k) {
      const int i = tid + k * APPLY_THREADS;
      const int lz = i / LX, lx = i - lz * LX;
      const int ix = lx0 + lx, iz = lz0 + lz;
      if (i < LZ * LX && ix >= 0 && ix < g.nnx && iz >= 0 && iz < g.nnz) sv[k] = corrected(ix, iz, sv[k], sf[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < NST; ++k) {
    const int i = tid + k * APPLY_THREADS;
    if (i < LZ * LX) {
      R2 v;
      v.x = sf[k].x ? R(0) : sv[k].x;
      v.y = sf[k].y ? R(0) : sv[k].y;
      su2[i] = v;
      sfix[i] = sf[k];
    }
  }
#pragma unroll
  for (int k = 0; k < NSP; ++k) {
    const int i = tid + k * APPLY_THREADS;
    if (use_p && i < PZ * PX) sp[i] = spv[k];
  }
  }
  __syncthreads();
  // ---- element products ----
  if (tid < NEL_T) {
    int lex = tid % EX, lez = tid / EX;
    int ex = ex0 - 1 + lex, ez = ez0 - 1 + lez;
    if (ex >= 0 && ex < g.nx && ez >= 0 && ez < g.nz) {
      __align__(16) R ue[18];
      R pe[4], ye[18], ype[4];
      const int bx = 2 * lex, bz = 2 * lez;          // staged lattice coords of local node 0
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        int li = (bz + q2_dz(k)) * LX + bx + q2_dx(k);
        ue[2 * k] = su[2 * li]; ue[2 * k + 1] = su[2 * li + 1];
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) pe[k] = use_p ? sp[(lez + q1_dz(k)) * PX + lex + q1_dx(k)] : R(0);
      const R sxe = R(2.0 / g.hx), sze = R(2.0 / g.hz), jace = R(g.hx * g.hz / 4.0), se = R(g.s);
      if (!use_u)                                   // G p only (the Schur iteration's G d, f - G P)
        element_apply<R, false, true>(sxe, sze, jace, se, ue, pe, eq, ye, ype, use_p);
      else if (!a.yV)                               // G^T u only
        element_apply<R, true, false>(sxe, sze, jace, se, ue, pe, eq, ye, ype, use_p);
      else
        element_apply<R>(sxe, sze, jace, se, ue, pe, eq, ye, ype, use_p);
#pragma unroll
      for (int k = 0; k < 18; ++k) sye[tid * 22 + k] = ye[k];
#pragma unroll
      for (int k = 0; k < 4; ++k) sye[tid * 22 + 18 + k] = ype[k];
    }
  }
  cp_async_wait_all();
  __syncthreads();
  // ---- owned nodes: sums over the incident elements in ascending element order ----
  // Each owned element's thread takes the four nodes of its lower-left quadrant (centre, bottom
  // and left edge midpoints, lower-left corner) and its lower-left pressure node, with the element
  // local indices known at compile time; the spare threads take the nodes on the right and top
  // mesh boundary, which belong to no element's lower-left quadrant.
  // prefetched value of array k (0 b, 1 diag, 2 d): slots 0-3 are an owned element's nodes,
  // slots 4-5 a spare thread's two boundary nodes
  auto pre_at = [&](int k, int slot) -> R2 {
    return slot < 4 ? spre[(4 * k + slot) * TX * TZ + tid] : sspare[(2 * k + slot - 4) * NJ + (tid - TX * TZ)];
  };
  // velocity node epilogue: Dirichlet rows, then the mode's output.  slot >= 0: b, diag, d were
  // prefetched; slot < 0: read them here.
  auto emit = [&](int ix, int iz, R y0, R y1, int slot) {
    const int64_t n = (int64_t)iz * g.nnx + ix;
    const int li = (iz - lz0) * LX + (ix - lx0);
    const uchar2 ff = sfix[li];
    const bool fixed = (ff.x | ff.y) && use_u;       // calls without a velocity (G p only) pass no diagonal
    const bool pre = NPRE && slot >= 0;
    // every load first, none depending on another
    R2 uu = su2[li];                                 // the staged velocity: exact on free dofs
    R2 dg{R(0), R(0)}, bb{R(0), R(0)}, dd{R(0), R(0)};
    if (CHEB) dg = pre ? pre_at(1, slot) : reinterpret_cast<const R2*>(a.diag)[n];
    else if (fixed) dg = reinterpret_cast<const R2*>(a.diag)[n];
    if (fixed && MODE != AM_CHEB_Z) {                // the fixed components' values (staged as 0);
      const R2 raw = reinterpret_cast<const R2*>(a.u)[n];   // a free one keeps its staged value,
      if (ff.x) uu.x = raw.x;                        // which under AM_CHEB_P carries P x_c
      if (ff.y) uu.y = raw.y;
    }
    if (MODE != AM_APPLY) bb = pre ? pre_at(0, slot) : reinterpret_cast<const R2*>(a.bV)[n];
    if (MODE == AM_CHEB && c1 != 0.0)                // restart steps never read the old direction
      dd = pre ? pre_at(2, slot) : reinterpret_cast<const R2*>(a.d)[n];
    if (MODE == AM_CHEB_Z) {                         // the first step's x and d, both x0
      const R2 x0{cz * bb.x / dg.x, cz * bb.y / dg.y};
      if (fixed) uu = x0;
      dd = x0;
    }
    R2 y;
    y.x = y0;
    y.y = y1;
    if (ff.x | ff.y) {                               // eliminated rows act as K_ii u_i
      const R2 fy = fixed ? R2{dg.x * uu.x, dg.y * uu.y} : R2{R(0), R(0)};
      if (ff.x) y.x = fy.x;
      if (ff.y) y.y = fy.y;
    }
    if (MODE == AM_APPLY) {
      reinterpret_cast<R2*>(a.yV)[n] = y;
    } else if (MODE == AM_RESID) {
      reinterpret_cast<R2*>(a.yV)[n] = R2{bb.x - y.x, bb.y - y.y};
    } else {   // Chebyshev step: d = c1 d + c2 D^-1 (b - y); x_out = u + d
      R2 dn{c2 * (bb.x - y.x) / dg.x, c2 * (bb.y - y.y) / dg.y};
      if (c1 != 0.0) {
        dn.x += R(c1) * dd.x;
        dn.y += R(c1) * dd.y;
      }
      reinterpret_cast<R2*>(a.d)[n] = dn;
      reinterpret_cast<R2*>(a.xo)[n] = R2{uu.x + dn.x, uu.y + dn.y};
    }
  };
  // any velocity node of the tile (incident elements found from the node's parity)
  auto node_generic = [&](int ix, int iz, int slot) {
    const bool xo = ix & 1, zo = iz & 1;
    const int xa = xo ? (ix >> 1) : (ix >> 1) - 1, xb = (ix >> 1);
    const int za = zo ? (iz >> 1) : (iz >> 1) - 1, zb = (iz >> 1);
    const bool vxa = xa >= 0, vxb = !xo && xb < g.nx;
    const bool vza = za >= 0, vzb = !zo && zb < g.nz;
    const int dxa = xo ? 1 : 2, dza = zo ? 1 : 2;   // offsets inside element xa / za; 0 inside xb / zb
    R y0 = 0, y1 = 0;
    if (vza) {
      const int lez = za - (ez0 - 1);
      if (vxa) { const R* ye = sye + (lez * EX + xa - (ex0 - 1)) * 22; int k = q2_local_idx(dxa, dza);
                 y0 += ye[2 * k]; y1 += ye[2 * k + 1]; }
      if (vxb) { const R* ye = sye + (lez * EX + xb - (ex0 - 1)) * 22; int k = q2_local_idx(0, dza);
                 y0 += ye[2 * k]; y1 += ye[2 * k + 1]; }
    }
    if (vzb) {
      const int lez = zb - (ez0 - 1);
      if (vxa) { const R* ye = sye + (lez * EX + xa - (ex0 - 1)) * 22; int k = q2_local_idx(dxa, 0);
                 y0 += ye[2 * k]; y1 += ye[2 * k + 1]; }
      if (vxb) { const R* ye = sye + (lez * EX + xb - (ex0 - 1)) * 22; int k = q2_local_idx(0, 0);
                 y0 += ye[2 * k]; y1 += ye[2 * k + 1]; }
    }
    emit(ix, iz, y0, y1, slot);
  };
  // any pressure node of the tile
  auto pnode_generic = [&](int px, int pz) {
    // incident elements (pz-1, px-1) k=2, (pz-1, px) k=3, (pz, px-1) k=1, (pz, px) k=0
    const bool l = px >= 1, rr = px < g.nx, bo = pz >= 1, to = pz < g.nz;
    const int lx = px - ex0, lz = pz - ez0;          // tile-local index of element (px, pz) is (lx+1, lz+1)
    R y = 0;
    if (bo && l) y += sye[((lz) * EX + lx) * 22 + 18 + 2];
    if (bo && rr) y += sye[((lz) * EX + lx + 1) * 22 + 18 + 3];
    if (to && l) y += sye[((lz + 1) * EX + lx) * 22 + 18 + 1];
    if (to && rr) y += sye[((lz + 1) * EX + lx + 1) * 22 + 18 + 0];
    const int64_t n = (int64_t)pz * (g.nx + 1) + px;
    a.yP[n] = (MODE == AM_RESID) ? a.bP[n] - y : y;
  };
  if (tid < TX * TZ) {
    const int lx = tid % TX, lz = tid / TX;          // TX is a power of two
    const int ex = ex0 + lx, ez = ez0 + lz;
    if (ex < g.nx && ez < g.nz) {
      const R* e00 = sye + ((lz + 1) * EX + lx + 1) * 22;   // element (ex, ez)
      const R* eL = e00 - 22;                                 // (ex-1, ez)
      const R* eB = e00 - EX * 22;                            // (ex, ez-1)
      const R* eBL = eB - 22;                                 // (ex-1, ez-1)
      const bool hasL = ex > 0, hasB = ez > 0;
      if (a.yV) {
        emit(2 * ex + 1, 2 * ez + 1, e00[16], e00[17], 0);   // centre: local node 8
        {                                                     // bottom edge midpoint: 6 of (ex,ez-1), 4
          R y0 = 0, y1 = 0;
          if (hasB) { y0 += eB[12]; y1 += eB[13]; }
          y0 += e00[8]; y1 += e00[9];
          emit(2 * ex + 1, 2 * ez, y0, y1, 1);
        }
        {                                                     // left edge midpoint: 5 of (ex-1,ez), 7
          R y0 = 0, y1 = 0;
          if (hasL) { y0 += eL[10]; y1 += eL[11]; }
          y0 += e00[14]; y1 += e00[15];
          emit(2 * ex, 2 * ez + 1, y0, y1, 2);
        }
        {                                                     // lower-left corner: 2, 3, 1, 0
          R y0 = 0, y1 = 0;
          if (hasB && hasL) { y0 += eBL[4]; y1 += eBL[5]; }
          if (hasB) { y0 += eB[6]; y1 += eB[7]; }
          if (hasL) { y0 += eL[2]; y1 += eL[3]; }
          y0 += e00[0]; y1 += e00[1];
          emit(2 * ex, 2 * ez, y0, y1, 3);
        }
      }
      if (a.yP) {                                             // pressure node (ex, ez): 2, 3, 1, 0
        R y = 0;
        if (hasB && hasL) y += eBL[18 + 2];
        if (hasB) y += eB[18 + 3];
        if (hasL) y += eL[18 + 1];
        y += e00[18 + 0];
        const int64_t n = (int64_t)ez * (g.nx + 1) + ex;
        a.yP[n] = (MODE == AM_RESID) ? a.bP[n] - y : y;
      }
    }
  } else if (lastx || lastz) {
    // right column ix = 2 nx (rows of this tile) and top row iz = 2 nz (columns of this tile,
    // the corner taken by the column)
    const int j0 = tid - TX * TZ, nj = NJ;
    if (a.yV) {
#pragma unroll
      for (int it = 0; it < 2; ++it) {                // the nodes whose vectors were prefetched
        const int j = j0 + it * nj;
        if (j < ncol_v + nrow_v) {
          if (j < ncol_v) node_generic(2 * g.nx, 2 * ez0 + j, 4 + it);
          else node_generic(2 * ex0 + (j - ncol_v), 2 * g.nz, 4 + it);
        }
      }
    }
    if (a.yP) {
      const int pz1 = lastz ? g.nz + 1 : ez0 + TZ;
      const int ncol = lastx ? pz1 - ez0 : 0;
      const int nrow = lastz ? (lastx ? g.nx - ex0 : TX) : 0;
      for (int j = j0; j < ncol + nrow; j += nj) {
        if (j < ncol) pnode_generic(g.nx, ez0 + j);
        else pnode_generic(ex0 + (j - ncol), g.nz);
      }
    }
  }
}

// The operator apply as a kernel, one tile per CTA.  It repeats apply_tile's arithmetic with its
// body inline and its own static shared arrays: compiled through apply_tile (parameters by value or
// by reference), the FP64 Chebyshev mode ran 43 % slower and the plain FP64 512x512 step took 106
// instead of 93 ms (FP32 the same), measured on one GPU; apply_tile serves the kernels that run
// several tiles per CTA (the ensemble's cluster solve), and its GPU tests check the two against
// each other through the solves.
template <typename R, int MODE>
__global__ void __launch_bounds__(APPLY_THREADS, sizeof(R) == 4 ? MW_APPLY_MINB : 1)
k_apply(LevelGeo g, ApplyArgs<R> a) {
  pdl_entry();
  typedef typename Vec2<R>::T R2;
  // node vectors the epilogue reads for the four nodes each owned element emits (b; b, diag, d),
  // fetched asynchronously while the element products run (FP32; the FP64 kernel's shared memory
  // is already at the 48 KB static limit)
  constexpr bool CHEB = MODE == AM_CHEB || MODE == AM_CHEB_Z || MODE == AM_CHEB_P;
  constexpr bool PRO = MODE == AM_CHEB_P;
  constexpr int NPRE = sizeof(R) == 8 ? 0 : (CHEB ? 3 : (MODE == AM_RESID ? 1 : 0));
  __shared__ __align__(16) R su[LZ * LX * 2];
  __shared__ __align__(16) R2 spre[(NPRE ? NPRE : 1) * 4 * TX * TZ];
  constexpr int NJ = APPLY_THREADS - TX * TZ;         // spare threads: right column and top row nodes
  static_assert(2 * TZ + 1 + 2 * TX <= 2 * NJ, "the spare threads take at most two boundary nodes each");
  __shared__ __align__(16) R2 sspare[(NPRE ? NPRE : 1) * 2 * NJ];
  __shared__ R sp[PZ * PX];
  __shared__ R sye[NEL_T * 22];
  __shared__ uchar2 sfix[LZ * LX];          // Dirichlet flags of the staged nodes
  __shared__ __align__(16) R2 scx[PRO ? CLZ * CLX : 1];   // AM_CHEB_P: the coarse correction tile
  const int ex0 = blockIdx.x * TX, ez0 = blockIdx.y * TZ;
  const int lx0 = 2 * ex0 - 2, lz0 = 2 * ez0 - 2;      // lattice origin of the staged nodes
  const int tid = threadIdx.x;
  const bool use_u = a.u != nullptr, use_p = a.p != nullptr;
  // Chebyshev coefficients, read now so that no epilogue load waits on them
  const double c1 = CHEB ? a.cheb[0] : 0.0;
  const R c2 = CHEB ? R(a.cheb[1]) : R(0);
  const R cz = MODE == AM_CHEB_Z ? R(a.cheb0[1]) : R(0);
  // ---- prefetch: the epilogue's node vectors (owned elements), the element viscosities ----
  // slot j of an owned element: 0 centre (2ex+1, 2ez+1), 1 bottom midpoint (2ex+1, 2ez),
  // 2 left midpoint (2ex, 2ez+1), 3 corner (2ex, 2ez)
  if (NPRE && a.yV && tid < TX * TZ) {
    const int ex = ex0 + tid % TX, ez = ez0 + tid / TX;
    if (ex < g.nx && ez < g.nz) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int ix = 2 * ex + (j < 2 ? 1 : 0), iz = 2 * ez + ((j & 1) ? 0 : 1);
        const int64_t n = (int64_t)iz * g.nnx + ix;
        cp_async_pair<R>(&spre[j * TX * TZ + tid], a.bV + 2 * n);
        if (NPRE == 3) {
          cp_async_pair<R>(&spre[(4 + j) * TX * TZ + tid], a.diag + 2 * n);
          if (MODE == AM_CHEB) cp_async_pair<R>(&spre[(8 + j) * TX * TZ + tid], a.d + 2 * n);
        }
      }
    }
  }
  // the spare threads' boundary nodes (at most 2 TZ + 1 + 2 TX = 49, two per spare thread)
  const bool lastx = ex0 + TX >= g.nx, lastz = ez0 + TZ >= g.nz;
  const int oz1 = lastz ? 2 * g.nz + 1 : 2 * (ez0 + TZ);
  const int ncol_v = lastx ? oz1 - 2 * ez0 : 0;
  const int nrow_v = lastz ? (lastx ? 2 * (g.nx - ex0) : 2 * TX) : 0;
  if (NPRE && a.yV && tid >= TX * TZ && (lastx || lastz)) {
#pragma unroll
    for (int it = 0; it < 2; ++it) {
      const int j = tid - TX * TZ + it * NJ;
      if (j < ncol_v + nrow_v) {
        const int ix = j < ncol_v ? 2 * g.nx : 2 * ex0 + (j - ncol_v);
        const int iz = j < ncol_v ? 2 * ez0 + j : 2 * g.nz;
        const int64_t n = (int64_t)iz * g.nnx + ix;
        const int q = tid - TX * TZ;
        cp_async_pair<R>(&sspare[it * NJ + q], a.bV + 2 * n);
        if (NPRE == 3) {
          cp_async_pair<R>(&sspare[(2 + it) * NJ + q], a.diag + 2 * n);
          if (MODE == AM_CHEB) cp_async_pair<R>(&sspare[(4 + it) * NJ + q], a.d + 2 * n);
        }
      }
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  R eq[9];
  if (tid < NEL_T) {
    const int ex = ex0 - 1 + tid % EX, ez = ez0 - 1 + tid / EX;
    if (ex >= 0 && ex < g.nx && ez >= 0 && ez < g.nz) {
      const R* eg = a.eta + ((int64_t)ez * g.nx + ex) * 9;
#pragma unroll
      for (int q = 0; q < 9; ++q) eq[q] = eg[q];
    }
  }
  // ---- AM_CHEB_P: the coarse correction tile (loaded now, stored after the fine loads) ----
  constexpr int NCT = PRO ? (CLZ * CLX + APPLY_THREADS - 1) / APPLY_THREADS : 1;
  R2 cv[NCT];
  const int cx0 = ex0 - 2, cz0 = ez0 - 2;
  if constexpr (PRO) {
#pragma unroll
    for (int k = 0; k < NCT; ++k) {
      const int i = tid + k * APPLY_THREADS;
      const int jz = i / CLX, jx = i - jz * CLX;
      const int cx = cx0 + jx, cz = cz0 + jz;
      cv[k].x = 0; cv[k].y = 0;
      if (i < CLZ * CLX && cx >= 0 && cx < a.gc.nnx && cz >= 0 && cz < a.gc.nnz)
        cv[k] = reinterpret_cast<const R2*>(a.xc)[(int64_t)cz * a.gc.nnx + cx];
    }
  }
  // x + P x_c on the free dofs of fine node (ix, iz) (the arithmetic of k_prolong_add)
  auto corrected = [&](int ix, int iz, R2 x, uchar2 ff) -> R2 {
    double s0, s1;
    prolong_taps(ix, iz, [&](int jz, int jx) { return scx[(jz - cz0) * CLX + (jx - cx0)]; }, &s0, &s1);
    if (!ff.x) x.x += (R)s0;
    if (!ff.y) x.y += (R)s1;
    return x;
  };
  // ---- stage velocity (masked; one vector load per node), pressure ----
  // A fixed number of nodes per thread, all loads issued before any shared-memory store, so the
  // staging costs one memory round trip rather than one per node.
  const R2* u2 = reinterpret_cast<const R2*>(a.u);
  const uchar2* f2 = reinterpret_cast<const uchar2*>(a.fix);
  R2* su2 = reinterpret_cast<R2*>(su);
  constexpr int NST = (LZ * LX + APPLY_THREADS - 1) / APPLY_THREADS;
  constexpr int NSP = (PZ * PX + APPLY_THREADS - 1) / APPLY_THREADS;
  R2 sv[NST];
  uchar2 sf[NST];
  R spv[NSP];
  if constexpr (sizeof(R) == 8) {                    // FP64: one node at a time (fewer live registers)
    if constexpr (PRO) {
#pragma unroll
      for (int k = 0; k < NCT; ++k)
        if (tid + k * APPLY_THREADS < CLZ * CLX) scx[tid + k * APPLY_THREADS] = cv[k];
      __syncthreads();
    }
    for (int i = tid; i < LZ * LX; i += APPLY_THREADS) {
      const int lz = i / LX, lx = i - lz * LX;
      const int ix = lx0 + lx, iz = lz0 + lz;
      R2 v;
      v.x = 0; v.y = 0;
      uchar2 ff = make_uchar2(0, 0);
      if (ix >= 0 && ix < g.nnx && iz >= 0 && iz < g.nnz) {
        const int64_t n = (int64_t)iz * g.nnx + ix;
        ff = f2[n];
        if (use_u) {
          R2 uu = u2[n];
          if constexpr (PRO) uu = corrected(ix, iz, uu, ff);
          v.x = ff.x ? R(0) : uu.x;
          v.y = ff.y ? R(0) : uu.y;
        }
      }
      su2[i] = v;
      sfix[i] = ff;
    }
    if (use_p)
      for (int i = tid; i < PZ * PX; i += APPLY_THREADS) {
        int jz = i / PX, jx = i % PX;
        int px = ex0 - 1 + jx, pz = ez0 - 1 + jz;
        sp[i] = (px >= 0 && px <= g.nx && pz >= 0 && pz <= g.nz) ? a.p[(int64_t)pz * (g.nx + 1) + px] : R(0);
      }
  } else {
#pragma unroll
  for (int k = 0; k < NST; ++k) {
    const int i = tid + k * APPLY_THREADS;
    const int lz = i / LX, lx = i - lz * LX;
    const int ix = lx0 + lx, iz = lz0 + lz;
    sv[k].x = 0; sv[k].y = 0;
    sf[k] = make_uchar2(0, 0);
    if (i < LZ * LX && ix >= 0 && ix < g.nnx && iz >= 0 && iz < g.nnz) {
      const int64_t n = (int64_t)iz * g.nnx + ix;
      sf[k] = f2[n];
      if (MODE == AM_CHEB_Z) {                       // x0 = (1/theta) D^-1 b
        const R2 bb = reinterpret_cast<const R2*>(a.bV)[n], dg = reinterpret_cast<const R2*>(a.diag)[n];
        sv[k].x = cz * bb.x / dg.x;
        sv[k].y = cz * bb.y / dg.y;
      } else if (use_u) {
        sv[k] = u2[n];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < NSP; ++k) {
    const int i = tid + k * APPLY_THREADS;
    const int jz = i / PX, jx = i % PX;
    const int px = ex0 - 1 + jx, pz = ez0 - 1 + jz;
    spv[k] = (use_p && i < PZ * PX && px >= 0 && px <= g.nx && pz >= 0 && pz <= g.nz)
                 ? a.p[(int64_t)pz * (g.nx + 1) + px] : R(0);
  }
  if constexpr (PRO) {
#pragma unroll
    for (int k = 0; k < NCT; ++k)
      if (tid + k * APPLY_THREADS < CLZ * CLX) scx[tid + k * APPLY_THREADS] = cv[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NST; ++k) {
      const int i = tid + k * APPLY_THREADS;
      const int lz = i / LX, lx = i - lz * LX;
      const int ix = lx0 + lx, iz = lz0 + lz;
      if (i < LZ * LX && ix >= 0 && ix < g.nnx && iz >= 0 && iz < g.nnz) sv[k] = corrected(ix, iz, sv[k], sf[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < NST; ++k) {
    const int i = tid + k * APPLY_THREADS;
    if (i < LZ * LX) {
      R2 v;
      v.x = sf[k].x ? R(0) : sv[k].x;
      v.y = sf[k].y ? R(0) : sv[k].y;
      su2[i] = v;
      sfix[i] = sf[k];
    }
  }
#pragma unroll
  for (int k = 0; k < NSP; ++k) {
    const int i = tid + k * APPLY_THREADS;
    if (use_p && i < PZ * PX) sp[i] = spv[k];
  }
  }
  __syncthreads();
  // ---- element products ----
  if (tid < NEL_T) {
    int lex = tid % EX, lez = tid / EX;
    int ex = ex0 - 1 + lex, ez = ez0 - 1 + lez;
    if (ex >= 0 && ex < g.nx && ez >= 0 && ez < g.nz) {
      __align__(16) R ue[18];
      R pe[4], ye[18], ype[4];
      const int bx = 2 * lex, bz = 2 * lez;          // staged lattice coords of local node 0
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        int li = (bz + q2_dz(k)) * LX + bx + q2_dx(k);
        ue[2 * k] = su[2 * li]; ue[2 * k + 1] = su[2 * li + 1];
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) pe[k] = use_p ? sp[(lez + q1_dz(k)) * PX + lex + q1_dx(k)] : R(0);
      const R sxe = R(2.0 / g.hx), sze = R(2.0 / g.hz), jace = R(g.hx * g.hz / 4.0), se = R(g.s);
      if (!use_u)                                   // G p only (the Schur iteration's G d, f - G P)
        element_apply<R, false, true>(sxe, sze, jace, se, ue, pe, eq, ye, ype, use_p);
      else if (!a.yV)                               // G^T u only
        element_apply<R, true, false>(sxe, sze, jace, se, ue, pe, eq, ye, ype, use_p);
      else
        element_apply<R>(sxe, sze, jace, se, ue, pe, eq, ye, ype, use_p);
#pragma unroll
      for (int k = 0; k < 18; ++k) sye[tid * 22 + k] = ye[k];
#pragma unroll
      for (int k = 0; k < 4; ++k) sye[tid * 22 + 18 + k] = ype[k];
    }
  }
  cp_async_wait_all();
  __syncthreads();
  // ---- owned nodes: sums over the incident elements in ascending element order ----
  // Each owned element's thread takes the four nodes of its lower-left quadrant (centre, bottom
  // and left edge midpoints, lower-left corner) and its lower-left pressure node, with the element
  // local indices known at compile time; the spare threads take the nodes on the right and top
  // mesh boundary, which belong to no element's lower-left quadrant.
  // prefetched value of array k (0 b, 1 diag, 2 d): slots 0-3 are an owned element's nodes,
  // slots 4-5 a spare thread's two boundary nodes
  auto pre_at = [&](int k, int slot) -> R2 {
    return slot < 4 ? spre[(4 * k + slot) * TX * TZ + tid] : sspare[(2 * k + slot - 4) * NJ + (tid - TX * TZ)];
  };
  // velocity node epilogue: Dirichlet rows, then the mode's output.  slot >= 0: b, diag, d were
  // prefetched; slot < 0: read them here.
  auto emit = [&](int ix, int iz, R y0, R y1, int slot) {
    const int64_t n = (int64_t)iz * g.nnx + ix;
    const int li = (iz - lz0) * LX + (ix - lx0);
    const uchar2 ff = sfix[li];
    const bool fixed = (ff.x | ff.y) && use_u;       // calls without a velocity (G p only) pass no diagonal
    const bool pre = NPRE && slot >= 0;
    // every load first, none depending on another
    R2 uu = su2[li];                                 // the staged velocity: exact on free dofs
    R2 dg{R(0), R(0)}, bb{R(0), R(0)}, dd{R(0), R(0)};
    if (CHEB) dg = pre ? pre_at(1, slot) : reinterpret_cast<const R2*>(a.diag)[n];
    else if (fixed) dg = reinterpret_cast<const R2*>(a.diag)[n];
    if (fixed && MODE != AM_CHEB_Z) {                // the fixed components' values (staged as 0);
      const R2 raw = reinterpret_cast<const R2*>(a.u)[n];   // a free one keeps its staged value,
      if (ff.x) uu.x = raw.x;                        // which under AM_CHEB_P carries P x_c
      if (ff.y) uu.y = raw.y;
    }
    if (MODE != AM_APPLY) bb = pre ? pre_at(0, slot) : reinterpret_cast<const R2*>(a.bV)[n];
    if (MODE == AM_CHEB && c1 != 0.0)                // restart steps never read the old direction
      dd = pre ? pre_at(2, slot) : reinterpret_cast<const R2*>(a.d)[n];
    if (MODE == AM_CHEB_Z) {                         // the first step's x and d, both x0
      const R2 x0{cz * bb.x / dg.x, cz * bb.y / dg.y};
      if (fixed) uu = x0;
      dd = x0;
    }
    R2 y;
    y.x = y0;
    y.y = y1;
    if (ff.x | ff.y) {                               // eliminated rows act as K_ii u_i
      const R2 fy = fixed ? R2{dg.x * uu.x, dg.y * uu.y} : R2{R(0), R(0)};
      if (ff.x) y.x = fy.x;
      if (ff.y) y.y = fy.y;
    }
    if (MODE == AM_APPLY) {
      reinterpret_cast<R2*>(a.yV)[n] = y;
    } else if (MODE == AM_RESID) {
      reinterpret_cast<R2*>(a.yV)[n] = R2{bb.x - y.x, bb.y - y.y};
    } else {   // Chebyshev step: d = c1 d + c2 D^-1 (b - y); x_out = u + d
      R2 dn{c2 * (bb.x - y.x) / dg.x, c2 * (bb.y - y.y) / dg.y};
      if (c1 != 0.0) {
        dn.x += R(c1) * dd.x;
        dn.y += R(c1) * dd.y;
      }
      reinterpret_cast<R2*>(a.d)[n] = dn;
      reinterpret_cast<R2*>(a.xo)[n] = R2{uu.x + dn.x, uu.y + dn.y};
    }
  };
  // any velocity node of the tile (incident elements found from the node's parity)
  auto node_generic = [&](int ix, int iz, int slot) {
    const bool xo = ix & 1, zo = iz & 1;
    const int xa = xo ? (ix >> 1) : (ix >> 1) - 1, xb = (ix >> 1);
    const int za = zo ? (iz >> 1) : (iz >> 1) - 1, zb = (iz >> 1);
    const bool vxa = xa >= 0, vxb = !xo && xb < g.nx;
    const bool vza = za >= 0, vzb = !zo && zb < g.nz;
    const int dxa = xo ? 1 : 2, dza = zo ? 1 : 2;   // offsets inside element xa / za; 0 inside xb / zb
    R y0 = 0, y1 = 0;
    if (vza) {
      const int lez = za - (ez0 - 1);
      if (vxa) { const R* ye = sye + (lez * EX + xa - (ex0 - 1)) * 22; int k = q2_local_idx(dxa, dza);
                 y0 += ye[2 * k]; y1 += ye[2 * k + 1]; }
      if (vxb) { const R* ye = sye + (lez * EX + xb - (ex0 - 1)) * 22; int k = q2_local_idx(0, dza);
                 y0 += ye[2 * k]; y1 += ye[2 * k + 1]; }
    }
    if (vzb) {
      const int lez = zb - (ez0 - 1);
      if (vxa) { const R* ye = sye + (lez * EX + xa - (ex0 - 1)) * 22; int k = q2_local_idx(dxa, 0);
                 y0 += ye[2 * k]; y1 += ye[2 * k + 1]; }
      if (vxb) { const R* ye = sye + (lez * EX + xb - (ex0 - 1)) * 22; int k = q2_local_idx(0, 0);
                 y0 += ye[2 * k]; y1 += ye[2 * k + 1]; }
    }
    emit(ix, iz, y0, y1, slot);
  };
  // any pressure node of the tile
  auto pnode_generic = [&](int px, int pz) {
    // incident elements (pz-1, px-1) k=2, (pz-1, px) k=3, (pz, px-1) k=1, (pz, px) k=0
    const bool l = px >= 1, rr = px < g.nx, bo = pz >= 1, to = pz < g.nz;
    const int lx = px - ex0, lz = pz - ez0;          // tile-local index of element (px, pz) is (lx+1, lz+1)
    R y = 0;
    if (bo && l) y += sye[((lz) * EX + lx) * 22 + 18 + 2];
    if (bo && rr) y += sye[((lz) * EX + lx + 1) * 22 + 18 + 3];
    if (to && l) y += sye[((lz + 1) * EX + lx) * 22 + 18 + 1];
    if (to && rr) y += sye[((lz + 1) * EX + lx + 1) * 22 + 18 + 0];
    const int64_t n = (int64_t)pz * (g.nx + 1) + px;
    a.yP[n] = (MODE == AM_RESID) ? a.bP[n] - y : y;
  };
  if (tid < TX * TZ) {
    const int lx = tid % TX, lz = tid / TX;          // TX is a power of two
    const int ex = ex0 + lx, ez = ez0 + lz;
    if (ex < g.nx && ez < g.nz) {
      const R* e00 = sye + ((lz + 1) * EX + lx + 1) * 22;   // element (ex, ez)
      const R* eL = e00 - 22;                                 // (ex-1, ez)
      const R* eB = e00 - EX * 22;                            // (ex, ez-1)
      const R* eBL = eB - 22;                                 // (ex-1, ez-1)
      const bool hasL = ex > 0, hasB = ez > 0;
      if (a.yV) {
        emit(2 * ex + 1, 2 * ez + 1, e00[16], e00[17], 0);   // centre: local node 8
        {                                                     // bottom edge midpoint: 6 of (ex,ez-1), 4
          R y0 = 0, y1 = 0;
          if (hasB) { y0 += eB[12]; y1 += eB[13]; }
          y0 += e00[8]; y1 += e00[9];
          emit(2 * ex + 1, 2 * ez, y0, y1, 1);
        }
        {                                                     // left edge midpoint: 5 of (ex-1,ez), 7
          R y0 = 0, y1 = 0;
          if (hasL) { y0 += eL[10]; y1 += eL[11]; }
          y0 += e00[14]; y1 += e00[15];
          emit(2 * ex, 2 * ez + 1, y0, y1, 2);
        }
        {                                                     // lower-left corner: 2, 3, 1, 0
          R y0 = 0, y1 = 0;
          if (hasB && hasL) { y0 += eBL[4]; y1 += eBL[5]; }
          if (hasB) { y0 += eB[6]; y1 += eB[7]; }
          if (hasL) { y0 += eL[2]; y1 += eL[3]; }
          y0 += e00[0]; y1 += e00[1];
          emit(2 * ex, 2 * ez, y0, y1, 3);
        }
      }
      if (a.yP) {                                             // pressure node (ex, ez): 2, 3, 1, 0
        R y = 0;
        if (hasB && hasL) y += eBL[18 + 2];
        if (hasB) y += eB[18 + 3];
        if (hasL) y += eL[18 + 1];
        y += e00[18 + 0];
        const int64_t n = (int64_t)ez * (g.nx + 1) + ex;
        a.yP[n] = (MODE == AM_RESID) ? a.bP[n] - y : y;
      }
    }
  } else if (lastx || lastz) {
    // right column ix = 2 nx (rows of this tile) and top row iz = 2 nz (columns of this tile,
    // the corner taken by the column)
    const int j0 = tid - TX * TZ, nj = NJ;
    if (a.yV) {
#pragma unroll
      for (int it = 0; it < 2; ++it) {                // the nodes whose vectors were prefetched
        const int j = j0 + it * nj;
        if (j < ncol_v + nrow_v) {
          if (j < ncol_v) node_generic(2 * g.nx, 2 * ez0 + j, 4 + it);
          else node_generic(2 * ex0 + (j - ncol_v), 2 * g.nz, 4 + it);
        }
      }
    }
    if (a.yP) {
      const int pz1 = lastz ? g.nz + 1 : ez0 + TZ;
      const int ncol = lastx ? pz1 - ez0 : 0;
      const int nrow = lastz ? (lastx ? g.nx - ex0 : TX) : 0;
      for (int j = j0; j < ncol + nrow; j += nj) {
        if (j < ncol) pnode_generic(g.nx, ez0 + j);
        else pnode_generic(ex0 + (j - ncol), g.nz);
      }
    }
  }
}

// diag(K): sum over incident elements of the element diagonal, ascending element order.
template <typename R>
__global__ void k_diag(LevelGeo g, const R* __restrict__ eta, R* __restrict__ diag) {
  pdl_entry();
  const int64_t nn = (int64_t)g.nnx * g.nnz;
  const double sx = 2.0 / g.hx, sz = 2.0 / g.hz, jac = g.hx * g.hz / 4.0;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    int ix = (int)(n % g.nnx), iz = (int)(n / g.nnx);
    int exs[2], ezs[2], nxe = 0, nze = 0;
    if (ix & 1) exs[nxe++] = ix >> 1;
    else { if (ix / 2 - 1 >= 0) exs[nxe++] = ix / 2 - 1; if (ix / 2 < g.nx) exs[nxe++] = ix / 2; }
    if (iz & 1) ezs[nze++] = iz >> 1;
    else { if (iz / 2 - 1 >= 0) ezs[nze++] = iz / 2 - 1; if (iz / 2 < g.nz) ezs[nze++] = iz / 2; }
    double d0 = 0, d1 = 0;
    for (int az = 0; az < nze; ++az)
      for (int ax = 0; ax < nxe; ++ax) {
        int k = q2_local_idx(ix - 2 * exs[ax], iz - 2 * ezs[az]);
        const R* eq = eta + ((int64_t)ezs[az] * g.nx + exs[ax]) * 9;
        for (int q = 0; q < 9; ++q) {
          double dx = sx * c_ref.dr[q * 9 + k], dz = sz * c_ref.dt[q * 9 + k];
          double e = (double)eq[q] * jac * c_ref.wq[q];
          d0 += e * (2 * dx * dx + dz * dz);
          d1 += e * (2 * dz * dz + dx * dx);
        }
      }
    diag[2 * n] = (R)d0;
    diag[2 * n + 1] = (R)d1;
  }
}

// coarse viscosity: mean of the 36 fine qpoint values of the 2x2 children (element constant)
template <typename R>
__global__ void k_coarsen_eta(LevelGeo gf, LevelGeo gc, const R* __restrict__ fine, R* __restrict__ coarse) {
  pdl_entry();
  const int64_t nel = (int64_t)gc.nx * gc.nz;
  const int fnx = gf.nx;
  const bool nested = nested_levels(gf, gc);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    int ex = (int)(e % gc.nx), ez = (int)(e / gc.nx);
    double s = 0;
    if (nested) {
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
          const R* f = fine + ((int64_t)(2 * ez + a) * fnx + (2 * ex + b)) * 9;
          for (int q = 0; q < 9; ++q) s += (double)f[q];
        }
      s /= 36.0;
    } else {
      // the mean over the coarse element of the fine elements' qpoint means, each weighted by its
      // overlap (coarse edges at e nf, fine edges at f nc, in units of L / (nf nc))
      auto range = [](int e, int nf, int nc, int* f0, int* f1) {
        *f0 = (int)(((int64_t)e * nf) / nc);
        *f1 = (int)(((int64_t)(e + 1) * nf + nc - 1) / nc) - 1;
        if (*f1 > nf - 1) *f1 = nf - 1;
      };
      auto overlap = [](int e, int f, int nf, int nc) {
        const int64_t a = std::max<int64_t>((int64_t)e * nf, (int64_t)f * nc);
        const int64_t b = std::min<int64_t>((int64_t)(e + 1) * nf, (int64_t)(f + 1) * nc);
        return b > a ? (double)(b - a) : 0.0;
      };
      int x0, x1, z0, z1;
      range(ex, gf.nx, gc.nx, &x0, &x1);
      range(ez, gf.nz, gc.nz, &z0, &z1);
      double wsum = 0;
      for (int fz = z0; fz <= z1; ++fz) {
        const double wz = overlap(ez, fz, gf.nz, gc.nz);
        for (int fx = x0; fx <= x1; ++fx) {
          const double w = wz * overlap(ex, fx, gf.nx, gc.nx);
          if (w == 0.0) continue;
          const R* f = fine + ((int64_t)fz * fnx + fx) * 9;
          double m = 0;
          for (int q = 0; q < 9; ++q) m += (double)f[q];
          s += w * (m / 9.0);
          wsum += w;
        }
      }
      s /= wsum;
    }
    R v = (R)s;
    for (int q = 0; q < 9; ++q) coarse[e * 9 + q] = v;
  }
}

// 1D Q2 restriction weights of coarse lattice node J from fine node 2J+o (o in -3..3)
MW_D double rw(int J, int o) {
  if (J & 1) return o == 0 ? 1.0 : ((o == -1 || o == 1) ? 0.75 : 0.0);
  if (o == 0) return 1.0;
  if (o == -1 || o == 1) return 0.375;
  if (o == -3 || o == 3) return -0.125;
  return 0.0;
}

// Full-weighting restriction of the fine residual to coarse node n (the transpose of the Q2
// prolongation below); with cheb_c also the coarse level's first Chebyshev step from a zero
// guess: x_c = d_c = (1/theta_c) D_c^-1 b_c.
// (no __restrict__: the cluster tail reads values written earlier in the same kernel)
// fetch(fz, fx, &v0, &v1) reads the residual pair of fine node (fx, fz) (global or shared memory).
template <typename R, typename Fetch>
MW_D void restrict_core(const LevelGeo& gf, const LevelGeo& gc, Fetch fetch, const uint8_t* fixc, R* bc, double c0,
                        bool cheb, const R* diag_c, R* xc, R* dc, int64_t n) {
  int I = (int)(n % gc.nnx), J = (int)(n / gc.nnx);
  // The nonzero taps lie at offsets -3, -1, 0, 1, 3 (the weight at +-2 is zero).  All stencil
  // values are loaded first (predicated), then summed in ascending offset order.
  constexpr int OFF[5] = {-3, -1, 0, 1, 3};
  R v0[5][5], v1[5][5];
#pragma unroll
  for (int tz = 0; tz < 5; ++tz)
#pragma unroll
    for (int tx = 0; tx < 5; ++tx) {
      const int fz = 2 * J + OFF[tz], fx = 2 * I + OFF[tx];
      const bool ok = rw(J, OFF[tz]) != 0.0 && rw(I, OFF[tx]) != 0.0 && fz >= 0 && fz < gf.nnz && fx >= 0 &&
                      fx < gf.nnx;
      v0[tz][tx] = R(0);
      v1[tz][tx] = R(0);
      if (ok) fetch(fz, fx, &v0[tz][tx], &v1[tz][tx]);
    }
  double s0 = 0, s1 = 0;
#pragma unroll
  for (int tz = 0; tz < 5; ++tz) {
    const double wz = rw(J, OFF[tz]);
    const int fz = 2 * J + OFF[tz];
    const bool okz = wz != 0.0 && fz >= 0 && fz < gf.nnz;
#pragma unroll
    for (int tx = 0; tx < 5; ++tx) {
      const double wx = rw(I, OFF[tx]);
      const int fx = 2 * I + OFF[tx];
      if (okz && wx != 0.0 && fx >= 0 && fx < gf.nnx) {
        s0 += wz * wx * (double)v0[tz][tx];
        s1 += wz * wx * (double)v1[tz][tx];
      }
    }
  }
  const R b0 = fixc[2 * n] ? R(0) : (R)s0, b1 = fixc[2 * n + 1] ? R(0) : (R)s1;
  bc[2 * n] = b0;
  bc[2 * n + 1] = b1;
  if (cheb) {
    const R x0 = R(c0) * b0 / diag_c[2 * n], x1 = R(c0) * b1 / diag_c[2 * n + 1];
    xc[2 * n] = x0; dc[2 * n] = x0;
    xc[2 * n + 1] = x1; dc[2 * n + 1] = x1;
  }
}

// 1D restriction taps of coarse node J (the transpose of pw_g): fine nodes idx with weights w,
// at most 10 (the fine nodes within the support of J's basis function, nf / nc <= 2)
constexpr int RMAXT = 10;
MW_D int restrict_taps_1d(int J, int nf, int nc, int* idx, double* w) {
  int k = 0;
  if (nested_1d(nf, nc)) {
    const int OFF[5] = {-3, -1, 0, 1, 3};
    for (int t = 0; t < 5; ++t) {
      const int i = 2 * J + OFF[t];
      const double v = rw(J, OFF[t]);
      if (v != 0.0 && i >= 0 && i <= 2 * nf) { idx[k] = i; w[k] = v; ++k; }
    }
    return k;
  }
  const int lo = J >= 2 ? (int)(((int64_t)(J - 2) * nf) / nc) : 0;
  int hi = (int)(((int64_t)(J + 2) * nf + nc - 1) / nc);
  if (hi > 2 * nf) hi = 2 * nf;
  for (int i = lo; i <= hi && k < RMAXT; ++i) {
    double q[3];
    const int E = q2_weights_1d(i, nf, nc, q);
    const int o = J - 2 * E;
    if (o >= 0 && o <= 2 && q[o] != 0.0) { idx[k] = i; w[k] = q[o]; ++k; }
  }
  return k;
}

// The restriction at coarse node n when a dimension is not nested: the same epilogue as
// restrict_core, the fine residual summed over the general taps (z outer, x inner)
template <typename R, typename Fetch>
MW_D void restrict_core_g(const LevelGeo& gf, const LevelGeo& gc, Fetch fetch, const uint8_t* fixc, R* bc, double c0,
                          bool cheb, const R* diag_c, R* xc, R* dc, int64_t n) {
  const int I = (int)(n % gc.nnx), J = (int)(n / gc.nnx);
  int ix[RMAXT], iz[RMAXT];
  double wx[RMAXT], wz[RMAXT];
  const int nx = restrict_taps_1d(I, gf.nx, gc.nx, ix, wx), nz = restrict_taps_1d(J, gf.nz, gc.nz, iz, wz);
  double s0 = 0, s1 = 0;
  for (int a = 0; a < nz; ++a)
    for (int b = 0; b < nx; ++b) {
      R v0, v1;
      fetch(iz[a], ix[b], &v0, &v1);
      s0 += wz[a] * wx[b] * (double)v0;
      s1 += wz[a] * wx[b] * (double)v1;
    }
  const R b0 = fixc[2 * n] ? R(0) : (R)s0, b1 = fixc[2 * n + 1] ? R(0) : (R)s1;
  bc[2 * n] = b0;
  bc[2 * n + 1] = b1;
  if (cheb) {
    const R x0 = R(c0) * b0 / diag_c[2 * n], x1 = R(c0) * b1 / diag_c[2 * n + 1];
    xc[2 * n] = x0; dc[2 * n] = x0;
    xc[2 * n + 1] = x1; dc[2 * n + 1] = x1;
  }
}

template <typename R>
MW_D void restrict_node(const LevelGeo& gf, const LevelGeo& gc, const R* rf, const uint8_t* fixc, R* bc, double c0,
                        bool cheb, const R* diag_c, R* xc, R* dc, int64_t n) {
  auto fetch = [&](int fz, int fx, R* a0, R* a1) {
    const int64_t m = (int64_t)fz * gf.nnx + fx;
    *a0 = rf[2 * m];
    *a1 = rf[2 * m + 1];
  };
  if (nested_levels(gf, gc)) restrict_core(gf, gc, fetch, fixc, bc, c0, cheb, diag_c, xc, dc, n);
  else restrict_core_g(gf, gc, fetch, fixc, bc, c0, cheb, diag_c, xc, dc, n);
}

// the restriction between levels that are not nested, one coarse node per thread
template <typename R>
__global__ void k_restrict_g(LevelGeo gf, LevelGeo gc, const R* __restrict__ rf, const uint8_t* __restrict__ fixc,
                             R* __restrict__ bc, const double* __restrict__ cheb_c, const R* __restrict__ diag_c,
                             R* __restrict__ xc, R* __restrict__ dc) {
  pdl_entry();
  const double c0 = cheb_c ? cheb_c[1] : 0.0;
  const int64_t nn = (int64_t)gc.nnx * gc.nnz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x)
    restrict_node(gf, gc, rf, fixc, bc, c0, cheb_c != nullptr, diag_c, xc, dc, n);
}

// The restriction over a tile of RTX x RTZ coarse nodes (one per thread): the fine residual the
// tile's stencils reach is staged in shared memory with coalesced loads (all issued before the
// stores), then each node sums its taps from there -- the same terms in the same order as
// restrict_node.
constexpr int RTX = 32, RTZ = 8;
constexpr int RFX = 2 * RTX + 5, RFZ = 2 * RTZ + 5;      // fine offsets -3 .. 2 (RT - 1) + 3

template <typename R>
__global__ void __launch_bounds__(RTX * RTZ) k_restrict(LevelGeo gf, LevelGeo gc, const R* __restrict__ rf,
                                                        const uint8_t* __restrict__ fixc, R* __restrict__ bc,
                                                        const double* __restrict__ cheb_c,
                                                        const R* __restrict__ diag_c, R* __restrict__ xc,
                                                        R* __restrict__ dc) {
  pdl_entry();
  typedef typename Vec2<R>::T R2;
  __shared__ R2 sr[RFZ * RFX];
  const double c0 = cheb_c ? cheb_c[1] : 0.0;
  const int I0 = blockIdx.x * RTX, J0 = blockIdx.y * RTZ;
  const int fx0 = 2 * I0 - 3, fz0 = 2 * J0 - 3;
  const int tid = threadIdx.x;
  constexpr int NL = (RFZ * RFX + RTX * RTZ - 1) / (RTX * RTZ);
  const R2* rf2 = reinterpret_cast<const R2*>(rf);
  R2 v[NL];
#pragma unroll
  for (int k = 0; k < NL; ++k) {
    const int i = tid + k * RTX * RTZ;
    const int lz = i / RFX, lx = i - lz * RFX;
    const int fx = fx0 + lx, fz = fz0 + lz;
    v[k].x = 0; v[k].y = 0;
    if (i < RFZ * RFX && fx >= 0 && fx < gf.nnx && fz >= 0 && fz < gf.nnz) v[k] = rf2[(int64_t)fz * gf.nnx + fx];
  }
#pragma unroll
  for (int k = 0; k < NL; ++k) {
    const int i = tid + k * RTX * RTZ;
    if (i < RFZ * RFX) sr[i] = v[k];
  }
  __syncthreads();
  const int I = I0 + tid % RTX, J = J0 + tid / RTX;
  if (I >= gc.nnx || J >= gc.nnz) return;
  auto fetch = [&](int fz, int fx, R* a0, R* a1) {
    const R2 t = sr[(fz - fz0) * RFX + (fx - fx0)];
    *a0 = t.x;
    *a1 = t.y;
  };
  restrict_core(gf, gc, fetch, fixc, bc, c0, cheb_c != nullptr, diag_c, xc, dc, (int64_t)J * gc.nnx + I);
}

// x_f += P x_c at fine node n (free dofs only)
template <typename R>
MW_D void prolong_node(const LevelGeo& gf, const LevelGeo& gc, const R* xc, const uint8_t* fixf, R* xf, int64_t n) {
  typedef typename Vec2<R>::T R2;
  const int ix = (int)(n % gf.nnx), iz = (int)(n / gf.nnx);
  double s0, s1;
  prolong_taps_g(gf, gc, ix, iz,
                 [&](int jz, int jx) { return reinterpret_cast<const R2*>(xc)[(int64_t)jz * gc.nnx + jx]; }, &s0, &s1);
  if (!fixf[2 * n]) xf[2 * n] += (R)s0;
  if (!fixf[2 * n + 1]) xf[2 * n + 1] += (R)s1;
}

// the prolongation between levels that are not nested, one fine node per thread
template <typename R>
__global__ void k_prolong_g(LevelGeo gf, LevelGeo gc, const R* __restrict__ xc, const uint8_t* __restrict__ fixf,
                            R* __restrict__ xf) {
  pdl_entry();
  const int64_t nn = (int64_t)gf.nnx * gf.nnz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x)
    prolong_node(gf, gc, xc, fixf, xf, n);
}

// The prolongation over a tile of PTX x PTZ fine nodes (one per thread): the coarse values the tile
// reaches (coarse x from X0/2 to X0/2 + PTX/2, z likewise) are staged in shared memory, then each
// node sums its taps from there in the order of prolong_node and updates its (u, w) pair with one
// vector load and store.
constexpr int PTX = 32, PTZ = 8;
constexpr int PCX = PTX / 2 + 1, PCZ = PTZ / 2 + 1;

template <typename R>
__global__ void __launch_bounds__(PTX * PTZ) k_prolong_add(LevelGeo gf, LevelGeo gc, const R* __restrict__ xc,
                                                           const uint8_t* __restrict__ fixf, R* __restrict__ xf) {
  pdl_entry();
  typedef typename Vec2<R>::T R2;
  __shared__ R2 sc2[PCZ * PCX];
  const int X0 = blockIdx.x * PTX, Z0 = blockIdx.y * PTZ;
  const int cx0 = X0 / 2, cz0 = Z0 / 2;
  const int tid = threadIdx.x;
  if (tid < PCZ * PCX) {
    const int jz = tid / PCX, jx = tid - jz * PCX;
    const int cx = cx0 + jx, cz = cz0 + jz;
    R2 v;
    v.x = 0; v.y = 0;
    if (cx < gc.nnx && cz < gc.nnz) v = reinterpret_cast<const R2*>(xc)[(int64_t)cz * gc.nnx + cx];
    sc2[tid] = v;
  }
  __syncthreads();
  const int ix = X0 + tid % PTX, iz = Z0 + tid / PTX;
  if (ix >= gf.nnx || iz >= gf.nnz) return;
  const int64_t n = (int64_t)iz * gf.nnx + ix;
  const uchar2 ff = reinterpret_cast<const uchar2*>(fixf)[n];
  R2 x = reinterpret_cast<const R2*>(xf)[n];
  double s0, s1;
  prolong_taps(ix, iz, [&](int jz, int jx) { return sc2[(jz - cz0) * PCX + (jx - cx0)]; }, &s0, &s1);
  if (!ff.x) x.x += (R)s0;
  if (!ff.y) x.y += (R)s1;
  reinterpret_cast<R2*>(xf)[n] = x;
}

template <typename R>
__global__ void k_fix_coarse(LevelGeo gf, LevelGeo gc, const uint8_t* __restrict__ fixf, uint8_t* __restrict__ fixc) {
  pdl_entry();
  // a coarse dof is fixed when the coincident fine dof is fixed (same boundaries); on a level that
  // is not nested, the fine node nearest to the coarse one (on the same side of the box: box
  // conditions depend only on the side)
  const int64_t nn = (int64_t)gc.nnx * gc.nnz;
  const int fnnx = gf.nnx;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    int I = (int)(n % gc.nnx), J = (int)(n / gc.nnx);
    const int fi = nested_1d(gf.nx, gc.nx) ? 2 * I : (int)(((int64_t)I * gf.nx + gc.nx / 2) / gc.nx);
    const int fj = nested_1d(gf.nz, gc.nz) ? 2 * J : (int)(((int64_t)J * gf.nz + gc.nz / 2) / gc.nz);
    int64_t m = (int64_t)fj * fnnx + fi;
    fixc[2 * n] = fixf[2 * m];
    fixc[2 * n + 1] = fixf[2 * m + 1];
  }
}

// ---------------------------------------------------------------- BLAS-1 with device scalars
template <typename R>
__global__ void k_dot_partial(int64_t n, const R* __restrict__ x, const R* __restrict__ y, double* __restrict__ part) {
  pdl_entry();
  __shared__ double sh[32];
  double v = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v += (double)x[i] * (double)y[i];
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

__global__ void k_dot_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
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

// y += sgn * (num/den) * x      (scalars on the device)
template <typename R, typename S>
__global__ void k_axpy_ratio(int64_t n, const double* __restrict__ num, const double* __restrict__ den, double sgn,
                             const S* __restrict__ x, R* __restrict__ y) {
  pdl_entry();
  const double a = sgn * (*num / *den);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (R)((double)y[i] + a * (double)x[i]);
}

// p = z + (num/den) * p
template <typename R>
__global__ void k_xpby_ratio(int64_t n, const R* __restrict__ z, const double* __restrict__ num,
                             const double* __restrict__ den, R* __restrict__ p) {
  pdl_entry();
  const double b = *num / *den;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (R)((double)z[i] + b * (double)p[i]);
}

template <typename R>
__global__ void k_axpy(int64_t n, double a, const R* __restrict__ x, R* __restrict__ y) {
  pdl_entry();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (R)((double)y[i] + a * (double)x[i]);
}

template <typename R, typename S>
__global__ void k_copy(int64_t n, const S* __restrict__ x, R* __restrict__ y) {
  pdl_entry();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (R)x[i];
}

template <typename R>
__global__ void k_set(int64_t n, R v, R* __restrict__ y) {
  pdl_entry();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) y[i] = v;
}

// x = c * Dinv * b ; d = x   (first Chebyshev step from a zero guess)
template <typename R>
__global__ void k_cheb_first(int64_t n, const double* __restrict__ cheb, const R* __restrict__ b,
                             const R* __restrict__ diag, R* __restrict__ x, R* __restrict__ d) {
  pdl_entry();
  const R c = (R)cheb[1];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    R v = c * b[i] / diag[i];
    x[i] = v; d[i] = v;
  }
}

// power iteration helpers for lambda_max(D^-1 K)
template <typename R>
__global__ void k_scale_dinv_norm(int64_t n, const R* __restrict__ y, const R* __restrict__ diag,
                                  const double* __restrict__ nrm2, R* __restrict__ x) {
  pdl_entry();
  const double inv = 1.0 / sqrt(fmax(*nrm2, 1e-300));
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (R)((double)y[i] / (double)diag[i] * inv);
}

template <typename R>
__global__ void k_dinv(int64_t n, const R* __restrict__ y, const R* __restrict__ diag, R* __restrict__ x) {
  pdl_entry();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = y[i] / diag[i];
}

// Chebyshev coefficients from lambda_max (stored at lam[0] as ||D^-1 K x||^2 with ||x|| = 1).
__global__ void k_cheb_coeffs(const double* __restrict__ lam2, int degree, double ratio, double safety,
                              double* __restrict__ coef) {
  pdl_entry();
  if (threadIdx.x || blockIdx.x) return;
  double lmax = sqrt(fmax(*lam2, 1e-300)) * safety;
  double lmin = lmax / ratio;
  double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
  double rho = 1.0 / sigma;
  coef[0] = 0.0;                             // step 0: d = (1/theta) D^-1 r
  coef[1] = 1.0 / theta;
  for (int k = 1; k < degree; ++k) {
    double rn = 1.0 / (2.0 * sigma - rho);
    coef[2 * k] = rn * rho;                  // c1: d = c1 d + c2 D^-1 r
    coef[2 * k + 1] = 2.0 * rn / delta;
    rho = rn;
  }
}

// ---------------------------------------------------------------- coarsest level: dense inverse
template <typename R>
__global__ void k_dense_assemble(LevelGeo g, const R* __restrict__ eta, const uint8_t* __restrict__ fix,
                                 double* __restrict__ A) {
  pdl_entry();
  const int nd = 2 * g.nnx * g.nnz;
  for (int i = threadIdx.x; i < nd * nd; i += blockDim.x) A[i] = 0.0;
  __syncthreads();
  const double sx = 2.0 / g.hx, sz = 2.0 / g.hz, jac = g.hx * g.hz / 4.0;
  for (int e = 0; e < g.nx * g.nz; ++e) {          // elements in order: deterministic sums
    int ex = e % g.nx, ez = e / g.nx;
    for (int t = threadIdx.x; t < 324; t += blockDim.x) {
      int ii = t / 18, jj = t % 18;
      int ki = ii >> 1, ci = ii & 1, kj = jj >> 1, cj = jj & 1;
      double v = 0;
      for (int q = 0; q < 9; ++q) {
        double dxi = sx * c_ref.dr[q * 9 + ki], dzi = sz * c_ref.dt[q * 9 + ki];
        double dxj = sx * c_ref.dr[q * 9 + kj], dzj = sz * c_ref.dt[q * 9 + kj];
        double bb;
        if (ci == 0 && cj == 0) bb = 2 * dxi * dxj + dzi * dzj;
        else if (ci == 0) bb = dzi * dxj;
        else if (cj == 0) bb = dxi * dzj;
        else bb = 2 * dzi * dzj + dxi * dxj;
        v += bb * (double)eta[(int64_t)e * 9 + q] * jac * c_ref.wq[q];
      }
      int gi = 2 * (int)q2_node(ex, ez, ki, g.nnx) + ci, gj = 2 * (int)q2_node(ex, ez, kj, g.nnx) + cj;
      A[(int64_t)gi * nd + gj] += v;
    }
    __syncthreads();
  }
  // Dirichlet elimination: zero fixed rows/cols except the diagonal
  for (int t = threadIdx.x; t < nd * nd; t += blockDim.x) {
    int i = t / nd, j = t % nd;
    if (i != j && (fix[i] || fix[j])) A[t] = 0.0;
  }
}

// In-place Gauss-Jordan inversion of an SPD matrix, one CTA.
// Same inversion with the whole matrix held in shared memory (nd*nd doubles + a column).
__global__ void k_gauss_jordan_smem(int nd, double* __restrict__ Ag) {
  pdl_entry();
  extern __shared__ double sm[];
  double* A = sm;
  double* col = sm + (size_t)nd * nd;
  for (int t = threadIdx.x; t < nd * nd; t += blockDim.x) A[t] = Ag[t];
  // rows over warps, columns over lanes: no index division in the elimination sweep
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int k = 0; k < nd; ++k) {
    __syncthreads();
    for (int i = threadIdx.x; i < nd; i += blockDim.x) col[i] = A[i * nd + k];
    __syncthreads();
    const double piv = 1.0 / col[k];
    for (int j = threadIdx.x; j < nd; j += blockDim.x) A[k * nd + j] = (j == k ? 1.0 : A[k * nd + j]) * piv;
    __syncthreads();
    const double* rk = A + k * nd;
    for (int i = warp; i < nd; i += nwarp) {
      if (i == k) continue;
      const double ci = col[i];
      double* ri = A + i * nd;
      for (int j = lane; j < nd; j += 32) ri[j] = (j == k ? 0.0 : ri[j]) - ci * rk[j];
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nd * nd; t += blockDim.x) Ag[t] = A[t];
}

__global__ void k_gauss_jordan(int nd, double* __restrict__ A) {
  pdl_entry();
  extern __shared__ double col[];
  for (int k = 0; k < nd; ++k) {
    __syncthreads();
    for (int i = threadIdx.x; i < nd; i += blockDim.x) col[i] = A[(int64_t)i * nd + k];
    __syncthreads();
    const double piv = 1.0 / col[k];
    for (int j = threadIdx.x; j < nd; j += blockDim.x) A[(int64_t)k * nd + j] = (j == k ? 1.0 : A[(int64_t)k * nd + j]) * piv;
    __syncthreads();
    for (int t = threadIdx.x; t < nd * nd; t += blockDim.x) {
      int i = t / nd, j = t % nd;
      if (i == k) continue;
      double f = col[i];
      double akj = A[(int64_t)k * nd + j];
      A[t] = (j == k ? 0.0 : A[t]) - f * akj;
    }
  }
}

template <typename R>
__global__ void k_dense_matvec(int nd, const double* __restrict__ Ainv, const R* __restrict__ b, R* __restrict__ x) {
  pdl_entry();
  // one warp per row
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nd) return;
  double s = 0;
  for (int j = lane; j < nd; j += 32) s += Ainv[(int64_t)warp * nd + j] * (double)b[j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) x[warp] = (R)s;
}

// ---------------------------------------------------------------- pressure mass matrices
// y = M_w p with M_w the Q1 mass matrix weighted per element by w_e (w = NULL -> 1):
// M_el = sum_q N_P N_P^T JxW (build_matrix_stokes.py:147), M_eta = M_el / eta_e (:264).
__global__ void k_mass_apply(LevelGeo g, const double* __restrict__ w, const double* __restrict__ p,
                             double* __restrict__ y) {
  pdl_entry();
  const int ncx = g.nx + 1;
  const int64_t np = (int64_t)ncx * (g.nz + 1);
  const double jac = g.hx * g.hz / 4.0;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < np; n += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(n % ncx), j = (int)(n / ncx);
    const int exs[4] = {i - 1, i, i - 1, i};
    const int ezs[4] = {j - 1, j - 1, j, j};
    const int kk[4] = {2, 3, 1, 0};
    double acc = 0;
    for (int s = 0; s < 4; ++s) {
      int ex = exs[s], ez = ezs[s];
      if (ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
      int64_t e = (int64_t)ez * g.nx + ex;
      double we = w ? w[e] : 1.0;
      double v = 0;
      for (int k2 = 0; k2 < 4; ++k2) {
        double m = 0;
        for (int q = 0; q < 9; ++q) m += c_ref.NP[q * 4 + kk[s]] * c_ref.NP[q * 4 + k2] * jac * c_ref.wq[q];
        v += m * p[q1_node(ex, ez, k2, g.nx)];
      }
      acc += we * v;
    }
    y[n] = acc;
  }
}

__global__ void k_mass_diag(LevelGeo g, const double* __restrict__ w, double* __restrict__ d) {
  pdl_entry();
  const int ncx = g.nx + 1;
  const int64_t np = (int64_t)ncx * (g.nz + 1);
  const double jac = g.hx * g.hz / 4.0;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < np; n += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(n % ncx), j = (int)(n / ncx);
    const int exs[4] = {i - 1, i, i - 1, i};
    const int ezs[4] = {j - 1, j - 1, j, j};
    const int kk[4] = {2, 3, 1, 0};
    double acc = 0;
    for (int s = 0; s < 4; ++s) {
      int ex = exs[s], ez = ezs[s];
      if (ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
      int64_t e = (int64_t)ez * g.nx + ex;
      double m = 0;
      for (int q = 0; q < 9; ++q) m += c_ref.NP[q * 4 + kk[s]] * c_ref.NP[q * 4 + kk[s]] * jac * c_ref.wq[q];
      acc += (w ? w[e] : 1.0) * m;
    }
    d[n] = acc;
  }
}

// the Q1 element mass matrix of the uniform box, Me[a * 4 + c] = sum_q N_a N_c JxW
MW_D double mass_entry(const LevelGeo& g, int a, int c) {
  const double jac = g.hx * g.hz / 4.0;
  double m = 0;
  for (int q = 0; q < 9; ++q) m += c_ref.NP[q * 4 + a] * c_ref.NP[q * 4 + c] * jac * c_ref.wq[q];
  return m;
}

// One fused Chebyshev-Jacobi step for M_w x = b:  r = b - M_w x_in ; d = c1 d + c2 D^-1 r ;
// x_out = x_in + d.  `first` means x_in = 0 (no product, no old direction).  For Q1 mass matrices
// with positive element weights, lambda(D^-1 M_w) lies in [0.25, 2.25] whatever the weights
// (element-by-element bound; the exactly integrated bilinear element matrix has D_e^-1 M_e eigenvalues
// 9/4, 3/4, 3/4, 1/4), so the coefficients are fixed and need no dot products.
// (the step at pressure node n; Me: the element mass matrix)
MW_D void mass_cheb_node(const LevelGeo& g, const double* w, const double* b, const double* xin, double* xout,
                         double* d, const double* dg, double c1, double c2, int first, const double* Me, int64_t n) {
  const int ncx = g.nx + 1;
  double y = 0;
  if (!first) {
    const int i = (int)(n % ncx), j = (int)(n / ncx);
    // incident elements (j-1,i-1) k=2, (j-1,i) k=3, (j,i-1) k=1, (j,i) k=0
    for (int s = 0; s < 4; ++s) {
      const int ex = (s & 1) ? i : i - 1, ez = (s & 2) ? j : j - 1;
      if (ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
      const int kl = s == 0 ? 2 : (s == 1 ? 3 : (s == 2 ? 1 : 0));
      const int64_t e = (int64_t)ez * g.nx + ex;
      double v = 0;
      for (int k2 = 0; k2 < 4; ++k2) v += Me[kl * 4 + k2] * xin[q1_node(ex, ez, k2, g.nx)];
      y += (w ? w[e] : 1.0) * v;
    }
  }
  const double r = b[n] - y;
  const double dn = first ? c2 * r / dg[n] : c1 * d[n] + c2 * r / dg[n];
  d[n] = dn;
  xout[n] = (first ? 0.0 : xin[n]) + dn;
}

__global__ void k_mass_cheb(LevelGeo g, const double* __restrict__ w, const double* __restrict__ b,
                            const double* __restrict__ xin, double* __restrict__ xout, double* __restrict__ d,
                            const double* __restrict__ dg, double c1, double c2, int first) {
  pdl_entry();
  __shared__ double Me[16];
  if (threadIdx.x < 16) Me[threadIdx.x] = mass_entry(g, threadIdx.x / 4, threadIdx.x % 4);
  __syncthreads();
  const int64_t np = (int64_t)(g.nx + 1) * (g.nz + 1);
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < np; n += (int64_t)gridDim.x * blockDim.x)
    mass_cheb_node(g, w, b, xin, xout, d, dg, c1, c2, first, Me, n);
}

// The grid-wide sum of one value per thread, finished in the same launch: block partials in
// part[block], the last block to arrive adds them in block order into *out and resets the counter
// (threadfence + arrival counter).  Called once, by every thread, at the end of a kernel.
MW_D void grid_sum_last(double v, double* part, unsigned* counter, double* out) {
  __shared__ double sh[32];
  __shared__ bool last;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) {
      part[blockIdx.x] = v;
      __threadfence();
      last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) t += ((volatile double*)part)[i];
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if (lane == 0) sh[wid] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh[k];
    out[0] = s;
    *counter = 0u;
  }
}

// Deterministic single-launch dot product: block partials, then the last block to finish sums
// them in block order (threadfence + arrival counter, reset for the next call).
template <typename R>
__global__ void k_dot1(int64_t n, const R* __restrict__ x, const R* __restrict__ y, double* __restrict__ part,
                       unsigned* __restrict__ counter, double* __restrict__ out) {
  pdl_entry();
  double v = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v += (double)x[i] * (double)y[i];
  grid_sum_last(v, part, counter, out);
}

// x += (num/den) p ; r -= (num/den) Ap, and (r, r) of the new residual into *rr, summed exactly as
// k_dot1 sums it on the same grid (one launch for the CG step and its convergence norm)
template <typename R>
__global__ void k_pcg_update_rr(int64_t n, const double* __restrict__ num, const double* __restrict__ den,
                                const R* __restrict__ p, const R* __restrict__ Ap, R* __restrict__ x,
                                R* __restrict__ r, double* __restrict__ part, unsigned* __restrict__ counter,
                                double* __restrict__ rr) {
  pdl_entry();
  const double a = *num / *den;
  double v = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = (R)((double)x[i] + a * (double)p[i]);
    const R ri = (R)((double)r[i] - a * (double)Ap[i]);
    r[i] = ri;
    v += (double)ri * (double)ri;
  }
  grid_sum_last(v, part, counter, rr);
}


// element weights 1/eta_e for M_eta (eta_e = mean of the qpoint viscosities of the element)
__global__ void k_inv_eta_e(int64_t nel, const double* __restrict__ etaq, const double* __restrict__ eta_e,
                            double* __restrict__ w) {
  pdl_entry();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    double v;
    if (eta_e) v = eta_e[e];
    else { v = 0; for (int q = 0; q < 9; ++q) v += etaq[e * 9 + q]; v /= 9.0; }
    w[e] = 1.0 / v;
  }
}

// remove the mean (pressure null space of a closed box): x -= sum(x)/n
__global__ void k_sub_mean(int64_t n, const double* __restrict__ sum, double* __restrict__ x) {
  pdl_entry();
  const double m = *sum / (double)n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] -= m;
}

__global__ void k_sum_partial(int64_t n, const double* __restrict__ x, double* __restrict__ part) {
  pdl_entry();
  __shared__ double sh[32];
  double v = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) v += x[i];
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

// ================================================================= solver object
constexpr int NB = 1184;          // reduction partials: up to 8 CTAs per SM

// CTAs of a reduction over n values: enough to keep HBM busy on long vectors (at least 4 values
// per thread), one on short ones
static int nb_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(NB, (n + 1023) / 1024)); }
constexpr int MAXLEV = 12;
constexpr int MAXDEG = 8;
constexpr int MAX_TAIL = 6;       // levels of the one-CTA V-cycle tail

template <typename R>
struct Level {
  LevelGeo g;
  int64_t nn, ndof, nel;
  R *eta, *diag, *x, *b, *r, *d, *t;
  uint8_t* fix;
  double* cheb;       // 2*MAXDEG coefficients
  int deg;            // Chebyshev steps per smoothing sweep on this level
  double* lam2;
  R* ev;              // power-iteration vector, kept between viscosity updates (warm start)
  bool ev_ready;
};

struct Arena {
  char* base;
  size_t off, cap;
  bool dry;
  void* take(size_t bytes) {
    off = (off + 255) & ~size_t(255);
    void* p = dry ? nullptr : base + off;
    off += bytes;
    return p;
  }
};

template <typename R>
struct Hierarchy {
  int nlev = 0;
  Level<R> L[MAXLEV];
  double* Ainv = nullptr;    // coarsest dense inverse (double)
  int nd = 0;
  bool dense = true;
  int tail0 = 0;             // first level of the cluster V-cycle tail (0: none)
  int64_t tail_len = 0;      // element products of its largest level (18 per element)
  R* tail_ye = nullptr;      // their global scratch
};

}  // namespace mw

struct mw_stokes {
  mw::LevelGeo fine;
  mw_stokes_params prm;
  mw::Hierarchy<double> H64;
  mw::Hierarchy<float> H32;
  bool has64 = false, has32 = false;
  // fine-level solver vectors (double): Uzawa and FP64 residuals
  double *V, *P, *f, *h, *z, *rP, *wP, *dP, *Gd, *GTz, *RV, *RP, *tP, *tP2, *minv_w, *mdiag, *medi;
  double *cV, *cP;       // refinement corrections
  double* diag64;        // assembled diag(K) of the fine level, FP64
  bool dirty64 = true, dirty32 = true;
  double* etae_w;        // 1/eta_e per element (M_eta weights)
  double* red;           // reduction partials
  double* sc;            // device scalars
  unsigned* counter;     // arrival counter of the single-launch dot products
  // inner PCG vectors (precision of the hierarchy): x, r, z, p, Ap
  double *pc64[5];
  float *pc32[5];
  const uint8_t* fixV;   // fine fixed mask (caller's)
  double* etaq64;        // fine viscosity (double copy)
  float* etaq32;
  mw_solve_info last;
  // Launch-bound sequences (V-cycles, mass-matrix Chebyshev solves) are recorded once into CUDA
  // graphs and replayed.  Capture needs a stream other than the legacy default stream, so the
  // solver works on its own non-blocking stream, ordered after / before the caller's stream by
  // events.  The graphs stay valid across viscosity updates (they read the coefficients through
  // device pointers that never move).
  struct GraphEntry {
    int kind;
    std::vector<void*> before, after;
    cudaGraphExec_t exec;
  };
  std::vector<GraphEntry> graphs;
  bool use_graphs = true;
  bool device_loops = true;    // loops as graph conditional nodes (no host synchronisation)
  cudaStream_t ws = nullptr;
  cudaStream_t bs[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};   // capture streams of loop bodies
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // side branch of the hierarchy setup (the coarsest level's dense inverse)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  ~mw_stokes() {
    for (auto& e : graphs) cudaGraphExecDestroy(e.exec);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
    if (ws) cudaStreamDestroy(ws);
    for (auto b : bs)
      if (b) cudaStreamDestroy(b);
  }
};

namespace mw {

template <typename R>
static void plan_levels(Hierarchy<R>& H, const LevelGeo& fine, const mw_stokes_params& prm) {
  H.nlev = 0;
  LevelGeo g = fine;
  while (true) {
    Level<R>& l = H.L[H.nlev++];
    l.g = g;
    l.deg = (H.nlev == 1 || prm.cheb_degree_coarse <= 0) ? prm.cheb_degree : prm.cheb_degree_coarse;
    l.nn = (int64_t)g.nnx * g.nnz; l.ndof = 2 * l.nn; l.nel = (int64_t)g.nx * g.nz;
    // even element counts halve (nested levels); odd ones, with coarsen_odd, go to ceil(n / 2)
    // elements over the same box (a level that is not nested in this one)
    const bool odd_ok = prm.coarsen_odd != 0;
    const int cx = (g.nx % 2 == 0) ? g.nx / 2 : (odd_ok ? (g.nx + 1) / 2 : 0);
    const int cz = (g.nz % 2 == 0) ? g.nz / 2 : (odd_ok ? (g.nz + 1) / 2 : 0);
    bool can = cx > 0 && cz > 0 && cx < g.nx && cz < g.nz && cx >= prm.coarse_min && cz >= prm.coarse_min &&
               H.nlev < MAXLEV && (l.nel > (int64_t)prm.coarse_min * prm.coarse_min);
    // below coarse_min, down to 2 elements a side, while this level has more unknowns than the
    // one-CTA shared-memory inverse takes (coarse_dense_max): a 6 x 6 coarsest level (338
    // unknowns) inverted through global memory took most of a small model's step
    if (!can && prm.coarse_dense_max > 0 && l.ndof > prm.coarse_dense_max && cx >= 2 && cz >= 2 && cx < g.nx &&
        cz < g.nz && H.nlev < MAXLEV)
      can = true;
    if (!can) break;
    LevelGeo c = g;
    c.nx = cx; c.nz = cz; c.nnx = 2 * c.nx + 1; c.nnz = 2 * c.nz + 1;
    c.hx = g.nx == 2 * cx ? 2 * g.hx : g.hx * g.nx / cx;
    c.hz = g.nz == 2 * cz ? 2 * g.hz : g.hz * g.nz / cz;
    g = c;
  }
  const Level<R>& lc = H.L[H.nlev - 1];
  H.nd = (int)lc.ndof;
  H.dense = H.nd <= prm.dense_max;
  // the one-CTA tail: from the first level (below the fine one) with at most tail_nel elements
  H.tail0 = 0;
  H.tail_len = 0;
  if (prm.tail_nel > 0)
    for (int l = 1; l < H.nlev; ++l)
      if (H.L[l].nel <= prm.tail_nel && H.nlev - l <= MAX_TAIL) { H.tail0 = l; break; }
  for (int l = H.tail0; H.tail0 && l < H.nlev; ++l) H.tail_len = std::max(H.tail_len, H.L[l].nel * 18);
}



template <typename R>
static void carve(Hierarchy<R>& H, Arena& A, const uint8_t* fine_fix) {
  for (int l = 0; l < H.nlev; ++l) {
    Level<R>& L = H.L[l];
    L.eta = (R*)A.take(sizeof(R) * L.nel * 9);
    L.diag = (R*)A.take(sizeof(R) * L.ndof);
    L.x = (R*)A.take(sizeof(R) * L.ndof);
    L.b = (R*)A.take(sizeof(R) * L.ndof);
    L.r = (R*)A.take(sizeof(R) * L.ndof);
    L.d = (R*)A.take(sizeof(R) * L.ndof);
    L.t = (R*)A.take(sizeof(R) * L.ndof);
    L.fix = l == 0 ? const_cast<uint8_t*>(fine_fix) : (uint8_t*)A.take(L.ndof);
    L.cheb = (double*)A.take(sizeof(double) * 2 * MAXDEG);
    L.lam2 = (double*)A.take(sizeof(double) * 4);
    L.ev = (R*)A.take(sizeof(R) * L.ndof);
    L.ev_ready = false;
  }
  H.Ainv = H.dense ? (double*)A.take(sizeof(double) * (size_t)H.nd * H.nd) : nullptr;
  H.tail_ye = H.tail0 ? (R*)A.take(sizeof(R) * H.tail_len) : nullptr;
}

static size_t layout(mw_stokes* S, Arena& A) {
  const LevelGeo& g = S->fine;
  const int64_t nv = 2LL * g.nnx * g.nnz, np = (int64_t)(g.nx + 1) * (g.nz + 1), nel = (int64_t)g.nx * g.nz;
  double** dv[] = {&S->V, &S->z, &S->f, &S->Gd, &S->RV, &S->cV, &S->diag64};
  for (auto p : dv) *p = (double*)A.take(sizeof(double) * nv);
  double** pv[] = {&S->P, &S->h, &S->rP, &S->wP, &S->dP, &S->GTz, &S->RP, &S->tP, &S->tP2, &S->minv_w, &S->mdiag,
                   &S->medi, &S->cP};
  for (auto p : pv) *p = (double*)A.take(sizeof(double) * np);
  S->etae_w = (double*)A.take(sizeof(double) * nel);
  S->red = (double*)A.take(sizeof(double) * NB * 4);
  S->sc = (double*)A.take(sizeof(double) * 256);
  S->counter = (unsigned*)A.take(sizeof(unsigned) * 4);
  if (S->has64) {
    for (int i = 0; i < 5; ++i) S->pc64[i] = (double*)A.take(sizeof(double) * nv);
    carve(S->H64, A, S->fixV);
    S->etaq64 = S->H64.L[0].eta;
  } else {
    S->etaq64 = (double*)A.take(sizeof(double) * nel * 9);
  }
  if (S->has32) {
    for (int i = 0; i < 5; ++i) S->pc32[i] = (float*)A.take(sizeof(float) * nv);
    carve(S->H32, A, S->fixV);
    S->etaq32 = S->H32.L[0].eta;
  }
  return A.off + 256;
}

// ---------------------------------------------------------------- launch helpers
template <typename R, int MODE>
static void launch_apply(const LevelGeo& g, const ApplyArgs<R>& a, cudaStream_t s) {
  dim3 grid((g.nx + TX - 1) / TX, (g.nz + TZ - 1) / TZ);
  pdl_launch(k_apply<R, MODE>, grid, APPLY_THREADS, 0, s, g, a);
}

template <typename R>
static ApplyArgs<R> args0() {
  ApplyArgs<R> a;
  memset(&a, 0, sizeof(a));
  return a;
}

template <typename R>
static void dot(mw_stokes* S, int64_t n, const R* x, const R* y, double* out, cudaStream_t s) {
  pdl_launch(k_dot1<R>, nb_for(n), 256, 0, s, n, x, y, S->red, S->counter, out);
}

static void dsum(mw_stokes* S, int64_t n, const double* x, double* out, cudaStream_t s) {
  const int nb = nb_for(n);
  pdl_launch(k_sum_partial, nb, 256, 0, s, n, x, S->red);
  pdl_launch(k_dot_final, 1, 256, 0, s, S->red, nb, out);
}

// y = G p (b == null) or b - G p on the fine level; y = G^T u
static void grad_p(mw_stokes* S, const double* p, const double* b, double* y, cudaStream_t s) {
  const LevelGeo& g = S->fine;
  dim3 grid((g.nnx + 127) / 128, std::min(g.nnz, 65535));
  pdl_launch(k_grad_p, grid, 128, 0, s, g, p, S->fixV, b, y);
}
static void div_u(mw_stokes* S, const double* u, double* y, cudaStream_t s) {
  const LevelGeo& g = S->fine;
  dim3 grid((g.nx + 1 + 127) / 128, std::min(g.nz + 1, 65535));
  pdl_launch(k_div_u, grid, 128, 0, s, g, u, S->fixV, y);
}

template <typename R>
static void k_only_apply(const Level<R>& L, const R* x, R* y, cudaStream_t s) {
  ApplyArgs<R> a = args0<R>();
  a.u = x; a.eta = L.eta; a.fix = L.fix; a.diag = L.diag; a.yV = y;
  launch_apply<R, AM_APPLY>(L.g, a, s);
}

// ---------------------------------------------------------------- coarse levels in one cluster
// The levels with at most tail_nel elements take part in every V-cycle as one launch of one thread
// block cluster (k_vtail): smoothing, residual, restriction, the coarsest solve and prolongation
// run as phases separated by cluster barriers (release / acquire at cluster scope, which orders
// the global-memory writes of one phase before the reads of the next on every SM of the cluster),
// in place of about six latency-bound launches per level.  Each phase repeats the arithmetic of the
// multi-launch path in the same order -- the same element products, node sums over the incident
// elements in ascending element order, the same epilogues, the shared restriction and
// prolongation bodies -- so both paths give identical results.  Pointers written in one phase and
// read in a later one carry no __restrict__, so their loads stay on the coherent path.
constexpr int TAIL_CLUSTER = 8;

MW_D void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

MW_D unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
template <typename R>
struct TailLevel {
  LevelGeo g;
  const R* eta;
  const uint8_t* fix;
  const R* diag;
  R *x, *t, *b, *r, *d;
  const double* cheb;
  int deg;
};

template <typename R>
struct TailArgs {
  TailLevel<R> L[MAX_TAIL];
  int n;               // tail levels (the last one is the coarsest)
  int first_done;      // the first tail level's x = d were written by the restriction into it
  int dense, nd;       // coarsest level: dense inverse Ainv (nd unknowns), else MAXDEG smoothing
  const double* Ainv;
  R* ye;               // element products (global scratch, 18 per element of the largest level)
  R* out_x;            // shared-memory tail: where the first level's final x goes (the buffer the
                       // host's record of the pointer swaps names)
};

struct ClusterBarrier {
  MW_D void operator()() const { cluster_barrier(); }
};
struct BlockBarrier {
  MW_D void operator()() const { __syncthreads(); }
};

template <typename R>
constexpr int tail_threads() { return sizeof(R) == 4 ? 512 : 256; }

// One operator apply of tail level L on u: AM_RESID writes r = b - K u, AM_CHEB the Chebyshev
// step (d, xo) with coefficient pair cheb.  Element products go through the global scratch sye;
// this is thread t0 of the nt threads of the cluster.
template <typename R, int MODE, typename B>
MW_D void tail_apply(const TailLevel<R>& L, const R* u, R* xo, const double* cheb, R* sye, int t0, int nt,
                     const B& barrier) {
  typedef typename Vec2<R>::T R2;
  const LevelGeo& g = L.g;
  const int nel = g.nx * g.nz;
  const R sxe = R(2.0 / g.hx), sze = R(2.0 / g.hz), jace = R(g.hx * g.hz / 4.0), se = R(g.s);
  for (int e = t0; e < nel; e += nt) {
    const int ex = e % g.nx, ez = e / g.nx;
    __align__(16) R ue[18];
    R pe[4] = {R(0), R(0), R(0), R(0)}, ye[18], ype[4], eq[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const int64_t n = q2_node(ex, ez, k, g.nnx);
      ue[2 * k] = L.fix[2 * n] ? R(0) : u[2 * n];
      ue[2 * k + 1] = L.fix[2 * n + 1] ? R(0) : u[2 * n + 1];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) eq[q] = L.eta[(int64_t)e * 9 + q];
    element_apply<R>(sxe, sze, jace, se, ue, pe, eq, ye, ype, false);
#pragma unroll
    for (int k = 0; k < 18; ++k) sye[e * 18 + k] = ye[k];
  }
  barrier();
  const int64_t nn = (int64_t)g.nnx * g.nnz;
  for (int64_t n = t0; n < nn; n += nt) {
    const int ix = (int)(n % g.nnx), iz = (int)(n / g.nnx);
    const bool xo_ = ix & 1, zo = iz & 1;
    const int xa = xo_ ? (ix >> 1) : (ix >> 1) - 1, xb = (ix >> 1);
    const int za = zo ? (iz >> 1) : (iz >> 1) - 1, zb = (iz >> 1);
    const bool vxa = xa >= 0, vxb = !xo_ && xb < g.nx;
    const bool vza = za >= 0, vzb = !zo && zb < g.nz;
    const int dxa = xo_ ? 1 : 2, dza = zo ? 1 : 2;
    R2 y;
    y.x = 0;
    y.y = 0;
    if (vza) {
      if (vxa) { const R* ye = sye + (za * g.nx + xa) * 18; int k = q2_local_idx(dxa, dza);
                 y.x += ye[2 * k]; y.y += ye[2 * k + 1]; }
      if (vxb) { const R* ye = sye + (za * g.nx + xb) * 18; int k = q2_local_idx(0, dza);
                 y.x += ye[2 * k]; y.y += ye[2 * k + 1]; }
    }
    if (vzb) {
      if (vxa) { const R* ye = sye + (zb * g.nx + xa) * 18; int k = q2_local_idx(dxa, 0);
                 y.x += ye[2 * k]; y.y += ye[2 * k + 1]; }
      if (vxb) { const R* ye = sye + (zb * g.nx + xb) * 18; int k = q2_local_idx(0, 0);
                 y.x += ye[2 * k]; y.y += ye[2 * k + 1]; }
    }
    const uint8_t f0 = L.fix[2 * n], f1 = L.fix[2 * n + 1];
    const R2 uu = reinterpret_cast<const R2*>(u)[n];
    if (f0 | f1) {                                   // eliminated rows act as K_ii u_i
      const R2 dg = reinterpret_cast<const R2*>(L.diag)[n];
      const R2 fy{dg.x * uu.x, dg.y * uu.y};
      if (f0) y.x = fy.x;
      if (f1) y.y = fy.y;
    }
    const R2 bb = reinterpret_cast<const R2*>(L.b)[n];
    if (MODE == AM_RESID) {
      reinterpret_cast<R2*>(L.r)[n] = R2{bb.x - y.x, bb.y - y.y};
    } else {                                         // d = c1 d + c2 D^-1 (b - y); xo = u + d
      const R2 dg = reinterpret_cast<const R2*>(L.diag)[n];
      const double c1 = cheb[0];
      const R c2 = R(cheb[1]);
      R2 dn{c2 * (bb.x - y.x) / dg.x, c2 * (bb.y - y.y) / dg.y};
      if (c1 != 0.0) {
        const R2 dd = reinterpret_cast<const R2*>(L.d)[n];
        dn.x += R(c1) * dd.x;
        dn.y += R(c1) * dd.y;
      }
      reinterpret_cast<R2*>(L.d)[n] = dn;
      reinterpret_cast<R2*>(xo)[n] = R2{uu.x + dn.x, uu.y + dn.y};
    }
  }
  barrier();
}

// The tail's V-cycle (levels sL[0 .. A.n-1], the last the coarsest) by the t0-th of nt threads, the
// phases separated by `barrier`; returns where level 0's final x is (the x/t ping-pong).
template <typename R, typename B>
MW_D R* tail_vcycle(const TailLevel<R>* sL, const TailArgs<R>& A, R* sye, int t0, int nt, const B& barrier) {
  R* xs[MAX_TAIL];
  R* ts[MAX_TAIL];
  for (int l = 0; l < A.n; ++l) { xs[l] = sL[l].x; ts[l] = sL[l].t; }
  auto cheb_step = [&](int l, int k) {             // Chebyshev step k: x_out in t, then swap
    tail_apply<R, AM_CHEB>(sL[l], xs[l], ts[l], sL[l].cheb + 2 * k, sye, t0, nt, barrier);
    R* tmp = xs[l]; xs[l] = ts[l]; ts[l] = tmp;
  };
  auto smooth_tail = [&](int l, int degree, bool zero_start, bool first_done) {
    const TailLevel<R>& L = sL[l];
    if (first_done) {
      // x = d = (1/theta) D^-1 b was written by the restriction
    } else if (zero_start) {
      const R c = (R)L.cheb[1];
      const int64_t n = 2LL * L.g.nnx * L.g.nnz;
      for (int64_t i = t0; i < n; i += nt) {
        R v = c * L.b[i] / L.diag[i];
        xs[l][i] = v; L.d[i] = v;
      }
      barrier();
    } else {
      cheb_step(l, 0);
    }
    for (int k = 1; k < degree; ++k) cheb_step(l, k);
  };
  // down: pre-smoothing, residual, restriction (with the coarse level's first Chebyshev step)
  for (int l = 0; l + 1 < A.n; ++l) {
    const bool fd = l == 0 ? A.first_done != 0 : true;
    smooth_tail(l, sL[l].deg, !fd, fd);
    tail_apply<R, AM_RESID>(sL[l], xs[l], nullptr, nullptr, sye, t0, nt, barrier);
    const TailLevel<R>& F = sL[l];
    const TailLevel<R>& C = sL[l + 1];
    const bool fuse = !(l + 2 == A.n && A.dense);
    const double c0 = fuse ? C.cheb[1] : 0.0;
    const int64_t ncn = (int64_t)C.g.nnx * C.g.nnz;
    for (int64_t n = t0; n < ncn; n += nt)
      restrict_node(F.g, C.g, F.r, C.fix, C.b, c0, fuse, C.diag, xs[l + 1], C.d, n);
    barrier();
  }
  {  // coarsest level
    const int l = A.n - 1;
    if (A.dense) {
      const int lane = t0 & 31, warp = t0 >> 5, nwarp = nt >> 5;
      const R* b = sL[l].b;
      for (int row = warp; row < A.nd; row += nwarp) {
        double sacc = 0;
        for (int j = lane; j < A.nd; j += 32) sacc += A.Ainv[(int64_t)row * A.nd + j] * (double)b[j];
        for (int o = 16; o > 0; o >>= 1) sacc += __shfl_down_sync(0xffffffffu, sacc, o);
        if (lane == 0) xs[l][row] = (R)sacc;
      }
      barrier();
    } else {
      const bool fd = A.n == 1 ? A.first_done != 0 : true;
      smooth_tail(l, MAXDEG, !fd, fd);
    }
  }
  // up: prolongation and post-smoothing
  for (int l = A.n - 2; l >= 0; --l) {
    const TailLevel<R>& F = sL[l];
    const TailLevel<R>& C = sL[l + 1];
    const int64_t nfn = (int64_t)F.g.nnx * F.g.nnz;
    for (int64_t n = t0; n < nfn; n += nt) prolong_node(F.g, C.g, xs[l + 1], F.fix, xs[l], n);
    barrier();
    smooth_tail(l, sL[l].deg, false, false);
  }
  return xs[0];
}

template <typename R>
__global__ void __cluster_dims__(TAIL_CLUSTER, 1, 1) __launch_bounds__(tail_threads<R>(), 1)
k_vtail(TailArgs<R> A) {
  pdl_entry();
  const int t0 = (int)(cluster_rank() * blockDim.x + threadIdx.x), nt = (int)(TAIL_CLUSTER * blockDim.x);
  __shared__ TailLevel<R> sL[MAX_TAIL];
#pragma unroll
  for (int l = 0; l < MAX_TAIL; ++l)
    if (threadIdx.x == l && l < A.n) sL[l] = A.L[l];
  __syncthreads();
  tail_vcycle<R>(sL, A, A.ye, t0, nt, ClusterBarrier());
}

// The same tail in one CTA with every level's vectors, viscosities, diagonals, masks and the
// element products in shared memory: each phase is a shared-memory round trip and a block
// barrier instead of a launch or a round trip through L2.  Reads the first level's b (and x, d
// when the restriction did the first Chebyshev step) and every level's eta, mask and diagonal,
// writes the first level's final x to A.out_x.  Same phases, same arithmetic, same order as the
// multi-launch V-cycle.
template <typename R>
__global__ void __launch_bounds__(tail_threads<R>(), 1) k_vtail_smem(TailArgs<R> A) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char tsm[];
  __shared__ TailLevel<R> sL[MAX_TAIL];
  const int t0 = threadIdx.x, nt = blockDim.x;
  if (threadIdx.x == 0) {                       // carve the shared memory (the host sized it alike)
    size_t off = 0;
    auto take = [&](size_t bytes) { void* p = tsm + off; off += (bytes + 15) & ~size_t(15); return p; };
    for (int l = 0; l < A.n; ++l) {
      TailLevel<R> L = A.L[l];
      const int64_t nd = 2LL * L.g.nnx * L.g.nnz, ne = (int64_t)L.g.nx * L.g.nz;
      L.eta = (const R*)take(sizeof(R) * ne * 9);
      L.diag = (const R*)take(sizeof(R) * nd);
      L.fix = (const uint8_t*)take(nd);
      L.x = (R*)take(sizeof(R) * nd);
      L.t = (R*)take(sizeof(R) * nd);
      L.b = (R*)take(sizeof(R) * nd);
      L.r = (R*)take(sizeof(R) * nd);
      L.d = (R*)take(sizeof(R) * nd);
      sL[l] = L;
    }
  }
  __syncthreads();
  R* sye = nullptr;
  {
    size_t off = 0;                             // the element products after the levels
    for (int l = 0; l < A.n; ++l) {
      const int64_t nd = 2LL * A.L[l].g.nnx * A.L[l].g.nnz, ne = (int64_t)A.L[l].g.nx * A.L[l].g.nz;
      off += ((sizeof(R) * ne * 9 + 15) & ~size_t(15)) + ((sizeof(R) * nd + 15) & ~size_t(15)) + ((nd + 15) & ~size_t(15)) +
             5 * ((sizeof(R) * nd + 15) & ~size_t(15));
    }
    sye = reinterpret_cast<R*>(tsm + off);
  }
  for (int l = 0; l < A.n; ++l) {               // stage the inputs
    const TailLevel<R>& G = A.L[l];
    const TailLevel<R>& S = sL[l];
    const int64_t nd = 2LL * G.g.nnx * G.g.nnz, ne = (int64_t)G.g.nx * G.g.nz;
    for (int64_t i = t0; i < ne * 9; i += nt) const_cast<R*>(S.eta)[i] = G.eta[i];
    for (int64_t i = t0; i < nd; i += nt) {
      const_cast<R*>(S.diag)[i] = G.diag[i];
      const_cast<uint8_t*>(S.fix)[i] = G.fix[i];
      if (l == 0) {
        S.b[i] = G.b[i];
        if (A.first_done) { S.x[i] = G.x[i]; S.d[i] = G.d[i]; }
      }
    }
  }
  __syncthreads();
  const R* xf = tail_vcycle<R>(sL, A, sye, t0, nt, BlockBarrier());
  const int64_t nd0 = 2LL * A.L[0].g.nnx * A.L[0].g.nnz;
  for (int64_t i = t0; i < nd0; i += nt) A.out_x[i] = xf[i];
}

// shared memory of the one-CTA tail over levels L[0 .. n-1] (the carving of k_vtail_smem)
template <typename R>
static size_t tail_smem_bytes(const TailArgs<R>& A) {
  size_t off = 0;
  auto r16 = [](size_t b) { return (b + 15) & ~size_t(15); };
  int64_t maxe = 0;
  for (int l = 0; l < A.n; ++l) {
    const int64_t nd = 2LL * A.L[l].g.nnx * A.L[l].g.nnz, ne = (int64_t)A.L[l].g.nx * A.L[l].g.nz;
    off += r16(sizeof(R) * ne * 9) + r16(sizeof(R) * nd) + r16(nd) + 5 * r16(sizeof(R) * nd);
    maxe = std::max(maxe, ne);
  }
  return off + sizeof(R) * maxe * 18;
}

// Chebyshev smoothing of level L: x (in/out) with rhs b, `steps` steps; zero_start -> x = 0 on entry.
template <typename R>
static void smooth(Level<R>& L, int degree, bool zero_start, cudaStream_t s, bool first_done = false) {
  const int64_t n = L.ndof;
  if (first_done) {
    // x = d = (1/theta) D^-1 b was written by the restriction kernel
  } else if (zero_start) {
    if constexpr (sizeof(R) == 4) if (degree >= 2) {  // steps 0 and 1 in one launch (FP32)
      ApplyArgs<R> a = args0<R>();
      a.u = L.x; a.eta = L.eta; a.fix = L.fix; a.diag = L.diag; a.yV = L.d; a.bV = L.b; a.d = L.d; a.xo = L.t;
      a.cheb = L.cheb + 2;
      a.cheb0 = L.cheb;
      launch_apply<R, AM_CHEB_Z>(L.g, a, s);
      std::swap(L.x, L.t);
      for (int k = 2; k < degree; ++k) {
        ApplyArgs<R> b = args0<R>();
        b.u = L.x; b.eta = L.eta; b.fix = L.fix; b.diag = L.diag; b.yV = L.d; b.bV = L.b; b.d = L.d; b.xo = L.t;
        b.cheb = L.cheb + 2 * k;
        launch_apply<R, AM_CHEB>(L.g, b, s);
        std::swap(L.x, L.t);
      }
      return;
    }
    pdl_launch(k_cheb_first<R>, grid_for(n, 256), 256, 0, s, n, L.cheb, L.b, L.diag, L.x, L.d);
  } else {
    // restart the recurrence from the current x: d = (1/theta) D^-1 r; x += d
    ApplyArgs<R> a = args0<R>();
    a.u = L.x; a.eta = L.eta; a.fix = L.fix; a.diag = L.diag; a.yV = L.d; a.bV = L.b; a.d = L.d; a.xo = L.t;
    a.cheb = L.cheb;                    // step-0 pair {0, 1/theta}
    launch_apply<R, AM_CHEB>(L.g, a, s);
    std::swap(L.x, L.t);
  }
  for (int k = 1; k < degree; ++k) {
    ApplyArgs<R> a = args0<R>();
    a.u = L.x; a.eta = L.eta; a.fix = L.fix; a.diag = L.diag; a.yV = L.d; a.bV = L.b; a.d = L.d; a.xo = L.t;
    a.cheb = L.cheb + 2 * k;
    launch_apply<R, AM_CHEB>(L.g, a, s);
    std::swap(L.x, L.t);
  }
}

// The host's record of the x/t pointer swaps the smoothing of levels l.. performs in one V-cycle
// (what the multi-launch path does as it launches, and k_vtail does on the device).
template <typename R>
static void smooth_swaps(Level<R>& L, int degree, bool zero_start, bool first_done) {
  const int n = (!first_done && !zero_start ? 1 : 0) + (degree - 1);
  for (int i = 0; i < n; ++i) std::swap(L.x, L.t);
}

template <typename R>
static void tail_swaps(Hierarchy<R>& H, int l, bool first_done) {
  Level<R>& L = H.L[l];
  if (l == H.nlev - 1) {
    if (!H.dense) smooth_swaps(L, MAXDEG, !first_done, first_done);
    return;
  }
  smooth_swaps(L, L.deg, !first_done, first_done);
  tail_swaps(H, l + 1, !(l + 1 == H.nlev - 1 && H.dense));
  smooth_swaps(L, L.deg, false, false);
}

template <typename R>
static void launch_tail(Hierarchy<R>& H, int l0, bool first_done, cudaStream_t s) {
  TailArgs<R> A;
  memset(&A, 0, sizeof(A));
  A.n = H.nlev - l0;
  for (int i = 0; i < A.n; ++i) {
    const Level<R>& L = H.L[l0 + i];
    A.L[i] = TailLevel<R>{L.g, L.eta, L.fix, L.diag, L.x, L.t, L.b, L.r, L.d, L.cheb, L.deg};
  }
  A.first_done = first_done ? 1 : 0;
  A.dense = H.dense ? 1 : 0;
  A.nd = H.nd;
  A.Ainv = H.Ainv;
  A.ye = H.tail_ye;
  // the one-CTA shared-memory tail when every tail level fits (MW_TAIL_SMEM=0 in the environment:
  // the cluster tail through global memory)
  static const bool smem_on = [] {
    const char* e = getenv("MW_TAIL_SMEM");
    return !(e && e[0] == '0');
  }();
  const size_t sm = tail_smem_bytes(A);
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t limit = (size_t)optin > 1024 ? (size_t)optin - 1024 : 0;   // static TailLevel copies
  if (smem_on && sm <= limit) {
    static size_t attr_set = 0;
    if (sm > attr_set &&
        cudaFuncSetAttribute(k_vtail_smem<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)limit) == cudaSuccess)
      attr_set = limit;
    if (sm <= attr_set) {
      tail_swaps(H, l0, first_done);          // the host's record of where level l0's x ends up
      A.out_x = H.L[l0].x;
      pdl_launch(k_vtail_smem<R>, 1, tail_threads<R>(), sm, s, A);
      return;
    }
    cudaGetLastError();
  }
  pdl_launch(k_vtail<R>, TAIL_CLUSTER, tail_threads<R>(), 0, s, A);
  tail_swaps(H, l0, first_done);
}

// The prolongation runs as its own launch (k_prolong_add) before the post-smoothing by default;
// MW_FUSED_PROLONG=1 in the environment (read at the first V-cycle) folds it into the first
// smoothing step (AM_CHEB_P) instead: the same arithmetic and results, one launch fewer per level
// and V-cycle, but the heavier smoothing kernel made the 512x512 FK step slower (26.50 against
// 26.15 ms; on the levels of at most 128^2 or 256^2 elements only: 24.84 / 24.86 against 24.76 ms,
// measured).
static bool fused_prolongation() {
  static const bool on = [] {
    const char* e = getenv("MW_FUSED_PROLONG");
    return e && e[0] == '1';
  }();
  return on;
}

template <typename R>
static void vcycle(Hierarchy<R>& H, int l, cudaStream_t s, bool first_done = false) {
  Level<R>& L = H.L[l];
  if (H.tail0 > 0 && l == H.tail0) {               // the coarse levels in one launch
    launch_tail(H, l, first_done, s);        // records the tail's pointer swaps too
    return;
  }
  if (l == H.nlev - 1) {
    if (H.dense) {
      int nd = H.nd;
      pdl_launch(k_dense_matvec<R>, (nd * 32 + 255) / 256, 256, 0, s, nd, H.Ainv, L.b, L.x);
    } else {
      smooth(L, MAXDEG, !first_done, s, first_done);
    }
    return;
  }
  Level<R>& C = H.L[l + 1];
  smooth(L, L.deg, !first_done, s, first_done);
  ApplyArgs<R> a = args0<R>();
  a.u = L.x; a.eta = L.eta; a.fix = L.fix; a.diag = L.diag; a.yV = L.r; a.bV = L.b;
  launch_apply<R, AM_RESID>(L.g, a, s);
  const bool fuse = !(l + 1 == H.nlev - 1 && H.dense);
  const bool nested = nested_levels(L.g, C.g);
  if (nested)
    pdl_launch(k_restrict<R>, dim3((C.g.nnx + RTX - 1) / RTX, (C.g.nnz + RTZ - 1) / RTZ), RTX * RTZ, 0, s, L.g, C.g,
               L.r, C.fix, C.b, fuse ? C.cheb : nullptr, C.diag,
               C.x, C.d);
  else
    pdl_launch(k_restrict_g<R>, grid_for(C.nn, 256), 256, 0, s, L.g, C.g, L.r, C.fix, C.b, fuse ? C.cheb : nullptr,
               C.diag, C.x, C.d);
  vcycle(H, l + 1, s, fuse);
  if (!fused_prolongation() || !nested) {          // x += P x_c as its own launch, then the smoothing
    if (nested)
      pdl_launch(k_prolong_add<R>, dim3((L.g.nnx + PTX - 1) / PTX, (L.g.nnz + PTZ - 1) / PTZ), PTX * PTZ, 0, s, L.g,
                 C.g, (const R*)C.x, L.fix, L.x);
    else
      pdl_launch(k_prolong_g<R>, grid_for(L.nn, 256), 256, 0, s, L.g, C.g, (const R*)C.x, L.fix, L.x);
    smooth(L, L.deg, false, s);
    return;
  }
  // x += P x_c folded into the first post-smoothing step (AM_CHEB_P: the restart step, which reads
  // the corrected x only through its staging), then the remaining steps
  {
    ApplyArgs<R> a = args0<R>();
    a.u = L.x; a.eta = L.eta; a.fix = L.fix; a.diag = L.diag; a.yV = L.d; a.bV = L.b; a.d = L.d; a.xo = L.t;
    a.cheb = L.cheb;                    // step-0 pair {0, 1/theta}
    a.xc = C.x; a.gc = C.g;
    launch_apply<R, AM_CHEB_P>(L.g, a, s);
    std::swap(L.x, L.t);
  }
  for (int k = 1; k < L.deg; ++k) {
    ApplyArgs<R> a = args0<R>();
    a.u = L.x; a.eta = L.eta; a.fix = L.fix; a.diag = L.diag; a.yV = L.d; a.bV = L.b; a.d = L.d; a.xo = L.t;
    a.cheb = L.cheb + 2 * k;
    launch_apply<R, AM_CHEB>(L.g, a, s);
    std::swap(L.x, L.t);
  }
}

// Replays the kernels `record` issues on s from a CUDA graph cached under (kind, host state).
// `save` returns the host-side state the sequence depends on (buffer pointers it reads and may
// permute), `load` reinstates one.  The first call per state records the graph (the capture only
// records, so the graph is then launched); when capture is unavailable (legacy default stream,
// an enclosing capture) the kernels are issued directly.
template <typename Rec, typename Save, typename Load>
static void graph_run(mw_stokes* S, int kind, Rec record, Save save, Load load, cudaStream_t s) {
  cudaStreamCaptureStatus cs0 = cudaStreamCaptureStatusNone;
  if (s != nullptr && cudaStreamIsCapturing(s, &cs0) == cudaSuccess && cs0 != cudaStreamCaptureStatusNone) {
    record();            // part of an enclosing capture
    return;
  }
  cudaGetLastError();
  std::vector<void*> st = save();
  if (S->use_graphs) {
    for (auto& e : S->graphs) {
      if (e.kind == kind && e.before == st) {
        if (cudaGraphLaunch(e.exec, s) == cudaSuccess) {
          load(e.after);
          return;
        }
        cudaGetLastError();
        record();
        return;
      }
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (S->graphs.size() < 256 && s != nullptr && cudaStreamIsCapturing(s, &cs) == cudaSuccess &&
        cs == cudaStreamCaptureStatusNone && cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      record();
      cudaGraph_t g = nullptr;
      cudaGraphExec_t ex = nullptr;
      const bool ok = cudaStreamEndCapture(s, &g) == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
      if (ok) {
        mw_stokes::GraphEntry e;
        e.kind = kind;
        e.before = st;
        e.after = save();
        e.exec = ex;
        S->graphs.push_back(e);
        if (cudaGraphLaunch(ex, s) == cudaSuccess) return;
      }
      cudaGetLastError();
      load(st);        // nothing ran: issue the kernels from the original state
    } else {
      cudaGetLastError();
    }
  }
  record();
}

template <typename R>
static std::vector<void*> vstate(const Hierarchy<R>& H) {
  std::vector<void*> v;
  for (int l = 0; l < H.nlev; ++l) {
    v.push_back(H.L[l].x);
    v.push_back(H.L[l].t);
  }
  v.push_back(H.L[0].b);
  return v;
}

template <typename R>
static void vload(Hierarchy<R>& H, const std::vector<void*>& v) {
  for (int l = 0; l < H.nlev; ++l) {
    H.L[l].x = (R*)v[2 * l];
    H.L[l].t = (R*)v[2 * l + 1];
  }
  H.L[0].b = (R*)v[2 * H.nlev];
}

// One V-cycle of hierarchy H (degree-`degree` Chebyshev smoothing) from a cached graph.
template <typename R>
static void vcycle_run(mw_stokes* S, Hierarchy<R>& H, cudaStream_t s) {
  const int kind = (sizeof(R) == 4 ? 1 : 2) * 64;
  graph_run(S, kind, [&]() { vcycle(H, 0, s); }, [&]() { return vstate(H); },
            [&](const std::vector<void*>& v) { vload(H, v); }, s);
}

template <typename R>
__global__ void k_power_init(int64_t n, R* __restrict__ v) {
  pdl_entry();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (R)(1.0 + 0.5 * sin(0.7 * (double)i));
}

template <typename R>
__global__ void k_normalize(int64_t n, const double* __restrict__ nrm2, R* __restrict__ v) {
  pdl_entry();
  const double inv = 1.0 / sqrt(fmax(*nrm2, 1e-300));
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (R)((double)v[i] * inv);
}

// Build the hierarchy for the fine viscosity already in L[0].eta: coarse viscosities, fixed
// masks, diagonals, lambda_max(D^-1 K) by power iteration and the Chebyshev coefficients, and the
// dense inverse of the coarsest operator.  No host synchronisation.
template <typename R>
static int setup_hierarchy(mw_stokes* S, Hierarchy<R>& H, cudaStream_t s) {
  const mw_stokes_params& prm = S->prm;
  // coarse viscosities, fixed masks and diagonals of every level (a short chain)
  for (int l = 0; l < H.nlev; ++l) {
    Level<R>& L = H.L[l];
    if (l > 0) {
      Level<R>& F = H.L[l - 1];
      pdl_launch(k_coarsen_eta<R>, grid_for(L.nel, 256), 256, 0, s, F.g, L.g, F.eta, L.eta);
      pdl_launch(k_fix_coarse<R>, grid_for(L.nn, 256), 256, 0, s, F.g, L.g, F.fix, L.fix);
    }
    pdl_launch(k_diag<R>, grid_for(L.nn, 128), 128, 0, s, L.g, L.eta, L.diag);
  }
  // the coarsest level's dense inverse occupies one SM for most of a millisecond: it runs on a
  // side branch (forked from and joined back into s by events, which a stream capture records as
  // two graph branches) while the power iterations of the other levels run on s
  const bool dense = H.dense;
  cudaStream_t ds = s;
  if (dense) {
    if (!S->side && (cudaStreamCreateWithFlags(&S->side, cudaStreamNonBlocking) != cudaSuccess ||
                     cudaEventCreateWithFlags(&S->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
                     cudaEventCreateWithFlags(&S->ev_join, cudaEventDisableTiming) != cudaSuccess)) {
      cudaGetLastError();
      if (S->side) cudaStreamDestroy(S->side);
      S->side = nullptr;
    }
    if (S->side && cudaEventRecord(S->ev_fork, s) == cudaSuccess &&
        cudaStreamWaitEvent(S->side, S->ev_fork, 0) == cudaSuccess)
      ds = S->side;
    else
      cudaGetLastError();
    Level<R>& L = H.L[H.nlev - 1];
    pdl_launch(k_dense_assemble<R>, 1, 1024, 0, ds, L.g, L.eta, L.fix, H.Ainv);
    const size_t smem = sizeof(double) * ((size_t)H.nd * H.nd + H.nd);
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // the kernel's shared-memory limit is raised once per device, to the device's maximum and under
    // a lock: solvers set up from several host threads never call it again (nor lower it under
    // another thread's launch, which setting it per size allowed), and a setup recorded into a CUDA
    // graph issues no attribute call after the first set-up
    static std::mutex attr_mu;
    static bool attr_set[64] = {false};
    bool smem_ok = false;
    if (smem <= (size_t)optin && dev >= 0 && dev < 64) {
      std::lock_guard<std::mutex> lock(attr_mu);
      if (!attr_set[dev])
        attr_set[dev] = cudaFuncSetAttribute(k_gauss_jordan_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             optin) == cudaSuccess;
      smem_ok = attr_set[dev];
    }
    if (smem_ok)
      pdl_launch(k_gauss_jordan_smem, 1, 1024, smem, ds, H.nd, H.Ainv);
    else
      pdl_launch(k_gauss_jordan, 1, 1024, sizeof(double) * H.nd, ds, H.nd, H.Ainv);
  }
  // Chebyshev intervals: power iteration v <- D^-1 K v / |v| per smoothed level, warm-started
  // from the previous viscosity's vector
  for (int l = 0; l < H.nlev - (dense ? 1 : 0); ++l) {
    Level<R>& L = H.L[l];
    const bool coarsest = l == H.nlev - 1;
    R* v = L.ev;
    int iters = prm.power_iters;
    if (!L.ev_ready) {
      pdl_launch(k_power_init<R>, grid_for(L.ndof, 256), 256, 0, s, L.ndof, v);
      L.ev_ready = true;
    } else {
      iters = prm.power_iters_warm > 0 ? prm.power_iters_warm : prm.power_iters;
    }
    for (int it = 0; it < iters; ++it) {
      dot<R>(S, L.ndof, v, v, L.lam2 + 1, s);
      pdl_launch(k_normalize<R>, grid_for(L.ndof, 256), 256, 0, s, L.ndof, L.lam2 + 1, v);
      k_only_apply<R>(L, v, L.d, s);
      pdl_launch(k_dinv<R>, grid_for(L.ndof, 256), 256, 0, s, L.ndof, L.d, L.diag, v);
    }
    dot<R>(S, L.ndof, v, v, L.lam2, s);          // ||D^-1 K v_prev||^2 with ||v_prev|| = 1
    int deg = coarsest ? MAXDEG : L.deg;
    pdl_launch(k_cheb_coeffs, 1, 32, 0, s, L.lam2, deg, prm.cheb_ratio, prm.cheb_safety, L.cheb);
  }
  if (ds != s) {
    cudaEventRecord(S->ev_join, ds);
    cudaStreamWaitEvent(s, S->ev_join, 0);
  }
  return cudaGetLastError() == cudaSuccess ? MW_OK : MW_ERR_CUDA;
}

static double read_scalar(const double* d, cudaStream_t s) {
  double h = 0;
  cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return h;
}

// Preconditioned CG for K x = b (b in double), MG V-cycle preconditioner at precision R.
// x is written (overwritten) in double.  Returns iterations; *relres = ||r|| / ||b||.
template <typename R>
static int pcg_K(mw_stokes* S, Hierarchy<R>& H, R** pc, const double* b, double* x, double rtol, int maxit,
                 double* relres, cudaStream_t s) {
  Level<R>& L = H.L[0];
  const int64_t n = L.ndof;
  R *xr = pc[0], *r = pc[1], *p = pc[3], *Ap = pc[4];
  R*& z = pc[2];
  double* sc = S->sc;   // [0] rz, [1] pAp, [2] rr, [3] bb, [4] rz_new
  pdl_launch(k_copy<R, double>, grid_for(n, 256), 256, 0, s, n, b, r);
  pdl_launch(k_set<R>, grid_for(n, 256), 256, 0, s, n, R(0), xr);
  dot<R>(S, n, r, r, sc + 3, s);
  double bb = read_scalar(sc + 3, s);
  if (!(bb > 0)) {
    pdl_launch(k_set<double>, grid_for(n, 256), 256, 0, s, n, 0.0, x);
    *relres = 0;
    return 0;
  }
  // preconditioner z = V(r): the fine level reads r in place and the result buffer is exchanged
  // with z (host pointers only, no copies)
  auto precond = [&](R* rin, R*& zout) {
    R* saved_b = L.b;
    L.b = rin;
    vcycle_run(S, H, s);
    L.b = saved_b;
    std::swap(zout, L.x);
  };
  precond(r, z);
  pdl_launch(k_copy<R, R>, grid_for(n, 256), 256, 0, s, n, z, p);
  dot<R>(S, n, r, z, sc + 0, s);
  int it = 0;
  double rr = bb;
  for (it = 1; it <= maxit; ++it) {
    k_only_apply<R>(L, p, Ap, s);
    dot<R>(S, n, p, Ap, sc + 1, s);
    pdl_launch(k_pcg_update_rr<R>, nb_for(n), 256, 0, s, n, sc + 0, sc + 1, p, Ap, xr, r, S->red, S->counter, sc + 2);
    rr = read_scalar(sc + 2, s);
    if (!std::isfinite(rr)) break;
    if (rr <= rtol * rtol * bb) break;
    precond(r, z);
    dot<R>(S, n, r, z, sc + 4, s);
    pdl_launch(k_xpby_ratio<R>, grid_for(n, 256), 256, 0, s, n, z, sc + 4, sc + 0, p);
    cudaMemcpyAsync(sc + 0, sc + 4, sizeof(double), cudaMemcpyDeviceToDevice, s);
  }
  pdl_launch(k_copy<double, R>, grid_for(n, 256), 256, 0, s, n, xr, x);
  *relres = std::sqrt(rr / bb);
  return it > maxit ? maxit : it;
}

// Jacobi-PCG for the (weighted) Q1 mass matrix: M_w x = b.  weights NULL -> M (uzawa3),
// weights = 1/eta_e -> M_eta (cd_u_eta).
// Solve M_w x = b (M_w = M for uzawa3, M_eta for cd_u_eta) by `iters` fixed-coefficient
// Chebyshev-Jacobi steps on lambda(D^-1 M_w) in [0.25, 2.25] (see k_mass_cheb): error reduction
// 2 (1/2)^iters, no dot products, no host synchronisation.  The diagonals are refreshed by
// mw_stokes_set_viscosity.  Replaces the splu solves of uzawa3_solver_L2.py:46-47 / cd_u_eta.py:284-289.
static void mass_solve_kernels(mw_stokes* S, const double* w, const double* b, double* x, int iters, cudaStream_t s);

static int mass_solve(mw_stokes* S, const double* w, const double* b, double* x, int iters, cudaStream_t s) {
  const int K = iters < 1 ? 1 : iters;
  std::vector<void*> key = {(void*)w, (void*)b, (void*)x, (void*)(intptr_t)K};
  graph_run(S, 1, [&]() { mass_solve_kernels(S, w, b, x, K, s); }, [&]() { return key; },
            [&](const std::vector<void*>&) {}, s);
  return K;
}

static void mass_solve_kernels(mw_stokes* S, const double* w, const double* b, double* x, int iters, cudaStream_t s) {
  const LevelGeo& g = S->fine;
  const int64_t n = (int64_t)(g.nx + 1) * (g.nz + 1);
  const double* dg = w ? S->medi : S->mdiag;
  const double a = 0.25 / 1.02, bb = 2.25 * 1.02;
  const double theta = 0.5 * (bb + a), delta = 0.5 * (bb - a), sigma = theta / delta;
  double rho = 1.0 / sigma;
  double* bufs[2] = {x, S->tP};
  const int K = iters < 1 ? 1 : iters;
  for (int k = 0; k < K; ++k) {
    double c1 = 0.0, c2 = 1.0 / theta;
    if (k > 0) {
      double rn = 1.0 / (2.0 * sigma - rho);
      c1 = rn * rho;
      c2 = 2.0 * rn / delta;
      rho = rn;
    }
    double* xin = bufs[(K - k) % 2];
    double* xout = bufs[(K - 1 - k) % 2];
    pdl_launch(k_mass_cheb, grid_for(n, 256), 256, 0, s, g, w, b, xin, xout, S->tP2, dg, c1, c2, k == 0);
  }
}

static void remove_mean(mw_stokes* S, int64_t n, double* x, cudaStream_t s) {
  dsum(S, n, x, S->sc + 40, s);
  pdl_launch(k_sub_mean, grid_for(n, 256), 256, 0, s, n, S->sc + 40, x);
}

// Full saddle residual in FP64: (RV, RP) = (f, h) - [K G; G^T 0] (V, P).  Returns ||R||/||b||
// when bnorm > 0 (bnorm = ||(f, h)||), else ||R||.
static double true_residual(mw_stokes* S, const double* V, const double* P, const double* f, const double* h,
                            double bnorm, cudaStream_t s) {
  const LevelGeo& g = S->fine;
  ApplyArgs<double> a = args0<double>();
  a.u = V; a.p = P; a.eta = S->etaq64; a.fix = S->fixV;
  a.diag = S->diag64;
  a.yV = S->RV; a.yP = S->RP; a.bV = f; a.bP = h;
  launch_apply<double, AM_RESID>(g, a, s);
  const int64_t nv = 2LL * g.nnx * g.nnz, np = (int64_t)(g.nx + 1) * (g.nz + 1);
  dot<double>(S, nv, S->RV, S->RV, S->sc + 50, s);
  dot<double>(S, np, S->RP, S->RP, S->sc + 51, s);
  double a2[2];
  cudaMemcpyAsync(a2, S->sc + 50, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  double r = std::sqrt(a2[0] + a2[1]);
  return bnorm > 0 ? r / bnorm : r;
}

// Inner K solve at the requested precision.
static int ensure_hierarchy(mw_stokes* S, int prec, cudaStream_t s) {
  if (prec == MW_F32) {
    if (!S->has32) return MW_ERR_BAD_ARG;
    if (S->dirty32) { int rc = setup_hierarchy<float>(S, S->H32, s); if (rc) return rc; S->dirty32 = false; }
  } else {
    if (!S->has64) return MW_ERR_BAD_ARG;
    if (S->dirty64) { int rc = setup_hierarchy<double>(S, S->H64, s); if (rc) return rc; S->dirty64 = false; }
  }
  return MW_OK;
}

static int solve_K(mw_stokes* S, int prec, const double* b, double* x, double rtol, int maxit, double* relres,
                   cudaStream_t s) {
  if (prec == MW_F32) return pcg_K<float>(S, S->H32, S->pc32, b, x, rtol, maxit, relres, s);
  return pcg_K<double>(S, S->H64, S->pc64, b, x, rtol, maxit, relres, s);
}

// Convergence history row k in the reference's terms (uzawa3_solver_L2.py:85-88, cd_u_eta.py):
// xiV = ||alpha d_k||, xiP = ||alpha p_k||, alpha, beta.  hist is [4][len] (xiV, xiP, alpha, beta).
__global__ void k_history(const double* __restrict__ sc, double* __restrict__ hist, int len, int k) {
  pdl_entry();
  const double alpha = sc[0] / sc[1];
  hist[k] = fabs(alpha) * sqrt(sc[6]);
  hist[len + k] = fabs(alpha) * sqrt(sc[5]);
  hist[2 * len + k] = alpha;
  hist[3 * len + k] = sc[2] / sc[0];
}

// Schur-complement PCG (uzawa3_solver_L2.py:21-99 / cd_u_eta.py:13-99) for the saddle system
// with right-hand side (f, h), starting from (V, P) (V is recomputed from P).  Stops when the
// Schur residual has dropped by `reduction` relative to its start, when the FP64 true residual
// meets `tol` (checked each iteration if check_true), or after max_outer iterations.
static int uzawa(mw_stokes* S, const mw_solve_params& sp, int prec, const double* f, const double* h, double* V,
                 double* P, double reduction, bool check_true, double bnorm, mw_solve_info* info, cudaStream_t s) {
  const LevelGeo& g = S->fine;
  const int64_t nv = 2LL * g.nnx * g.nnz, np = (int64_t)(g.nx + 1) * (g.nz + 1);
  const double* w = sp.scheme == MW_SCHEME_UZAWA3 ? nullptr : S->etae_w;
  double rel;
  // V = K^-1 (f - G P)
  grad_p(S, P, f, S->Gd, s);                                // Gd = f - G P
  int inner = solve_K(S, prec, S->Gd, V, sp.inner_rtol, sp.max_inner, &rel, s);
  info->inner_iters += inner;
  // rho = G^T V - h
  div_u(S, V, S->rP, s);                                    // rP = G^T V
  if (h) pdl_launch(k_axpy<double>, grid_for(np, 256), 256, 0, s, np, -1.0, h, S->rP);
  remove_mean(S, np, S->rP, s);
  mass_solve(S, w, S->rP, S->wP, sp.mass_iters, s);
  remove_mean(S, np, S->wP, s);
  pdl_launch(k_copy<double, double>, grid_for(np, 256), 256, 0, s, np, S->wP, S->dP);
  double* sc = S->sc + 24;    // [0] rw, [1] dSd, [2] rw_new, [3] rr0, [4] rr
  dot<double>(S, np, S->rP, S->wP, sc + 0, s);
  dot<double>(S, np, S->rP, S->rP, sc + 3, s);
  const double rr0 = read_scalar(sc + 3, s);
  int k;
  for (k = 0; k < sp.max_outer; ++k) {
    // z = K^-1 G d
    grad_p(S, S->dP, nullptr, S->Gd, s);
    inner = solve_K(S, prec, S->Gd, S->z, sp.inner_rtol, sp.max_inner, &rel, s);
    info->inner_iters += inner;
    // G^T z, step length alpha = (rho, w) / (d, G^T z)
    div_u(S, S->z, S->GTz, s);
    dot<double>(S, np, S->dP, S->GTz, sc + 1, s);
    const bool hist = sp.history && info->outer_iters < sp.history_len;
    if (hist) {                                               // ||d_k||^2, ||z_k||^2 before the updates
      dot<double>(S, np, S->dP, S->dP, sc + 5, s);
      dot<double>(S, nv, S->z, S->z, sc + 6, s);
    }
    pdl_launch(k_axpy_ratio<double, double>, grid_for(np, 256), 256, 0, s, np, sc + 0, sc + 1, 1.0, S->dP, P);
    pdl_launch(k_axpy_ratio<double, double>, grid_for(nv, 256), 256, 0, s, nv, sc + 0, sc + 1, -1.0, S->z, V);
    pdl_launch(k_axpy_ratio<double, double>, grid_for(np, 256), 256, 0, s, np, sc + 0, sc + 1, -1.0, S->GTz, S->rP);
    remove_mean(S, np, S->rP, s);
    mass_solve(S, w, S->rP, S->wP, sp.mass_iters, s);
    remove_mean(S, np, S->wP, s);
    dot<double>(S, np, S->rP, S->wP, sc + 2, s);
    if (hist) pdl_launch(k_history, 1, 1, 0, s, sc, sp.history, sp.history_len, info->outer_iters);
    pdl_launch(k_xpby_ratio<double>, grid_for(np, 256), 256, 0, s, np, S->wP, sc + 2, sc + 0, S->dP);
    cudaMemcpyAsync(sc + 0, sc + 2, sizeof(double), cudaMemcpyDeviceToDevice, s);
    info->outer_iters += 1;
    dot<double>(S, np, S->rP, S->rP, sc + 4, s);
    double rr = read_scalar(sc + 4, s);
    if (!std::isfinite(rr)) return MW_ERR_NOT_CONVERGED;
    if (check_true) {
      double tr = true_residual(S, V, P, f, h, bnorm, s);
      info->rel_residual = tr;
      if (tr <= sp.tol) { ++k; break; }
    }
    if (rr <= reduction * reduction * rr0) { ++k; break; }
  }
  return MW_OK;
}

// ================================================================ device-side loops
// The whole solve as one CUDA graph: the iterations run as conditional WHILE nodes whose bodies end
// with a one-thread kernel that updates the loop scalars and sets the condition, so no iteration
// waits for the host.  Every loop is bounded by its iteration cap (max_inner, max_outer,
// max_refine) and by a total work cap, both decided on the device.  Scalars live in S->sc from
// slot 64 on.
// Schur-residual reduction of a refinement sweep that starts at relative residual `rel`: the fixed
// sweep_reduction, or with target > 0 the smaller reduction target * tol / rel (at most 0.5).
MW_HD double sweep_target_reduction(double sweep_reduction, double target, double tol, double rel) {
  if (!(target > 0) || !(rel > 0)) return sweep_reduction;
  double r = target * tol / rel;
  if (r > 0.5) r = 0.5;
  return r > sweep_reduction ? r : sweep_reduction;
}

enum DevSlot {
  P_RZ = 64, P_PAP, P_RR, P_BB, P_RZN, P_IT,                 // inner PCG
  U_RW = 72, U_DSD, U_RWN, U_RR0, U_RR, U_IT, U_D2, U_Z2,    // Schur CG
  T_RV = 84, T_RP, T_REL,                                     // true residual
  S_BB = 88, S_BH, S_BNORM, S_REL0, S_NREF, S_RED,           // solve
  I_OUTER = 96, I_INNER, I_STATUS                             // info
};

// Work caps of one solve on top of the per-loop caps: a stagnating solve ends with status 3 after
// this many inner (multigrid-PCG) or outer (Schur) iterations in total.
constexpr double DEV_INNER_BUDGET = 40000, DEV_OUTER_BUDGET = 4000;

__global__ void k_dev_pcg_init(double* sc, cudaGraphConditionalHandle hw) {
  pdl_entry();
  sc[P_IT] = 0;
  const double bb = sc[P_BB];
  cudaGraphSetConditional(hw, (bb > 0 && isfinite(bb)) ? 1u : 0u);
}

__global__ void k_dev_pcg_check(double* sc, double rtol, int maxit, cudaGraphConditionalHandle hw,
                                cudaGraphConditionalHandle hi) {
  pdl_entry();
  const double it = sc[P_IT] + 1;
  sc[P_IT] = it;
  const double rr = sc[P_RR];
  bool go = isfinite(rr) && rr > rtol * rtol * sc[P_BB] && it < (double)maxit;
  if (go && sc[I_INNER] + it >= DEV_INNER_BUDGET) { sc[I_STATUS] = 3; go = false; }
  cudaGraphSetConditional(hw, go ? 1u : 0u);
  cudaGraphSetConditional(hi, go ? 1u : 0u);
}

__global__ void k_dev_pcg_done(double* sc) {
  pdl_entry(); sc[I_INNER] += sc[P_IT]; }

__global__ void k_dev_uz_init(double* sc, int max_outer, cudaGraphConditionalHandle hw) {
  pdl_entry();
  sc[U_IT] = 0;
  cudaGraphSetConditional(hw, (max_outer > 0 && isfinite(sc[U_RR0]) && sc[I_STATUS] == 0) ? 1u : 0u);
}

// one Schur iteration done: stop on a non-finite residual (status 2), on the FP64 true residual
// (check_true), on the Schur residual reduction, at max_outer or at the work cap (status 3)
__global__ void k_dev_uz_check(double* sc, double reduction, int check_true, double tol, int max_outer,
                               cudaGraphConditionalHandle hw) {
  pdl_entry();
  const double it = sc[U_IT] + 1;
  sc[U_IT] = it;
  sc[I_OUTER] += 1;
  const double rr = sc[U_RR];
  if (reduction < 0) reduction = sc[S_RED];                   // this sweep's target (k_dev_sweep_red)
  bool go = it < (double)max_outer;
  if (!isfinite(rr)) { sc[I_STATUS] = 2; go = false; }
  if (sc[I_OUTER] >= DEV_OUTER_BUDGET && sc[I_STATUS] == 0) sc[I_STATUS] = 3;
  if (sc[I_STATUS] != 0) go = false;
  if (check_true && sc[T_REL] <= tol) go = false;
  if (rr <= reduction * reduction * sc[U_RR0]) go = false;
  cudaGraphSetConditional(hw, go ? 1u : 0u);
}

__global__ void k_dev_hist(const double* sc, double* hist, int len) {
  pdl_entry();
  const int k = (int)sc[I_OUTER];
  if (k < 0 || k >= len) return;
  const double alpha = sc[U_RW] / sc[U_DSD];
  hist[k] = fabs(alpha) * sqrt(sc[U_Z2]);
  hist[len + k] = fabs(alpha) * sqrt(sc[U_D2]);
  hist[2 * len + k] = alpha;
  hist[3 * len + k] = sc[U_RWN] / sc[U_RW];
}

__global__ void k_dev_rel(double* sc) {
  pdl_entry(); sc[T_REL] = sqrt(sc[T_RV] + sc[T_RP]) / sc[S_BNORM]; }

__global__ void k_dev_solve_init(double* sc) {
  pdl_entry();
  sc[S_BNORM] = sqrt(sc[S_BB] + sc[S_BH]);
  sc[S_NREF] = 0;
  sc[I_OUTER] = 0;
  sc[I_INNER] = 0;
  sc[I_STATUS] = 0;
}

__global__ void k_dev_ref_init(double* sc, double tol, int max_refine, cudaGraphConditionalHandle hw) {
  pdl_entry();
  sc[S_REL0] = sc[T_REL];
  const double r = sc[T_REL];
  cudaGraphSetConditional(hw, (isfinite(r) && r > tol && max_refine > 0) ? 1u : 0u);
}

__global__ void k_dev_ref_check(double* sc, double tol, int max_refine, cudaGraphConditionalHandle hw) {
  pdl_entry();
  sc[S_NREF] += 1;
  const double r = sc[T_REL];
  const bool go = isfinite(r) && r > tol && sc[S_NREF] < (double)max_refine && sc[I_STATUS] == 0;
  cudaGraphSetConditional(hw, go ? 1u : 0u);
}

// the reduction a refinement sweep's Schur iteration aims for: sweep_reduction, or -- with
// target > 0 -- the smaller reduction that takes the current residual to target * tol
__global__ void k_dev_sweep_red(double* sc, double sweep_reduction, double target, double tol) {
  pdl_entry();
  sc[S_RED] = sweep_target_reduction(sweep_reduction, target, tol, sc[T_REL]);
}

__global__ void k_copy1(const double* src, double* dst) {
  pdl_entry(); *dst = *src; }

// A conditional handle in the graph being captured on s (its value is set by kernels of that graph).
static bool cond_handle(cudaStream_t s, cudaGraphConditionalHandle* h) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  if (cudaStreamGetCaptureInfo(s, &st, nullptr, &g, nullptr, nullptr) != cudaSuccess || st != cudaStreamCaptureStatusActive)
    return false;
  return cudaGraphConditionalHandleCreate(h, g, 0, cudaGraphCondAssignDefault) == cudaSuccess;
}

// Append a conditional node (handle h) to the graph captured on s, after everything captured so far,
// and start capturing its body on bs.  cond_end(bs) closes the body.
static bool cond_node(cudaStream_t s, cudaStream_t bs, cudaGraphConditionalNodeType type, cudaGraphConditionalHandle h) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  if (cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd) != cudaSuccess || st != cudaStreamCaptureStatusActive)
    return false;
  cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
  p.conditional.handle = h;
  p.conditional.type = type;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, g, deps, nd, &p) != cudaSuccess) return false;
  if (cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) return false;
  return cudaStreamBeginCaptureToGraph(bs, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                       cudaStreamCaptureModeThreadLocal) == cudaSuccess;
}

static bool cond_end(cudaStream_t bs) {
  cudaGraph_t g = nullptr;
  return cudaStreamEndCapture(bs, &g) == cudaSuccess;
}

// capture stream of nesting level `depth` (0: the solve's stream)
static cudaStream_t lvl(mw_stokes* S, cudaStream_t s, int depth) { return depth == 0 ? s : S->bs[depth - 1]; }

// Inner PCG for K x = b recorded with a device WHILE loop (capture only), at nesting level `depth`
// (uses the body streams depth and depth + 1).  Adds its iteration count to sc[I_INNER].
template <typename R>
static bool pcg_K_dev(mw_stokes* S, Hierarchy<R>& H, R** pc, const double* b, double* x, double rtol, int maxit,
                      cudaStream_t s0, int depth) {
  if (depth + 2 > 6) return false;
  cudaStream_t s = lvl(S, s0, depth), b1 = S->bs[depth], b2 = S->bs[depth + 1];
  Level<R>& L = H.L[0];
  const int64_t n = L.ndof;
  R *xr = pc[0], *r = pc[1], *p = pc[3], *Ap = pc[4];
  R*& z = pc[2];
  double* sc = S->sc;
  auto precond = [&](R* rin, R*& zout, cudaStream_t st) {
    R* saved_b = L.b;
    L.b = rin;
    vcycle(H, 0, st);
    L.b = saved_b;
    std::swap(zout, L.x);
  };
  pdl_launch(k_copy<R, double>, grid_for(n, 256), 256, 0, s, n, b, r);
  pdl_launch(k_set<R>, grid_for(n, 256), 256, 0, s, n, R(0), xr);
  dot<R>(S, n, r, r, sc + P_BB, s);
  precond(r, z, s);
  pdl_launch(k_copy<R, R>, grid_for(n, 256), 256, 0, s, n, z, p);
  dot<R>(S, n, r, z, sc + P_RZ, s);
  cudaGraphConditionalHandle hw, hi;
  if (!cond_handle(s, &hw)) return false;
  pdl_launch(k_dev_pcg_init, 1, 1, 0, s, sc, hw);
  if (!cond_node(s, b1, cudaGraphCondTypeWhile, hw)) return false;
  // body: one CG step and the convergence test, then (if continuing) the next search direction
  k_only_apply<R>(L, p, Ap, b1);
  dot<R>(S, n, p, Ap, sc + P_PAP, b1);
  pdl_launch(k_pcg_update_rr<R>, nb_for(n), 256, 0, b1, n, sc + P_RZ, sc + P_PAP, p, Ap, xr, r, S->red, S->counter,
             sc + P_RR);
  if (!cond_handle(b1, &hi)) return false;
  pdl_launch(k_dev_pcg_check, 1, 1, 0, b1, sc, rtol, maxit, hw, hi);
  if (!cond_node(b1, b2, cudaGraphCondTypeIf, hi)) return false;
  precond(r, z, b2);
  dot<R>(S, n, r, z, sc + P_RZN, b2);
  pdl_launch(k_xpby_ratio<R>, grid_for(n, 256), 256, 0, b2, n, z, sc + P_RZN, sc + P_RZ, p);
  pdl_launch(k_copy1, 1, 1, 0, b2, sc + P_RZN, sc + P_RZ);
  if (!cond_end(b2) || !cond_end(b1)) return false;
  pdl_launch(k_copy<double, R>, grid_for(n, 256), 256, 0, s, n, xr, x);
  pdl_launch(k_dev_pcg_done, 1, 1, 0, s, sc);
  return true;
}

static bool solve_K_dev(mw_stokes* S, int prec, const double* b, double* x, double rtol, int maxit, cudaStream_t s0,
                        int depth) {
  if (prec == MW_F32) return pcg_K_dev<float>(S, S->H32, S->pc32, b, x, rtol, maxit, s0, depth);
  return pcg_K_dev<double>(S, S->H64, S->pc64, b, x, rtol, maxit, s0, depth);
}

// FP64 true residual into sc[T_REL] (relative to sc[S_BNORM]); RV, RP hold the residual.
static void true_residual_dev(mw_stokes* S, const double* V, const double* P, const double* f, const double* h,
                              cudaStream_t s) {
  const LevelGeo& g = S->fine;
  ApplyArgs<double> a = args0<double>();
  a.u = V; a.p = P; a.eta = S->etaq64; a.fix = S->fixV;
  a.diag = S->diag64;
  a.yV = S->RV; a.yP = S->RP; a.bV = f; a.bP = h;
  launch_apply<double, AM_RESID>(g, a, s);
  const int64_t nv = 2LL * g.nnx * g.nnz, np = (int64_t)(g.nx + 1) * (g.nz + 1);
  dot<double>(S, nv, S->RV, S->RV, S->sc + T_RV, s);
  dot<double>(S, np, S->RP, S->RP, S->sc + T_RP, s);
  pdl_launch(k_dev_rel, 1, 1, 0, s, S->sc);
}

// Schur-complement CG (the recurrences of the host version `uzawa`) recorded with a device WHILE
// loop at nesting level `depth` (uses body streams depth .. depth + 3).
static bool uzawa_dev(mw_stokes* S, const mw_solve_params& sp, int prec, const double* f, const double* h, double* V,
                      double* P, double reduction, bool check_true, cudaStream_t s0, int depth) {
  if (depth + 4 > 6) return false;
  cudaStream_t s = lvl(S, s0, depth), b1 = S->bs[depth];
  const LevelGeo& g = S->fine;
  const int64_t nv = 2LL * g.nnx * g.nnz, np = (int64_t)(g.nx + 1) * (g.nz + 1);
  const double* w = sp.scheme == MW_SCHEME_UZAWA3 ? nullptr : S->etae_w;
  double* sc = S->sc;
  grad_p(S, P, f, S->Gd, s);                                // V = K^-1 (f - G P)
  if (!solve_K_dev(S, prec, S->Gd, V, sp.inner_rtol, sp.max_inner, s0, depth)) return false;
  div_u(S, V, S->rP, s);                                    // rho = G^T V - h
  if (h) pdl_launch(k_axpy<double>, grid_for(np, 256), 256, 0, s, np, -1.0, h, S->rP);
  remove_mean(S, np, S->rP, s);
  mass_solve(S, w, S->rP, S->wP, sp.mass_iters, s);
  remove_mean(S, np, S->wP, s);
  pdl_launch(k_copy<double, double>, grid_for(np, 256), 256, 0, s, np, S->wP, S->dP);
  dot<double>(S, np, S->rP, S->wP, sc + U_RW, s);
  dot<double>(S, np, S->rP, S->rP, sc + U_RR0, s);
  cudaGraphConditionalHandle hw;
  if (!cond_handle(s, &hw)) return false;
  pdl_launch(k_dev_uz_init, 1, 1, 0, s, sc, sp.max_outer, hw);
  if (!cond_node(s, b1, cudaGraphCondTypeWhile, hw)) return false;
  grad_p(S, S->dP, nullptr, S->Gd, b1);
  if (!solve_K_dev(S, prec, S->Gd, S->z, sp.inner_rtol, sp.max_inner, s0, depth + 1)) return false;
  div_u(S, S->z, S->GTz, b1);
  dot<double>(S, np, S->dP, S->GTz, sc + U_DSD, b1);
  const bool hist = sp.history && sp.history_len > 0;
  if (hist) {
    dot<double>(S, np, S->dP, S->dP, sc + U_D2, b1);
    dot<double>(S, nv, S->z, S->z, sc + U_Z2, b1);
  }
  pdl_launch(k_axpy_ratio<double, double>, grid_for(np, 256), 256, 0, b1, np, sc + U_RW, sc + U_DSD, 1.0, S->dP, P);
  pdl_launch(k_axpy_ratio<double, double>, grid_for(nv, 256), 256, 0, b1, nv, sc + U_RW, sc + U_DSD, -1.0, S->z, V);
  pdl_launch(k_axpy_ratio<double, double>, grid_for(np, 256), 256, 0, b1, np, sc + U_RW, sc + U_DSD, -1.0, S->GTz,
             S->rP);
  remove_mean(S, np, S->rP, b1);
  mass_solve(S, w, S->rP, S->wP, sp.mass_iters, b1);
  remove_mean(S, np, S->wP, b1);
  dot<double>(S, np, S->rP, S->wP, sc + U_RWN, b1);
  if (hist) pdl_launch(k_dev_hist, 1, 1, 0, b1, sc, sp.history, sp.history_len);
  pdl_launch(k_xpby_ratio<double>, grid_for(np, 256), 256, 0, b1, np, S->wP, sc + U_RWN, sc + U_RW, S->dP);
  pdl_launch(k_copy1, 1, 1, 0, b1, sc + U_RWN, sc + U_RW);
  dot<double>(S, np, S->rP, S->rP, sc + U_RR, b1);
  if (check_true) true_residual_dev(S, V, P, f, h, b1);
  pdl_launch(k_dev_uz_check, 1, 1, 0, b1, sc, reduction, check_true ? 1 : 0, sp.tol, sp.max_outer, hw);
  return cond_end(b1);
}

// The whole solve (FP64, or mixed: FP64 refinement around FP32-inner Schur sweeps), recorded.
static bool stokes_solve_record(mw_stokes* S, const double* f, const double* h, double* V, double* P,
                                const mw_solve_params& sp, cudaStream_t s) {
  const LevelGeo& g = S->fine;
  const int64_t nv = 2LL * g.nnx * g.nnz, np = (int64_t)(g.nx + 1) * (g.nz + 1);
  double* sc = S->sc;
  if (!sp.use_guess) {
    pdl_launch(k_set<double>, grid_for(nv, 256), 256, 0, s, nv, 0.0, V);
    pdl_launch(k_set<double>, grid_for(np, 256), 256, 0, s, np, 0.0, P);
  }
  dot<double>(S, nv, f, f, sc + S_BB, s);
  dot<double>(S, np, h, h, sc + S_BH, s);
  pdl_launch(k_dev_solve_init, 1, 1, 0, s, sc);
  true_residual_dev(S, V, P, f, h, s);
  cudaGraphConditionalHandle hc;
  if (!cond_handle(s, &hc)) return false;
  if (sp.precision == MW_F64) {
    pdl_launch(k_dev_ref_init, 1, 1, 0, s, sc, sp.tol, 1, hc);        // records the initial residual; gate on tol
    if (!cond_node(s, S->bs[0], cudaGraphCondTypeIf, hc)) return false;
    if (!uzawa_dev(S, sp, MW_F64, f, h, V, P, 0.0, true, s, 1)) return false;
    if (!cond_end(S->bs[0])) return false;
    true_residual_dev(S, V, P, f, h, s);
  } else {
    pdl_launch(k_dev_ref_init, 1, 1, 0, s, sc, sp.tol, sp.max_refine, hc);
    if (!cond_node(s, S->bs[0], cudaGraphCondTypeWhile, hc)) return false;
    cudaStream_t b = S->bs[0];
    pdl_launch(k_copy<double, double>, grid_for(nv, 256), 256, 0, b, nv, S->RV, S->f);
    pdl_launch(k_copy<double, double>, grid_for(np, 256), 256, 0, b, np, S->RP, S->h);
    pdl_launch(k_set<double>, grid_for(nv, 256), 256, 0, b, nv, 0.0, S->cV);
    pdl_launch(k_set<double>, grid_for(np, 256), 256, 0, b, np, 0.0, S->cP);
    pdl_launch(k_dev_sweep_red, 1, 1, 0, b, sc, sp.sweep_reduction, sp.sweep_target, sp.tol);
    if (!uzawa_dev(S, sp, MW_F32, S->f, S->h, S->cV, S->cP, -1.0, false, s, 1)) return false;
    pdl_launch(k_axpy<double>, grid_for(nv, 256), 256, 0, b, nv, 1.0, S->cV, V);
    pdl_launch(k_axpy<double>, grid_for(np, 256), 256, 0, b, np, 1.0, S->cP, P);
    true_residual_dev(S, V, P, f, h, b);
    pdl_launch(k_dev_ref_check, 1, 1, 0, b, sc, sp.tol, sp.max_refine, hc);
    if (!cond_end(b)) return false;
  }
  return true;
}

template <typename R>
static int transfer_level(Hierarchy<R>& H, int level, int restrict_dir, const void* in, void* out, cudaStream_t s) {
  if (level < 0 || level + 1 >= H.nlev) return MW_ERR_BAD_ARG;
  const Level<R>& F = H.L[level];
  const Level<R>& C = H.L[level + 1];
  if (restrict_dir)
    pdl_launch(k_restrict_g<R>, grid_for(C.nn, 256), 256, 0, s, F.g, C.g, (const R*)in, (const uint8_t*)C.fix,
               (R*)out, (const double*)nullptr, (const R*)nullptr, (R*)nullptr, (R*)nullptr);
  else
    pdl_launch(k_prolong_g<R>, grid_for(F.nn, 256), 256, 0, s, F.g, C.g, (const R*)in, (const uint8_t*)F.fix,
               (R*)out);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

template <typename R>
__global__ void k_cast(int64_t n, const double* __restrict__ a, R* __restrict__ b) {
  pdl_entry();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (R)a[i];
}

}  // namespace mw

using namespace mw;

extern "C" {

static size_t do_layout(mw_stokes* S, char* base, bool dry) {
  Arena A{base, 0, 0, dry};
  return layout(S, A);
}

static void init_params(mw_stokes* S, mw_box box, const mw_stokes_params& prm) {
  S->prm = prm;
  S->fine.nx = box.nelx; S->fine.nz = box.nelz;
  S->fine.nnx = 2 * box.nelx + 1; S->fine.nnz = 2 * box.nelz + 1;
  S->fine.hx = box.hx; S->fine.hz = box.hz;
  S->fine.s = prm.eta_ref / prm.L_ref;
  S->has64 = (prm.precisions & 1) != 0;
  S->has32 = (prm.precisions & 2) != 0;
  S->pc64[0] = nullptr;
  if (S->has64) plan_levels(S->H64, S->fine, prm);
  if (S->has32) plan_levels(S->H32, S->fine, prm);
}

void mw_stokes_default_params(mw_stokes_params* p) {
  memset(p, 0, sizeof(*p));
  p->eta_ref = 1.0; p->L_ref = 1.0; p->precisions = 3;
  p->coarse_min = 4; p->dense_max = 700; p->cheb_degree = 2; p->cheb_ratio = 8.0; p->cheb_safety = 1.1;
  // 40 cold power iterations: with 12 the lambda_max estimate of the RT set-up's K (no slip top and
  // bottom, 0.9142 x 1 box) came out low enough on the 128x128 and 256x256 levels that the Chebyshev
  // smoother amplified the top of the spectrum and multigrid-PCG stalled (500 iterations); with 40
  // it converges in 6 (FP64) / 16 (mixed) Schur iterations from a cold start (measured).  The
  // warm-started updates of later viscosities keep their own count.
  p->power_iters = 40;
  p->power_iters_warm = 3;
  p->tail_nel = 0;
  p->coarsen_odd = 1;
  p->coarse_dense_max = 168;
}

void mw_solve_default_params(mw_solve_params* p) {
  memset(p, 0, sizeof(*p));
  p->scheme = MW_SCHEME_CD_U_ETA; p->precision = MW_F64; p->tol = 1e-8; p->max_outer = 200;
  p->max_inner = 500; p->inner_rtol = 1e-10; p->max_refine = 20; p->sweep_reduction = 1e-3; p->sweep_target = 0.0;
  p->mass_iters = 12; p->use_guess = 0;
}

size_t mw_stokes_workspace_bytes(mw_box box, mw_stokes_params prm) {
  mw_stokes S;
  init_params(&S, box, prm);
  S.fixV = nullptr;
  return do_layout(&S, nullptr, true);
}

int mw_stokes_create(mw_box box, mw_stokes_params prm, const uint8_t* bc_fix_V, void* work, size_t work_bytes,
                     mw_stokes** out) {
  if (box.nelx < 2 || box.nelz < 2 || !bc_fix_V || !work || !out || !(prm.precisions & 3)) return MW_ERR_BAD_ARG;
  if (ensure_ref_tables()) return MW_ERR_CUDA;
  mw_stokes* S = new mw_stokes();
  init_params(S, box, prm);
  S->fixV = bc_fix_V;
  size_t need = do_layout(S, nullptr, true);
  if (work_bytes < need) { delete S; return MW_ERR_WORKSPACE; }
  do_layout(S, (char*)work, false);
  if (cudaMemset(S->counter, 0, sizeof(unsigned) * 4) != cudaSuccess) { delete S; return MW_ERR_CUDA; }
  *out = S;
  return MW_OK;
}

int mw_stokes_destroy(mw_stokes* S) {
  delete S;
  return MW_OK;
}

int mw_stokes_device_info(mw_stokes* S, double tol, mw_solve_info* info, void* stream) {
  if (!info) return MW_ERR_BAD_ARG;
  double q[40];
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemcpyAsync(q, S->sc + 64, sizeof(q), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return MW_ERR_CUDA;
  const double bnorm = q[S_BNORM - 64];
  memset(info, 0, sizeof(*info));
  info->outer_iters = (int)q[I_OUTER - 64];
  info->inner_iters = (int)q[I_INNER - 64];
  info->refinements = (int)q[S_NREF - 64];
  info->initial_rel_residual = bnorm > 0 ? q[S_REL0 - 64] : 0.0;
  info->rel_residual = bnorm > 0 ? q[T_REL - 64] : 0.0;
  if (q[I_STATUS - 64] != 0 || !std::isfinite(bnorm)) info->rel_residual = NAN;
  info->converged = info->rel_residual <= tol ? 1 : 0;
  return MW_OK;
}

int mw_stokes_device_loops(const mw_stokes* S) {
  if (!S->device_loops) return 0;
  for (const auto& e : S->graphs)
    if (e.kind == 1000) return 1;
  return 0;
}

int mw_stokes_levels(const mw_stokes* S, int32_t precision) {
  return precision == MW_F32 ? S->H32.nlev : S->H64.nlev;
}

int mw_stokes_set_viscosity(mw_stokes* S, const double* etaq, const double* eta_e, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nel = (int64_t)S->fine.nx * S->fine.nz;
  pdl_launch(k_cast<double>, grid_for(nel * 9, 256), 256, 0, s, nel * 9, etaq, S->etaq64);
  if (S->has32) pdl_launch(k_cast<float>, grid_for(nel * 9, 256), 256, 0, s, nel * 9, etaq, S->etaq32);
  pdl_launch(k_inv_eta_e, grid_for(nel, 256), 256, 0, s, nel, etaq, eta_e, S->etae_w);
  pdl_launch(k_diag<double>, grid_for((int64_t)S->fine.nnx * S->fine.nnz, 128), 128, 0, s, S->fine, S->etaq64,
             S->diag64);
  const int64_t np = (int64_t)(S->fine.nx + 1) * (S->fine.nz + 1);
  pdl_launch(k_mass_diag, grid_for(np, 256), 256, 0, s, S->fine, nullptr, S->mdiag);      // M
  pdl_launch(k_mass_diag, grid_for(np, 256), 256, 0, s, S->fine, S->etae_w, S->medi);     // M_eta
  S->dirty64 = S->dirty32 = true;
  if (cudaGetLastError() != cudaSuccess) return MW_ERR_CUDA;
  return MW_OK;
}

// The kernels read and write velocity vectors one (u, w) node pair per access, so velocity arrays
// passed in must be aligned to a pair: 16 bytes in FP64, 8 in FP32 (a misaligned array is refused
// here instead of faulting on the device).
static bool pair_aligned(const void* p, size_t pair_bytes) { return ((uintptr_t)p % pair_bytes) == 0; }

int mw_stokes_apply(mw_stokes* S, const double* u, const double* p, double* yV, double* yP, void* stream) {
  if (!pair_aligned(u, 16) || !pair_aligned(yV, 16)) return MW_ERR_BAD_ARG;
  ApplyArgs<double> a = args0<double>();
  a.u = u; a.p = p; a.eta = S->etaq64; a.fix = S->fixV; a.diag = S->diag64; a.yV = yV; a.yP = yP;
  launch_apply<double, AM_APPLY>(S->fine, a, (cudaStream_t)stream);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_stokes_grad(mw_stokes* S, const double* p, double* yV, void* stream) {
  if (!p || !pair_aligned(yV, 16)) return MW_ERR_BAD_ARG;
  grad_p(S, p, nullptr, yV, (cudaStream_t)stream);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_stokes_div(mw_stokes* S, const double* u, double* yP, void* stream) {
  if (!pair_aligned(u, 16) || !yP) return MW_ERR_BAD_ARG;
  div_u(S, u, yP, (cudaStream_t)stream);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_stokes_apply_f32(mw_stokes* S, const float* u, const float* p, float* yV, float* yP, void* stream) {
  if (!S->has32 || !pair_aligned(u, 8) || !pair_aligned(yV, 8)) return MW_ERR_BAD_ARG;
  if (ensure_hierarchy(S, MW_F32, (cudaStream_t)stream)) return MW_ERR_CUDA;
  ApplyArgs<float> a = args0<float>();
  a.u = u; a.p = p; a.eta = S->etaq32; a.fix = S->fixV; a.diag = S->H32.L[0].diag; a.yV = yV; a.yP = yP;
  launch_apply<float, AM_APPLY>(S->fine, a, (cudaStream_t)stream);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_stokes_cheb_step_f32(mw_stokes* S, const float* b, const float* x, float* xo, float* d, int32_t step,
                            void* stream) {
  if (!S->has32 || !b || !pair_aligned(x, 8) || !pair_aligned(xo, 8) || !d || step < 0 || step >= MAXDEG)
    return MW_ERR_BAD_ARG;
  if (ensure_hierarchy(S, MW_F32, (cudaStream_t)stream)) return MW_ERR_CUDA;
  Level<float>& L = S->H32.L[0];
  if (step >= L.deg && step > 0) return MW_ERR_BAD_ARG;
  ApplyArgs<float> a = args0<float>();
  a.u = x; a.eta = L.eta; a.fix = L.fix; a.diag = L.diag; a.yV = d; a.bV = b; a.d = d; a.xo = xo;
  a.cheb = L.cheb + 2 * step;
  launch_apply<float, AM_CHEB>(L.g, a, (cudaStream_t)stream);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_stokes_vcycle(mw_stokes* S, int32_t precision, const void* b, void* x, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (int rc = ensure_hierarchy(S, precision, s)) return rc;
  if (precision == MW_F32) {
    Level<float>& L = S->H32.L[0];
    pdl_launch(k_copy<float, float>, grid_for(L.ndof, 256), 256, 0, s, L.ndof, (const float*)b, L.b);
    vcycle(S->H32, 0, s);
    pdl_launch(k_copy<float, float>, grid_for(L.ndof, 256), 256, 0, s, L.ndof, L.x, (float*)x);
  } else {
    Level<double>& L = S->H64.L[0];
    pdl_launch(k_copy<double, double>, grid_for(L.ndof, 256), 256, 0, s, L.ndof, (const double*)b, L.b);
    vcycle(S->H64, 0, s);
    pdl_launch(k_copy<double, double>, grid_for(L.ndof, 256), 256, 0, s, L.ndof, L.x, (double*)x);
  }
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_stokes_transfer(mw_stokes* S, int32_t precision, int32_t level, int32_t restrict_dir, const void* in,
                       void* out, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!S || !in || !out) return MW_ERR_BAD_ARG;
  if (int rc = ensure_hierarchy(S, precision, s)) return rc;
  return precision == MW_F32 ? transfer_level(S->H32, level, restrict_dir, in, out, s)
                             : transfer_level(S->H64, level, restrict_dir, in, out, s);
}

int mw_stokes_level_shape(const mw_stokes* S, int32_t precision, int32_t level, int32_t* nx, int32_t* nz) {
  const auto& H32 = S->H32;
  const auto& H64 = S->H64;
  const int nlev = precision == MW_F32 ? H32.nlev : H64.nlev;
  if (!nx || !nz || level < 0 || level >= nlev) return MW_ERR_BAD_ARG;
  *nx = precision == MW_F32 ? H32.L[level].g.nx : H64.L[level].g.nx;
  *nz = precision == MW_F32 ? H32.L[level].g.nz : H64.L[level].g.nz;
  return MW_OK;
}

static cudaStream_t enter(mw_stokes* S, cudaStream_t caller);
static void leave(mw_stokes* S, cudaStream_t caller, cudaStream_t s);

int mw_stokes_solve_K(mw_stokes* S, int32_t precision, const double* b, double* x, double rtol, int32_t maxit,
                      int32_t* iters, double* relres, void* stream) {
  if (!b || !x || !pair_aligned(b, 16) || !pair_aligned(x, 16)) return MW_ERR_BAD_ARG;
  double rr = 0;
  cudaStream_t caller = (cudaStream_t)stream;
  cudaStream_t s = enter(S, caller);
  int rc = ensure_hierarchy(S, precision, s);
  int it = rc ? 0 : solve_K(S, precision, b, x, rtol, maxit, &rr, s);
  leave(S, caller, s);
  if (rc) return rc;
  if (iters) *iters = it;
  if (relres) *relres = rr;
  if (cudaGetLastError() != cudaSuccess) return MW_ERR_CUDA;
  return rr <= rtol ? MW_OK : MW_ERR_NOT_CONVERGED;
}

// Uzawa residual of a pressure candidate P: the Schur iteration recomputes the velocity from the
// pressure (V = K^-1 (f - G P), inner PCG to rtol), so its starting point is judged by the 2-norm
// of G^T V - h with its mean removed.
int mw_stokes_uzawa_residual(mw_stokes* S, int32_t precision, const double* f, const double* h, const double* P,
                             double rtol, int32_t maxit, double* V, double* norm_out, void* stream) {
  if (!f || !h || !P || !norm_out || !pair_aligned(f, 16) || !pair_aligned(V, 16)) return MW_ERR_BAD_ARG;
  cudaStream_t caller = (cudaStream_t)stream;
  cudaStream_t s = enter(S, caller);
  int rc = ensure_hierarchy(S, precision, s);
  if (!rc) {
    const LevelGeo& g = S->fine;
    const int64_t np = (int64_t)(g.nx + 1) * (g.nz + 1);
    grad_p(S, P, f, S->Gd, s);                              // Gd = f - G P
    double rr = 0;
    double* Vo = V ? V : S->z;
    solve_K(S, precision, S->Gd, Vo, rtol, maxit, &rr, s);
    div_u(S, Vo, S->rP, s);                                 // rP = G^T V
    pdl_launch(k_axpy<double>, grid_for(np, 256), 256, 0, s, np, -1.0, h, S->rP);
    remove_mean(S, np, S->rP, s);
    dot<double>(S, np, S->rP, S->rP, S->sc + 54, s);
    double v = 0;
    cudaMemcpyAsync(&v, S->sc + 54, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = MW_ERR_CUDA;
    *norm_out = std::sqrt(v);
  }
  leave(S, caller, s);
  if (!rc && cudaGetLastError() != cudaSuccess) rc = MW_ERR_CUDA;
  return rc;
}

int mw_stokes_residual(mw_stokes* S, const double* V, const double* P, const double* f, const double* h, double* RV,
                       double* RP, double* norm_out, void* stream) {
  if (!f || !h || !pair_aligned(V, 16) || !pair_aligned(f, 16)) return MW_ERR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  double r = true_residual(S, V, P, f, h, 0.0, s);
  if (RV) cudaMemcpyAsync(RV, S->RV, sizeof(double) * 2 * S->fine.nnx * S->fine.nnz, cudaMemcpyDeviceToDevice, s);
  if (RP) cudaMemcpyAsync(RP, S->RP, sizeof(double) * (S->fine.nx + 1) * (S->fine.nz + 1), cudaMemcpyDeviceToDevice, s);
  if (norm_out) *norm_out = r;
  return cudaGetLastError() == cudaSuccess ? MW_OK : MW_ERR_CUDA;
}

// The solver's own stream, ordered after everything already queued on the caller's stream; leave()
// orders the caller's stream after the solver's work.  Falls back to the caller's stream when a
// stream or event cannot be created.
static cudaStream_t enter(mw_stokes* S, cudaStream_t caller) {
  if (!S->ws) {
    if (cudaStreamCreateWithFlags(&S->ws, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->ev_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->ev_out, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      if (S->ws) cudaStreamDestroy(S->ws);
      S->ws = nullptr;
      return caller;
    }
  }
  cudaEventRecord(S->ev_in, caller);
  cudaStreamWaitEvent(S->ws, S->ev_in, 0);
  return S->ws;
}

static void leave(mw_stokes* S, cudaStream_t caller, cudaStream_t s) {
  if (s == caller) return;
  cudaEventRecord(S->ev_out, s);
  cudaStreamWaitEvent(caller, S->ev_out, 0);
}

static int stokes_solve(mw_stokes* S, const double* f, const double* h, double* solV, double* solP,
                        const mw_solve_params& sp, mw_solve_info* info, cudaStream_t s);
static int stokes_solve_host(mw_stokes* S, const double* f, const double* h, double* solV, double* solP,
                             const mw_solve_params& sp, mw_solve_info* info, cudaStream_t s);

// The caller is recording a CUDA graph (a whole time step) on `caller`: record the solve into that
// capture -- its loops as conditional nodes -- and leave the result scalars on the device
// (mw_stokes_device_info reads them after a replay).
static int stokes_solve_in_capture(mw_stokes* S, const double* f, const double* h, double* solV, double* solP,
                                   const mw_solve_params& sp, mw_solve_info* info, cudaStream_t caller) {
  if (!f || !h || !solV || !solP || sp.host_loops) return MW_ERR_BAD_ARG;
  for (auto& b : S->bs)
    if (!b && cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking) != cudaSuccess) return MW_ERR_CUDA;
  if (int rc = ensure_hierarchy(S, sp.precision == MW_F32 ? MW_F32 : MW_F64, caller)) return rc;
  if (!stokes_solve_record(S, f, h, solV, solP, sp, caller)) return MW_ERR_CUDA;
  if (info) memset(info, 0, sizeof(*info));
  return MW_OK;
}

int mw_stokes_solve(mw_stokes* S, const double* f, const double* h, double* solV, double* solP, mw_solve_params sp,
                    mw_solve_info* info, void* stream) {
  if (!pair_aligned(f, 16) || !pair_aligned(solV, 16)) return MW_ERR_BAD_ARG;
  cudaStream_t caller = (cudaStream_t)stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (caller != nullptr && cudaStreamIsCapturing(caller, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
    return stokes_solve_in_capture(S, f, h, solV, solP, sp, info, caller);
  cudaGetLastError();
  cudaStream_t s = enter(S, caller);
  int rc = stokes_solve(S, f, h, solV, solP, sp, info, s);
  leave(S, caller, s);
  return rc;
}

static void key_add(std::vector<void*>& k, double v) {
  uint64_t u;
  memcpy(&u, &v, sizeof(u));
  k.push_back((void*)(uintptr_t)u);
}

// Runs the whole solve from a recorded graph (recorded on first use for these buffers, parameters
// and multigrid pointer state) and reads the loop scalars back once.  Returns false when the
// graph cannot be recorded or launched; the caller then runs the host-driven loops.
static bool stokes_solve_graph(mw_stokes* S, const double* f, const double* h, double* V, double* P,
                               const mw_solve_params& sp, mw_solve_info* inf, cudaStream_t s) {
  if (!S->device_loops || !S->use_graphs || s == nullptr) return false;
  for (auto& b : S->bs)
    if (!b && cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
  std::vector<void*> key = {(void*)f, (void*)h, (void*)V, (void*)P, (void*)sp.history,
                            (void*)(intptr_t)((sp.scheme << 24) ^ (sp.precision << 20) ^ (sp.use_guess << 16) ^
                                              sp.history_len),
                            (void*)(intptr_t)sp.max_outer, (void*)(intptr_t)sp.max_inner,
                            (void*)(intptr_t)sp.max_refine, (void*)(intptr_t)sp.mass_iters};
  key_add(key, sp.tol);
  key_add(key, sp.inner_rtol);
  key_add(key, sp.sweep_reduction);
  key_add(key, sp.sweep_target);
  std::vector<void*> h32 = vstate(S->H32), h64 = vstate(S->H64);
  key.insert(key.end(), h32.begin(), h32.end());
  key.insert(key.end(), h64.begin(), h64.end());
  const int kind = 1000;
  int hit = -1;
  for (size_t i = 0; i < S->graphs.size(); ++i)
    if (S->graphs[i].kind == kind && S->graphs[i].before == key) { hit = (int)i; break; }
  if (hit < 0) {
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) { cudaGetLastError(); return false; }
    bool ok = stokes_solve_record(S, f, h, V, P, sp, s);
    for (auto b : S->bs) {      // close any body capture left open by a failed recording
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(b, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t gb = nullptr;
        cudaStreamEndCapture(b, &gb);
        ok = false;
      }
    }
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    const bool captured = cudaStreamEndCapture(s, &g) == cudaSuccess && g;
    ok = ok && captured && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {                       // the recording ran nothing: restore the pointer state
      cudaGetLastError();
      vload(S->H32, h32);
      vload(S->H64, h64);
      S->device_loops = false;       // this device cannot record the loops: keep the host loops
      return false;
    }
    if (S->graphs.size() >= 192) {
      cudaGraphExecDestroy(S->graphs.front().exec);
      S->graphs.erase(S->graphs.begin());
    }
    mw_stokes::GraphEntry e;
    e.kind = kind;
    e.before = key;
    std::vector<void*> a32 = vstate(S->H32), a64 = vstate(S->H64);
    e.after = a32;
    e.after.insert(e.after.end(), a64.begin(), a64.end());
    e.exec = ex;
    S->graphs.push_back(e);
    hit = (int)S->graphs.size() - 1;
    vload(S->H32, h32);            // the after-state is applied below, once the graph ran
    vload(S->H64, h64);
  }
  mw_stokes::GraphEntry& e = S->graphs[hit];
  if (cudaGraphLaunch(e.exec, s) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  {
    const size_t n32 = h32.size();
    std::vector<void*> a32(e.after.begin(), e.after.begin() + n32), a64(e.after.begin() + n32, e.after.end());
    vload(S->H32, a32);
    vload(S->H64, a64);
  }
  double q[40];
  cudaMemcpyAsync(q, S->sc + 64, sizeof(q), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return false;
  const double bnorm = q[S_BNORM - 64];
  inf->outer_iters = (int)q[I_OUTER - 64];
  inf->inner_iters = (int)q[I_INNER - 64];
  inf->refinements = (int)q[S_NREF - 64];
  inf->initial_rel_residual = bnorm > 0 ? q[S_REL0 - 64] : 0.0;
  inf->rel_residual = bnorm > 0 ? q[T_REL - 64] : 0.0;
  if (!std::isfinite(bnorm)) inf->rel_residual = inf->initial_rel_residual = bnorm;
  if (q[I_STATUS - 64] != 0) inf->rel_residual = NAN;
  return true;
}

static int stokes_solve(mw_stokes* S, const double* f, const double* h, double* solV, double* solP,
                        const mw_solve_params& sp, mw_solve_info* info, cudaStream_t s) {
  if (!f || !h || !solV || !solP) return MW_ERR_BAD_ARG;
  if (int rc = ensure_hierarchy(S, sp.precision == MW_F32 ? MW_F32 : MW_F64, s)) return rc;
  {
    mw_solve_info inf;
    memset(&inf, 0, sizeof(inf));
    if (!sp.host_loops && stokes_solve_graph(S, f, h, solV, solP, sp, &inf, s)) {
      inf.converged = inf.rel_residual <= sp.tol ? 1 : 0;
      S->last = inf;
      if (info) *info = inf;
      if (cudaGetLastError() != cudaSuccess) return MW_ERR_CUDA;
      return inf.converged ? MW_OK : MW_ERR_NOT_CONVERGED;
    }
  }
  return stokes_solve_host(S, f, h, solV, solP, sp, info, s);
}

static int stokes_solve_host(mw_stokes* S, const double* f, const double* h, double* solV, double* solP,
                             const mw_solve_params& sp, mw_solve_info* info, cudaStream_t s) {
  const LevelGeo& g = S->fine;
  const int64_t nv = 2LL * g.nnx * g.nnz, np = (int64_t)(g.nx + 1) * (g.nz + 1);
  mw_solve_info inf;
  memset(&inf, 0, sizeof(inf));
  if (!f || !h || !solV || !solP) return MW_ERR_BAD_ARG;
  if (int rc = ensure_hierarchy(S, sp.precision == MW_F32 ? MW_F32 : MW_F64, s)) return rc;
  if (!sp.use_guess) {
    pdl_launch(k_set<double>, grid_for(nv, 256), 256, 0, s, nv, 0.0, solV);
    pdl_launch(k_set<double>, grid_for(np, 256), 256, 0, s, np, 0.0, solP);
  }
  // ||b||
  dot<double>(S, nv, f, f, S->sc + 52, s);
  if (h) dot<double>(S, np, h, h, S->sc + 53, s);
  double bb[2] = {0, 0};
  cudaMemcpyAsync(bb, S->sc + 52, (h ? 2 : 1) * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  const double bnorm = std::sqrt(bb[0] + bb[1]);
  if (!std::isfinite(bnorm)) {
    inf.rel_residual = inf.initial_rel_residual = bnorm;
    if (info) *info = inf;
    return MW_ERR_NOT_CONVERGED;
  }
  if (!(bnorm > 0)) { if (info) *info = inf; return MW_OK; }
  inf.initial_rel_residual = true_residual(S, solV, solP, f, h, bnorm, s);
  int rc = MW_OK;
  if (sp.precision == MW_F64) {
    // plain FP64: one Schur-PCG run with the true residual checked every iteration
    inf.rel_residual = inf.initial_rel_residual;
    if (inf.rel_residual > sp.tol)
      rc = uzawa(S, sp, MW_F64, f, h, solV, solP, 0.0, true, bnorm, &inf, s);
    inf.rel_residual = true_residual(S, solV, solP, f, h, bnorm, s);
  } else {
    // mixed: FP64 iterative refinement around an FP32-inner Uzawa correction solve
    double rel = inf.initial_rel_residual;
    for (int it = 0; it < sp.max_refine && rel > sp.tol; ++it) {
      // residual (RV, RP) is current in S->RV / S->RP from true_residual
      double* cV = S->cV;
      // solve A (cV, cP) = (RV, RP): copy the residual into f/h slots, zero guess
      double* fr = S->f;
      double* hr = S->h;
      pdl_launch(k_copy<double, double>, grid_for(nv, 256), 256, 0, s, nv, S->RV, fr);
      pdl_launch(k_copy<double, double>, grid_for(np, 256), 256, 0, s, np, S->RP, hr);
      pdl_launch(k_set<double>, grid_for(nv, 256), 256, 0, s, nv, 0.0, cV);
      double* cPr = S->cP;
      pdl_launch(k_set<double>, grid_for(np, 256), 256, 0, s, np, 0.0, cPr);
      rc = uzawa(S, sp, MW_F32, fr, hr, cV, cPr, sweep_target_reduction(sp.sweep_reduction, sp.sweep_target, sp.tol, rel),
                 false, 0.0, &inf, s);
      if (rc) break;
      pdl_launch(k_axpy<double>, grid_for(nv, 256), 256, 0, s, nv, 1.0, cV, solV);
      pdl_launch(k_axpy<double>, grid_for(np, 256), 256, 0, s, np, 1.0, cPr, solP);
      inf.refinements += 1;
      rel = true_residual(S, solV, solP, f, h, bnorm, s);
      inf.rel_residual = rel;
    }
    inf.rel_residual = rel;
  }
  inf.converged = inf.rel_residual <= sp.tol ? 1 : 0;
  S->last = inf;
  if (info) *info = inf;
  if (cudaGetLastError() != cudaSuccess) return MW_ERR_CUDA;
  if (rc) return rc;
  return inf.converged ? MW_OK : MW_ERR_NOT_CONVERGED;
}

}  // extern "C"

// the Stokes solves of an ensemble of models in one launch (one cluster per model)
#include "stokes_ensemble.cuh"
