// Element assembly kernels (sm_100a): Q2xQ1 Stokes and Q2 Crank-Nicolson energy.
//
// Reference: build_matrix_stokes.py:18-278 (box, plane strain) and build_matrix_energy.py:12-141.
// One CTA per batch of EB elements; 18 (Stokes) or 9 (energy) threads per element, one element
// matrix row each.  The 3x3 Gauss basis tables and the batch's per-qpoint inputs are staged in
// shared memory; the element outputs are staged in shared memory too and leave with coalesced
// stores in the reference's VV order (build_matrix_stokes.py:235-276, build_matrix_energy.py:133-137).
//
// Dirichlet elimination (build_matrix_stokes.py:206-217, build_matrix_energy.py:118-130) is done
// row-locally: eliminating fixed dofs in ascending order leaves a free row i with
// f_i - sum_{fixed j ascending} K0_ij v_j and zeros in the fixed columns, and a fixed row with
// only its diagonal and rhs K0_ii v_i -- the same values the reference's sequential loop yields.
//
// Right-hand sides: each element writes its local vector to a scratch buffer; a node-centric
// gather then sums the (up to 4) element contributions in ascending element order, the order of
// the reference's scatter loop.  No atomics; results are run-to-run identical.
#include "common.cuh"

namespace mw {

constexpr int EB_S = 16;   // elements per CTA, Stokes
constexpr int EB_T = 24;   // elements per CTA, energy (static shared memory stays under 48 KB)

// local Q2 node index from its lattice offset (dx, dz) in {0,1,2}^2
MW_HD int q2_local(int dx, int dz) {
  if (dz == 0) return dx == 0 ? 0 : (dx == 1 ? 4 : 1);
  if (dz == 1) return dx == 0 ? 7 : (dx == 1 ? 8 : 5);
  return dx == 0 ? 3 : (dx == 1 ? 6 : 2);
}

template <typename R, typename S>
__global__ void __launch_bounds__(EB_S * 18)
k_assemble_stokes(mw_box b, mw_stokes_in in, int blocks, S* __restrict__ vv_full, S* __restrict__ vv_K,
                  S* __restrict__ vv_G, S* __restrict__ vv_GT, S* __restrict__ vv_M, S* __restrict__ vv_Meta,
                  S* __restrict__ vv_H, double* __restrict__ f_el, double* __restrict__ h_el) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tab = reinterpret_cast<R*>(smem_raw);                 // 351 table values
  R* NV = tab;            // 81
  R* NP = tab + 81;       // 36
  R* dNdx_V = tab + 117;  // EB*81  (per element, per q, per node)
  R* dNdz_V = dNdx_V + EB_S * 81;
  R* dNdx_P = dNdz_V + EB_S * 81;  // EB*36
  R* dNdz_P = dNdx_P + EB_S * 36;
  R* qin = dNdz_P + EB_S * 36;     // 5 arrays * EB*9 : rho, eta, JxW, gx, gz
  R* G0 = qin + 5 * EB_S * 9;      // EB*18*4 (fixed rows of G, for h)
  // the float instantiation ends G0 at a 4-byte boundary: realign before the double array
  double* bcv = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(G0 + EB_S * 72) + 15) & ~uintptr_t(15));
  int* bcf = reinterpret_cast<int*>(bcv + EB_S * 18);        // EB*18 flags
  S* outs = reinterpret_cast<S*>(bcf + EB_S * 18);           // staged element outputs

  const int64_t nel = (int64_t)b.nelx * b.nelz;
  const int64_t e0 = (int64_t)blockIdx.x * EB_S;
  const int ne = (int)((nel - e0) < EB_S ? (nel - e0) : EB_S);
  const int tid = threadIdx.x;
  const int nnx = 2 * b.nelx + 1;

  __shared__ R dNdr_V[81], dNdt_V[81], dNdr_P[36], dNdt_P[36];
  for (int i = tid; i < 81; i += blockDim.x) {
    NV[i] = (R)in.N_V[i]; dNdr_V[i] = (R)in.dNdr_V[i]; dNdt_V[i] = (R)in.dNdt_V[i];
  }
  for (int i = tid; i < 36; i += blockDim.x) {
    NP[i] = (R)in.N_P[i]; dNdr_P[i] = (R)in.dNdr_P[i]; dNdt_P[i] = (R)in.dNdt_P[i];
  }
  for (int i = tid; i < ne * 9; i += blockDim.x) {
    int64_t g = e0 * 9 + i;
    qin[i] = (R)in.rhoq[g];
    qin[EB_S * 9 + i] = (R)in.etaq[g];
    qin[2 * EB_S * 9 + i] = (R)in.JxWq[g];
    qin[3 * EB_S * 9 + i] = (R)in.gxq[g];
    qin[4 * EB_S * 9 + i] = (R)in.gzq[g];
  }
  for (int i = tid; i < ne * 18; i += blockDim.x) {
    int el = i / 18, ikk = i % 18;
    int64_t e = e0 + el;
    int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
    int64_t dof = 2 * q2_node(ex, ez, ikk / 2, nnx) + (ikk & 1);     // local_to_globalV, meeuuw.py:874-882
    bcf[i] = in.bc_fix_V[dof] ? 1 : 0;
    bcv[i] = in.bc_val_V[dof];
  }
  __syncthreads();
  // derivatives at qpoints: build_matrix_stokes.py:131-134
  for (int i = tid; i < ne * 9; i += blockDim.x) {
    int el = i / 9, q = i % 9;
    int64_t g = (e0 + el) * 9 + q;
    R j00 = (R)in.jcbi00q[g], j01 = (R)in.jcbi01q[g], j10 = (R)in.jcbi10q[g], j11 = (R)in.jcbi11q[g];
    for (int k = 0; k < 9; ++k) {
      dNdx_V[el * 81 + q * 9 + k] = j00 * dNdr_V[q * 9 + k] + j01 * dNdt_V[q * 9 + k];
      dNdz_V[el * 81 + q * 9 + k] = j10 * dNdr_V[q * 9 + k] + j11 * dNdt_V[q * 9 + k];
    }
    for (int k = 0; k < 4; ++k) {
      dNdx_P[el * 36 + q * 4 + k] = j00 * dNdr_P[q * 4 + k] + j01 * dNdt_P[q * 4 + k];
      dNdz_P[el * 36 + q * 4 + k] = j10 * dNdr_P[q * 4 + k] + j11 * dNdt_P[q * 4 + k];
    }
  }
  __syncthreads();

  const int el = tid / 18, ikk = tid % 18;
  const bool live = el < ne;
  const int i = ikk >> 1, c = ikk & 1;
  R K[18], G[4], H[4], Mv = 0, f = 0;
#pragma unroll
  for (int j = 0; j < 18; ++j) K[j] = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) { G[k] = 0; H[k] = 0; }
  if (live) {
    for (int q = 0; q < 9; ++q) {
      const R eta = qin[EB_S * 9 + el * 9 + q], jxw = qin[2 * EB_S * 9 + el * 9 + q];
      const R rho = qin[el * 9 + q];
      const R g = c == 0 ? qin[3 * EB_S * 9 + el * 9 + q] : qin[4 * EB_S * 9 + el * 9 + q];
      const R* dx = dNdx_V + el * 81 + q * 9;
      const R* dz = dNdz_V + el * 81 + q * 9;
      const R dxi = dx[i], dzi = dz[i];
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        R a, bb;   // B^T C B entries (build_matrix_stokes.py:140), C = diag(2, 2, 1)
        if (c == 0) { a = dxi * (R(2) * dx[j]) + dzi * dz[j]; bb = dzi * dx[j]; }
        else        { a = dxi * dz[j]; bb = dzi * (R(2) * dz[j]) + dxi * dx[j]; }
        K[2 * j] += a * eta * jxw;
        K[2 * j + 1] += bb * eta * jxw;
      }
      f += NV[q * 9 + i] * jxw * rho * g;                              // :142-143
      const R d = c == 0 ? dxi : dzi;
      const R* dP = (c == 0 ? dNdx_P : dNdz_P) + el * 36 + q * 4;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        G[k] -= d * NP[q * 4 + k] * jxw;                                 // :144-146
        H[k] += dP[k] * NV[q * 9 + i] * jxw;                             // :148-153
      }
      if (ikk < 16) Mv += NP[q * 4 + (ikk >> 2)] * NP[q * 4 + (ikk & 3)] * jxw;   // :147
    }
    const R s = (R)(in.eta_ref / in.L_ref);                                // :157
#pragma unroll
    for (int k = 0; k < 4; ++k) G[k] *= s;
  }
  // ---- Dirichlet elimination (row-local form) ----
  const int* fx = bcf + el * 18;
  const double* fv = bcv + el * 18;
  bool fixed_row = live && fx[ikk];
  R frow = f;
  if (live) {
    if (fixed_row) {
      R kd = 0;
#pragma unroll
      for (int j = 0; j < 18; ++j) if (j == ikk) kd = K[j];
#pragma unroll
      for (int k = 0; k < 4; ++k) G0[el * 72 + ikk * 4 + k] = G[k];
#pragma unroll
      for (int j = 0; j < 18; ++j) K[j] = (j == ikk) ? kd : R(0);
      frow = kd * (R)fv[ikk];
#pragma unroll
      for (int k = 0; k < 4; ++k) G[k] = 0;
    } else {
#pragma unroll
      for (int j = 0; j < 18; ++j)
        if (fx[j]) { frow -= K[j] * (R)fv[j]; K[j] = 0; }
    }
  }
  __syncthreads();
  if (live) {
    f_el[(e0 + el) * 18 + ikk] = (double)frow;
    if (ikk < 4) {
      R h = 0;
      for (int r2 = 0; r2 < 18; ++r2)
        if (fx[r2]) h -= G0[el * 72 + r2 * 4 + ikk] * (R)fv[r2];
      h_el[(e0 + el) * 4 + ikk] = (double)h;
    }
  }
  // ---- stage outputs and store coalesced (skipped in rhs-only mode) ----
  if (vv_full == nullptr && vv_K == nullptr) return;
  if (!blocks) {
    if (live) {
      S* o = outs + el * 468 + ikk * 26;                                   // :268-276
#pragma unroll
      for (int j = 0; j < 18; ++j) o[j] = (S)K[j];
#pragma unroll
      for (int k = 0; k < 4; ++k) { o[18 + 2 * k] = (S)G[k]; o[19 + 2 * k] = (S)G[k]; }
    }
    __syncthreads();
    S* dst = vv_full + e0 * 468;
    for (int x = tid; x < ne * 468; x += blockDim.x) dst[x] = outs[x];
  } else {
    S* oK = outs;                    // EB*324
    S* oG = oK + EB_S * 324;         // EB*72
    S* oGT = oG + EB_S * 72;
    S* oH = oGT + EB_S * 72;
    S* oM = oH + EB_S * 72;          // EB*16
    S* oMe = oM + EB_S * 16;
    if (live) {
#pragma unroll
      for (int j = 0; j < 18; ++j) oK[el * 324 + ikk * 18 + j] = (S)K[j];       // :237-240
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        oG[el * 72 + ikk * 4 + k] = (S)G[k];                                    // :243-246
        oGT[el * 72 + k * 18 + ikk] = (S)G[k];                                  // :249-252
        oH[el * 72 + k * 18 + ikk] = (S)H[k];                                   // :255-258
      }
      if (ikk < 16) {
        oM[el * 16 + ikk] = (S)Mv;                                              // :261-265
        oMe[el * 16 + ikk] = (S)(Mv / (R)in.eta_e[e0 + el]);
      }
    }
    __syncthreads();
    for (int x = tid; x < ne * 324; x += blockDim.x) vv_K[e0 * 324 + x] = oK[x];
    for (int x = tid; x < ne * 72; x += blockDim.x) {
      vv_G[e0 * 72 + x] = oG[x]; vv_GT[e0 * 72 + x] = oGT[x]; vv_H[e0 * 72 + x] = oH[x];
    }
    for (int x = tid; x < ne * 16; x += blockDim.x) { vv_M[e0 * 16 + x] = oM[x]; vv_Meta[e0 * 16 + x] = oMe[x]; }
  }
}

// Sum element-local vectors onto Q2 nodes (ndof per node) in ascending element order.
__global__ void k_gather_q2(mw_box b, int ndof, const double* __restrict__ vel, double* __restrict__ out) {
  const int nnx = 2 * b.nelx + 1, nnz = 2 * b.nelz + 1;
  const int64_t nn = (int64_t)nnx * nnz;
  const int per = 9 * ndof;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    int ix = (int)(n % nnx), iz = (int)(n / nnx);
    int exs[2], ezs[2], nx = 0, nz = 0;
    if (ix & 1) exs[nx++] = ix >> 1;
    else { if (ix / 2 - 1 >= 0) exs[nx++] = ix / 2 - 1; if (ix / 2 < b.nelx) exs[nx++] = ix / 2; }
    if (iz & 1) ezs[nz++] = iz >> 1;
    else { if (iz / 2 - 1 >= 0) ezs[nz++] = iz / 2 - 1; if (iz / 2 < b.nelz) ezs[nz++] = iz / 2; }
    for (int c = 0; c < ndof; ++c) {
      double acc = 0.0;
      for (int a = 0; a < nz; ++a)
        for (int bb = 0; bb < nx; ++bb) {
          int ex = exs[bb], ez = ezs[a];
          int k = q2_local(ix - 2 * ex, iz - 2 * ez);
          acc += vel[((int64_t)ez * b.nelx + ex) * per + k * ndof + c];
        }
      out[n * ndof + c] = acc;
    }
  }
}

// Sum element-local Q1 vectors (4 per element) onto pressure nodes in ascending element order.
__global__ void k_gather_q1(mw_box b, const double* __restrict__ hel, double* __restrict__ out) {
  const int ncx = b.nelx + 1;
  const int64_t nn = (int64_t)ncx * (b.nelz + 1);
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(n % ncx), j = (int)(n / ncx);
    double acc = 0.0;
    const int ex[4] = {i - 1, i, i - 1, i};
    const int ez[4] = {j - 1, j - 1, j, j};
    const int kk[4] = {2, 3, 1, 0};
    for (int s = 0; s < 4; ++s) {
      if (ex[s] < 0 || ex[s] >= b.nelx || ez[s] < 0 || ez[s] >= b.nelz) continue;
      acc += hel[((int64_t)ez[s] * b.nelx + ex[s]) * 4 + kk[s]];
    }
    out[n] = acc;
  }
}

// ------------------------------------------------------------------------------------------
template <typename R, typename S>
__global__ void __launch_bounds__(EB_T * 9)
k_assemble_energy(mw_box b, mw_energy_in in, S* __restrict__ vv, double* __restrict__ b_el) {
  __shared__ R NT[81], dNdr[81], dNds[81];
  __shared__ R dNdx[EB_T * 81], dNdy[EB_T * 81];
  __shared__ R Tloc[EB_T * 9];
  __shared__ int bfix[EB_T * 9];
  __shared__ double bval[EB_T * 9];
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  const int64_t e0 = (int64_t)blockIdx.x * EB_T;
  const int ne = (int)((nel - e0) < EB_T ? (nel - e0) : EB_T);
  const int tid = threadIdx.x;
  const int nnx = 2 * b.nelx + 1;
  for (int i = tid; i < 81; i += blockDim.x) {
    NT[i] = (R)in.N_T[i]; dNdr[i] = (R)in.dNdr_T[i]; dNds[i] = (R)in.dNds_T[i];
  }
  for (int i = tid; i < ne * 9; i += blockDim.x) {
    int el = i / 9, k = i % 9;
    int64_t e = e0 + el;
    int64_t node = q2_node((int)(e % b.nelx), (int)(e / b.nelx), k, nnx);
    Tloc[i] = (R)in.T[node];                                                // :63
    bfix[i] = in.bc_fix_T[node] ? 1 : 0;
    bval[i] = in.bc_val_T[node];
  }
  __syncthreads();
  for (int i = tid; i < ne * 9; i += blockDim.x) {
    int el = i / 9, q = i % 9;
    int64_t g = (e0 + el) * 9 + q;
    R j00 = (R)in.jcbi00q[g], j01 = (R)in.jcbi01q[g], j10 = (R)in.jcbi10q[g], j11 = (R)in.jcbi11q[g];
    for (int k = 0; k < 9; ++k) {
      dNdx[el * 81 + q * 9 + k] = j00 * dNdr[q * 9 + k] + j01 * dNds[q * 9 + k];   // :71
      dNdy[el * 81 + q * 9 + k] = j10 * dNdr[q * 9 + k] + j11 * dNds[q * 9 + k];   // :72
    }
  }
  __syncthreads();
  const int el = tid / 9, i = tid % 9;
  if (el >= ne) return;
  const int64_t e = e0 + el;
  R MM[9], Kd[9], Ka[9], bs = 0;
#pragma unroll
  for (int j = 0; j < 9; ++j) { MM[j] = 0; Kd[j] = 0; Ka[j] = 0; }
  const R rho0 = (R)in.rho0;
  for (int q = 0; q < 9; ++q) {
    const int64_t g = e * 9 + q;
    const R jxw = (R)in.JxWq[g], hc = (R)in.hcapaq[g], hk = (R)in.hcondq[g];
    const R u = (R)in.uq[g], w = (R)in.wq[g];
    const R* N = NT + q * 9;
    const R* dx = dNdx + el * 81 + q * 9;
    const R* dy = dNdy + el * 81 + q * 9;
    const R Ni = N[i];
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      MM[j] += Ni * N[j] * rho0 * hc * jxw;                                     // :77
      Kd[j] += (dx[i] * dx[j] + dy[i] * dy[j]) * hk * jxw;                      // :79
      Ka[j] += Ni * (u * dx[j] + w * dy[j]) * rho0 * hc * jxw;                  // :81
    }
    bs += Ni * (R)in.hprodq[g] * jxw;                                          // :83
    if (in.formulation == 1) {                                                  // :85-110 (EBA)
      const R exx = (R)in.exxq[g], ezz = (R)in.ezzq[g], exz = (R)in.exzq[g];
      bs += Ni * 2 * (R)in.etaq[g] *
            (R(2.0 / 3.0) * exx * exx + R(2.0 / 3.0) * ezz * ezz - R(2.0 / 3.0) * exx * ezz + 2 * exz * exz) * jxw;
      bs += Ni * (R)in.alphaq[g] * (R)in.Tq[g] * (-w * rho0 * 10) * jxw;
    }
  }
  const R dt = (R)(in.dt_dev ? *in.dt_dev : in.dt);
  bs *= dt;                                                                     // :112
  R A[9];
  R rhs = bs;
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    A[j] = MM[j] + (Ka[j] + Kd[j]) * dt * R(0.5);                               // :114
    rhs += (MM[j] - (Ka[j] + Kd[j]) * dt * R(0.5)) * Tloc[el * 9 + j];          // :115
  }
  const int* fx = bfix + el * 9;
  const double* fv = bval + el * 9;
  if (fx[i]) {                                                                  // :118-130
    R ad = 0;
#pragma unroll
    for (int j = 0; j < 9; ++j) if (j == i) ad = A[j];
#pragma unroll
    for (int j = 0; j < 9; ++j) A[j] = (j == i) ? ad : R(0);
    rhs = ad * (R)fv[i];
  } else {
#pragma unroll
    for (int j = 0; j < 9; ++j)
      if (fx[j]) { rhs -= A[j] * (R)fv[j]; A[j] = 0; }
  }
  S* o = vv + e * 81 + i * 9;                                                   // :133-137
#pragma unroll
  for (int j = 0; j < 9; ++j) o[j] = (S)A[j];
  b_el[e * 9 + i] = (double)rhs;
}

// Body-force element vectors f_el[2i+c] = sum_q N_V[q,i] JxW rho g_c (build_matrix_stokes.py:141-143)
// without the element matrices; fixed dofs get 0 (their rhs is K_ii * bc_val = 0 when every
// Dirichlet value is zero, :215).
__global__ void k_body_force(mw_box b, const double* __restrict__ rhoq, const double* __restrict__ gxq,
                             const double* __restrict__ gzq, const double* __restrict__ JxWq,
                             const double* __restrict__ NV, const uint8_t* __restrict__ fix, double* __restrict__ fel) {
  __shared__ double N[81];
  for (int i = threadIdx.x; i < 81; i += blockDim.x) N[i] = NV[i];
  __syncthreads();
  const int64_t n = (int64_t)b.nelx * b.nelz * 9;
  const int nnx = 2 * b.nelx + 1;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = g / 9;
    const int i = (int)(g % 9);
    double fx = 0.0, fz = 0.0;
    for (int q = 0; q < 9; ++q) {
      const int64_t gq = e * 9 + q;
      const double t = N[q * 9 + i] * JxWq[gq] * rhoq[gq];
      fx += t * gxq[gq];
      fz += t * gzq[gq];
    }
    const int64_t node = q2_node((int)(e % b.nelx), (int)(e / b.nelx), i, nnx);
    fel[e * 18 + 2 * i] = fix[2 * node] ? 0.0 : fx;
    fel[e * 18 + 2 * i + 1] = fix[2 * node + 1] ? 0.0 : fz;
  }
}

template <typename R>
static size_t stokes_smem_bytes() {
  size_t n = 117 + 2 * EB_S * 81 + 2 * EB_S * 36 + 5 * EB_S * 9 + EB_S * 72;
  size_t bytes = n * sizeof(R);
  bytes = ((bytes + 15) & ~size_t(15)) + 16;
  bytes += EB_S * 18 * sizeof(double) + EB_S * 18 * sizeof(int);
  bytes += (size_t)EB_S * 572 * sizeof(double);   // largest staged output (blocks layout, f64)
  return bytes;
}

template <typename R, typename S>
static int launch_stokes(const mw_box& b, const mw_stokes_in& in, const mw_stokes_out& out, int blocks, double* fel,
                         double* hel, cudaStream_t s) {
  int64_t nel = (int64_t)b.nelx * b.nelz;
  size_t sm = stokes_smem_bytes<R>();
  auto kern = k_assemble_stokes<R, S>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
    return MW_ERR_CUDA;
  unsigned grid = (unsigned)((nel + EB_S - 1) / EB_S);
  kern<<<grid, EB_S * 18, sm, s>>>(b, in, blocks, (S*)out.VV_Stokes, (S*)out.VV_K, (S*)out.VV_G, (S*)out.VV_GT,
                                   (S*)out.VV_M, (S*)out.VV_M_eta, (S*)out.VV_H, fel, hel);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

}  // namespace mw

using namespace mw;

extern "C" {

size_t mw_assemble_stokes_workspace_bytes(mw_box box) {
  return (size_t)box.nelx * box.nelz * 22 * sizeof(double);
}

int mw_assemble_stokes(mw_box box, int32_t blocks, int32_t precision, mw_stokes_in in, mw_stokes_out out, void* work,
                       size_t work_bytes, void* stream) {
  if (box.nelx <= 0 || box.nelz <= 0 || !out.rhs_f || !out.rhs_h) return MW_ERR_BAD_ARG;
  const bool rhs_only = !out.VV_Stokes && !out.VV_K;
  if (!rhs_only && (blocks ? !(out.VV_K && out.VV_G && out.VV_GT && out.VV_M && out.VV_M_eta && out.VV_H)
                           : !out.VV_Stokes))
    return MW_ERR_BAD_ARG;
  if (work_bytes < mw_assemble_stokes_workspace_bytes(box)) return MW_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  int64_t nel = (int64_t)box.nelx * box.nelz;
  double* fel = (double*)work;
  double* hel = fel + nel * 18;
  int rc = precision == MW_F32 ? launch_stokes<float, float>(box, in, out, blocks, fel, hel, s)
                               : launch_stokes<double, double>(box, in, out, blocks, fel, hel, s);
  if (rc) return rc;
  int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  k_gather_q2<<<grid_for(nn, 256), 256, 0, s>>>(box, 2, fel, out.rhs_f);
  MW_CHECK_LAUNCH();
  int64_t np = (int64_t)(box.nelx + 1) * (box.nelz + 1);
  k_gather_q1<<<grid_for(np, 256), 256, 0, s>>>(box, hel, out.rhs_h);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_stokes_rhs_body(mw_box box, const double* rhoq, const double* gxq, const double* gzq, const double* JxWq,
                       const double* N_V, const uint8_t* bc_fix_V, double* rhs_f, double* rhs_h, void* work,
                       size_t work_bytes, void* stream) {
  if (box.nelx <= 0 || box.nelz <= 0 || !rhs_f || !rhs_h) return MW_ERR_BAD_ARG;
  if (work_bytes < mw_assemble_stokes_workspace_bytes(box)) return MW_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nel = (int64_t)box.nelx * box.nelz;
  double* fel = (double*)work;
  k_body_force<<<grid_for(nel * 9, 256), 256, 0, s>>>(box, rhoq, gxq, gzq, JxWq, N_V, bc_fix_V, fel);
  MW_CHECK_LAUNCH();
  const int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  k_gather_q2<<<grid_for(nn, 256), 256, 0, s>>>(box, 2, fel, rhs_f);
  MW_CHECK_LAUNCH();
  const int64_t np = (int64_t)(box.nelx + 1) * (box.nelz + 1);
  if (cudaMemsetAsync(rhs_h, 0, sizeof(double) * np, s) != cudaSuccess) return MW_ERR_CUDA;
  return MW_OK;
}

size_t mw_assemble_energy_workspace_bytes(mw_box box) {
  return (size_t)box.nelx * box.nelz * 9 * sizeof(double);
}

int mw_assemble_energy(mw_box box, int32_t precision, mw_energy_in in, void* VV_T, double* rhs, void* work,
                       size_t work_bytes, void* stream) {
  if (box.nelx <= 0 || box.nelz <= 0 || !VV_T || !rhs) return MW_ERR_BAD_ARG;
  if (work_bytes < mw_assemble_energy_workspace_bytes(box)) return MW_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  int64_t nel = (int64_t)box.nelx * box.nelz;
  double* bel = (double*)work;
  unsigned grid = (unsigned)((nel + EB_T - 1) / EB_T);
  if (precision == MW_F32) k_assemble_energy<float, float><<<grid, EB_T * 9, 0, s>>>(box, in, (float*)VV_T, bel);
  else k_assemble_energy<double, double><<<grid, EB_T * 9, 0, s>>>(box, in, (double*)VV_T, bel);
  MW_CHECK_LAUNCH();
  int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  k_gather_q2<<<grid_for(nn, 256), 256, 0, s>>>(box, 1, bel, rhs);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

}  // extern "C"
