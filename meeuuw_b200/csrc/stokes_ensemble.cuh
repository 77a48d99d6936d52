// The Stokes solves of an ensemble of models in one launch: one thread-block cluster per model runs
// that model's whole mixed-precision solve -- FP64 iterative refinement around Schur-complement CG
// sweeps (cd_u_eta / uzawa3) whose inner K solves are multigrid-preconditioned CG in FP32 -- with
// cluster barriers between its phases instead of kernel launches and graph conditional nodes.
// Every model keeps its own hierarchy, iteration counts and convergence tests; the clusters never
// wait on one another.
//
// Part of stokes.cu's translation unit (included at its end): it runs the same tile apply
// (apply_tile), restriction and prolongation bodies, node stencils of G and G^T and mass-matrix
// Chebyshev steps as the per-model launches, in the same phase order.  The dot products are summed
// in a different order (per-thread, per-warp, per-CTA, then over the cluster's CTAs in rank order),
// so results agree with the per-model solve to rounding, not bit for bit.
//
// Reference: the solver loops of cd_u_eta / uzawa3 (the Schur-complement CG recurrences that
// stokes_solve_record records per model); mixed refinement and inner multigrid are this library's.

#include <cooperative_groups.h>

namespace mw {

constexpr int ENS_CLUSTER = 8;                     // CTAs per model
constexpr int ENS_THREADS = APPLY_THREADS;         // one tile apply per CTA at a time
constexpr int ENS_NT = ENS_CLUSTER * ENS_THREADS;
constexpr int ENS_WARPS = ENS_THREADS / 32;
#ifndef MW_ENS_MINB
#define MW_ENS_MINB 4                              // resident CTAs per SM the registers are sized for
#endif

// one model of the ensemble: its FP32 hierarchy, inner PCG vectors, FP64 fine-level vectors and
// the solve's result scalars (the slots mw_stokes_device_info reads)
struct EnsMember {
  int nlev, dense, nd, pad;
  const double* Ainv;
  TailLevel<float> L[MAXLEV];
  float *xr, *r, *p, *Ap;
  LevelGeo g;
  const uint8_t* fixV;
  const double *eta64, *diag64, *etae_w, *mdiag, *medi;
  const double *f, *h;
  double *V, *P;
  double *fr, *hr, *cV, *cP, *z, *rP, *wP, *dP, *Gd, *GTz, *RV, *RP, *tP, *tP2;
  double* sc;
};

struct EnsParams {
  double tol, inner_rtol, sweep_reduction, sweep_target;
  int max_inner, max_outer, max_refine, mass_iters, use_guess, weighted;
};

// Shared memory of the cluster solve: the tile apply's arrays (one layout at a time), cluster
// reduction slots, the G tables and element mass matrix, the model's descriptor.
union EnsApplySmem {
  ApplySmem<float, AM_APPLY> a0;
  ApplySmem<float, AM_RESID> a1;
  ApplySmem<float, AM_CHEB> a2;
  ApplySmem<float, AM_CHEB_Z> a3;
  ApplySmem<double, AM_RESID> d1;
};

struct EnsCtx {
  EnsApplySmem* tile;
  double* swarp;      // [ENS_WARPS][4]
  double* sred;       // [2][4], read by every CTA of the cluster
  const double *gx, *gz, *Me;
  const EnsMember* M;
  int rank, t0;
  int phase;
};

// Sum of NV values over the cluster's threads, returned to every thread (deterministic: warp
// shuffles, warps in order, then the CTAs' sums in rank order).  Ends with a cluster barrier
// (release / acquire), so it also orders every global write before it with every read after it.
template <int NV>
MW_D void ens_sum(EnsCtx& c, double (&v)[NV]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i)
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) c.swarp[wid * 4 + i] = v[i];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double s = 0;
      for (int w = 0; w < ENS_WARPS; ++w) s += c.swarp[w * 4 + i];
      c.sred[c.phase * 4 + i] = s;
    }
  cluster_barrier();
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double s = 0;
    for (int r = 0; r < ENS_CLUSTER; ++r) s += cl.map_shared_rank(c.sred, r)[c.phase * 4 + i];
    v[i] = s;
  }
  c.phase ^= 1;     // the other slot next time: a CTA rewrites this one only after another barrier
}

// One operator apply of level g by the cluster: its element tiles dealt to the CTAs in turn.
template <typename R, int MODE>
MW_D void ens_apply(EnsCtx& c, const LevelGeo& g, const ApplyArgs<R>& a) {
  const int ntx = (g.nx + TX - 1) / TX, ntz = (g.nz + TZ - 1) / TZ;
  const ApplyPtrs<R> sm = apply_ptrs(*reinterpret_cast<ApplySmem<R, MODE>*>(c.tile));
  for (int t = c.rank; t < ntx * ntz; t += ENS_CLUSTER) {
    __syncthreads();
    apply_tile<R, MODE>(g, a, t % ntx, t / ntx, sm);
  }
  cluster_barrier();
}

// Chebyshev smoothing of level l (x in xs, the other buffer ts), as smooth() launches it
MW_D void ens_smooth(EnsCtx& c, const TailLevel<float>& L, const float* b, float*& xs, float*& ts, int degree,
                     bool zero_start, bool first_done) {
  auto step = [&](int mode_z, int k) {
    ApplyArgs<float> a;
    memset(&a, 0, sizeof(a));
    a.u = xs; a.eta = L.eta; a.fix = L.fix; a.diag = L.diag; a.yV = L.d; a.bV = b; a.d = L.d; a.xo = ts;
    a.cheb = L.cheb + 2 * k;
    if (mode_z) {
      a.cheb0 = L.cheb;
      ens_apply<float, AM_CHEB_Z>(c, L.g, a);
    } else {
      ens_apply<float, AM_CHEB>(c, L.g, a);
    }
    float* t = xs; xs = ts; ts = t;
  };
  int k0 = 1;
  if (first_done) {
    // x = d = (1/theta) D^-1 b were written by the restriction
  } else if (zero_start) {
    if (degree >= 2) {                               // steps 0 and 1 in one pass
      step(1, 1);
      k0 = 2;
    } else {
      const float cf = (float)L.cheb[1];
      const int64_t n = 2LL * L.g.nnx * L.g.nnz;
      for (int64_t i = c.t0; i < n; i += ENS_NT) {
        const float v = cf * b[i] / L.diag[i];
        xs[i] = v; L.d[i] = v;
      }
      cluster_barrier();
    }
  } else {
    step(0, 0);                                      // restart from the current x
  }
  for (int k = k0; k < degree; ++k) step(0, k);
}

// One V-cycle with right-hand side b0 on the finest level; xs / ts hold every level's x / other
// buffer (kept across cycles).  Returns where the finest level's x is.
MW_D float* ens_vcycle(EnsCtx& c, const float* b0, float** xs, float** ts) {
  const EnsMember& M = *c.M;
  const int nl = M.nlev;
  for (int l = 0; l + 1 < nl; ++l) {
    const TailLevel<float>& F = M.L[l];
    const TailLevel<float>& C = M.L[l + 1];
    const float* b = l == 0 ? b0 : F.b;
    ens_smooth(c, F, b, xs[l], ts[l], F.deg, l == 0, l > 0);
    ApplyArgs<float> a;
    memset(&a, 0, sizeof(a));
    a.u = xs[l]; a.eta = F.eta; a.fix = F.fix; a.diag = F.diag; a.yV = F.r; a.bV = b;
    ens_apply<float, AM_RESID>(c, F.g, a);
    const bool fuse = !(l + 2 == nl && M.dense);
    const double c0 = fuse ? C.cheb[1] : 0.0;
    const int64_t ncn = (int64_t)C.g.nnx * C.g.nnz;
    for (int64_t n = c.t0; n < ncn; n += ENS_NT)
      restrict_node(F.g, C.g, F.r, C.fix, C.b, c0, fuse, C.diag, xs[l + 1], C.d, n);
    cluster_barrier();
  }
  {                                                  // coarsest level
    const int l = nl - 1;
    const TailLevel<float>& L = M.L[l];
    const float* b = l == 0 ? b0 : L.b;
    if (M.dense) {
      const int lane = threadIdx.x & 31, warp = c.t0 >> 5;
      for (int row = warp; row < M.nd; row += ENS_NT / 32) {
        double s = 0;
        for (int j = lane; j < M.nd; j += 32) s += M.Ainv[(int64_t)row * M.nd + j] * (double)b[j];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) xs[l][row] = (float)s;
      }
      cluster_barrier();
    } else {
      const bool fd = l > 0;
      ens_smooth(c, L, b, xs[l], ts[l], MAXDEG, !fd, fd);
    }
  }
  for (int l = nl - 2; l >= 0; --l) {
    const TailLevel<float>& F = M.L[l];
    const TailLevel<float>& C = M.L[l + 1];
    const int64_t nfn = (int64_t)F.g.nnx * F.g.nnz;
    for (int64_t n = c.t0; n < nfn; n += ENS_NT) prolong_node(F.g, C.g, xs[l + 1], F.fix, xs[l], n);
    cluster_barrier();
    ens_smooth(c, F, l == 0 ? b0 : F.b, xs[l], ts[l], F.deg, false, false);
  }
  return xs[0];
}

constexpr double ENS_INNER_BUDGET = 40000, ENS_OUTER_BUDGET = 4000;

// Multigrid-preconditioned CG for K x = b in FP32 (b, x in FP64), the recurrences of pcg_K_dev.
MW_D void ens_pcg(EnsCtx& c, float** xs, float** ts, const double* b, double* x, double rtol, int maxit,
                  double& inner, int& status) {
  const EnsMember& M = *c.M;
  const int64_t n = 2LL * M.g.nnx * M.g.nnz;
  float *xr = M.xr, *r = M.r, *p = M.p, *Ap = M.Ap;
  double v1[1] = {0.0};
  for (int64_t i = c.t0; i < n; i += ENS_NT) {
    const float ri = (float)b[i];
    r[i] = ri;
    xr[i] = 0.0f;
    v1[0] += (double)ri * (double)ri;
  }
  ens_sum<1>(c, v1);
  const double bb = v1[0];
  float* z = ens_vcycle(c, r, xs, ts);
  v1[0] = 0.0;
  for (int64_t i = c.t0; i < n; i += ENS_NT) {
    p[i] = z[i];
    v1[0] += (double)r[i] * (double)z[i];
  }
  ens_sum<1>(c, v1);
  double rz = v1[0];
  int it = 0;
  bool go = bb > 0 && isfinite(bb);
  while (go) {
    ApplyArgs<float> a;
    memset(&a, 0, sizeof(a));
    a.u = p; a.eta = M.L[0].eta; a.fix = M.L[0].fix; a.diag = M.L[0].diag; a.yV = Ap;
    ens_apply<float, AM_APPLY>(c, M.L[0].g, a);
    v1[0] = 0.0;
    for (int64_t i = c.t0; i < n; i += ENS_NT) v1[0] += (double)p[i] * (double)Ap[i];
    ens_sum<1>(c, v1);
    const double al = rz / v1[0];
    v1[0] = 0.0;
    for (int64_t i = c.t0; i < n; i += ENS_NT) {
      xr[i] = (float)((double)xr[i] + al * (double)p[i]);
      const float ri = (float)((double)r[i] - al * (double)Ap[i]);
      r[i] = ri;
      v1[0] += (double)ri * (double)ri;
    }
    ens_sum<1>(c, v1);
    const double rr = v1[0];
    ++it;
    go = isfinite(rr) && rr > rtol * rtol * bb && it < maxit;
    if (go && inner + it >= ENS_INNER_BUDGET) { status = 3; go = false; }
    if (go) {
      z = ens_vcycle(c, r, xs, ts);
      v1[0] = 0.0;
      for (int64_t i = c.t0; i < n; i += ENS_NT) v1[0] += (double)r[i] * (double)z[i];
      ens_sum<1>(c, v1);
      const double be = v1[0] / rz;
      for (int64_t i = c.t0; i < n; i += ENS_NT) p[i] = (float)((double)z[i] + be * (double)p[i]);
      rz = v1[0];
      cluster_barrier();
    }
  }
  for (int64_t i = c.t0; i < n; i += ENS_NT) x[i] = (double)xr[i];
  cluster_barrier();
  inner += it;
}

// y = b - G p (b may be null: y = G p) on the velocity nodes
MW_D void ens_grad(EnsCtx& c, const double* p, const double* b, double* y) {
  const EnsMember& M = *c.M;
  double cx, cz;
  grad_scales(M.g, &cx, &cz);
  const int64_t nn = (int64_t)M.g.nnx * M.g.nnz;
  for (int64_t n = c.t0; n < nn; n += ENS_NT)
    grad_node(M.g, p, M.fixV, b, y, (int)(n % M.g.nnx), (int)(n / M.g.nnx), c.gx, c.gz, cx, cz);
  cluster_barrier();
}

// x -= mean(x) over the pressure nodes
MW_D void ens_remove_mean(EnsCtx& c, double* x, int64_t n) {
  double v1[1] = {0.0};
  for (int64_t i = c.t0; i < n; i += ENS_NT) v1[0] += x[i];
  ens_sum<1>(c, v1);
  const double m = v1[0] / (double)n;
  for (int64_t i = c.t0; i < n; i += ENS_NT) x[i] -= m;
  cluster_barrier();
}

// x = (the fixed-interval Chebyshev-Jacobi steps of mass_solve_kernels) M_w^-1 b
MW_D void ens_mass_solve(EnsCtx& c, const double* w, const double* b, double* x, int iters) {
  const EnsMember& M = *c.M;
  const int64_t n = (int64_t)(M.g.nx + 1) * (M.g.nz + 1);
  const double* dg = w ? M.medi : M.mdiag;
  const double a = 0.25 / 1.02, bb = 2.25 * 1.02;
  const double theta = 0.5 * (bb + a), delta = 0.5 * (bb - a), sigma = theta / delta;
  double rho = 1.0 / sigma;
  double* bufs[2] = {x, M.tP};
  const int K = iters < 1 ? 1 : iters;
  for (int k = 0; k < K; ++k) {
    double c1 = 0.0, c2 = 1.0 / theta;
    if (k > 0) {
      const double rn = 1.0 / (2.0 * sigma - rho);
      c1 = rn * rho;
      c2 = 2.0 * rn / delta;
      rho = rn;
    }
    const double* xin = bufs[(K - k) % 2];
    double* xout = bufs[(K - 1 - k) % 2];
    for (int64_t i = c.t0; i < n; i += ENS_NT) mass_cheb_node(M.g, w, b, xin, xout, M.tP2, dg, c1, c2, k == 0, c.Me, i);
    cluster_barrier();
  }
}

// Schur-complement CG (uzawa_dev's recurrences) on (f, h) for the correction (V, P), FP32 inner
// solves, until the Schur residual has dropped by `red`.
MW_D void ens_uzawa(EnsCtx& c, const EnsParams& prm, float** xs, float** ts, const double* f, const double* h,
                    double* V, double* P, double red, double& inner, double& outer, int& status) {
  const EnsMember& M = *c.M;
  const LevelGeo& g = M.g;
  const int64_t nv = 2LL * g.nnx * g.nnz, np = (int64_t)(g.nx + 1) * (g.nz + 1);
  const double* w = prm.weighted ? M.etae_w : nullptr;
  double cx, cz;
  grad_scales(g, &cx, &cz);
  const int ncx = g.nx + 1;
  ens_grad(c, P, f, M.Gd);                                      // V = K^-1 (f - G P)
  ens_pcg(c, xs, ts, M.Gd, V, prm.inner_rtol, prm.max_inner, inner, status);
  for (int64_t n = c.t0; n < np; n += ENS_NT) {                 // rho = G^T V - h
    const double t = div_node(g, V, M.fixV, (int)(n % ncx), (int)(n / ncx), c.gx, c.gz, cx, cz);
    M.rP[n] = t + -1.0 * h[n];
  }
  cluster_barrier();
  ens_remove_mean(c, M.rP, np);
  ens_mass_solve(c, w, M.rP, M.wP, prm.mass_iters);
  ens_remove_mean(c, M.wP, np);
  double v2[2] = {0.0, 0.0};
  for (int64_t n = c.t0; n < np; n += ENS_NT) {
    M.dP[n] = M.wP[n];
    v2[0] += M.rP[n] * M.wP[n];
    v2[1] += M.rP[n] * M.rP[n];
  }
  ens_sum<2>(c, v2);
  double rw = v2[0];
  const double rr0 = v2[1];
  int it = 0;
  bool go = prm.max_outer > 0 && isfinite(rr0) && status == 0;
  while (go) {
    ens_grad(c, M.dP, nullptr, M.Gd);
    ens_pcg(c, xs, ts, M.Gd, M.z, prm.inner_rtol, prm.max_inner, inner, status);
    double v1[1] = {0.0};
    for (int64_t n = c.t0; n < np; n += ENS_NT) {
      const double t = div_node(g, M.z, M.fixV, (int)(n % ncx), (int)(n / ncx), c.gx, c.gz, cx, cz);
      M.GTz[n] = t;
      v1[0] += M.dP[n] * t;
    }
    ens_sum<1>(c, v1);
    const double ap = 1.0 * (rw / v1[0]), am = -1.0 * (rw / v1[0]);
    for (int64_t n = c.t0; n < nv; n += ENS_NT) V[n] = V[n] + am * M.z[n];
    v1[0] = 0.0;
    for (int64_t n = c.t0; n < np; n += ENS_NT) {
      P[n] = P[n] + ap * M.dP[n];
      const double t = M.rP[n] + am * M.GTz[n];
      M.rP[n] = t;
      v1[0] += t;
    }
    ens_sum<1>(c, v1);                                          // remove_mean(rP)
    {
      const double m = v1[0] / (double)np;
      for (int64_t n = c.t0; n < np; n += ENS_NT) M.rP[n] -= m;
      cluster_barrier();
    }
    ens_mass_solve(c, w, M.rP, M.wP, prm.mass_iters);
    ens_remove_mean(c, M.wP, np);
    v1[0] = 0.0;
    for (int64_t n = c.t0; n < np; n += ENS_NT) v1[0] += M.rP[n] * M.wP[n];
    ens_sum<1>(c, v1);
    const double rwn = v1[0], be = rwn / rw;
    v1[0] = 0.0;
    for (int64_t n = c.t0; n < np; n += ENS_NT) {
      M.dP[n] = M.wP[n] + be * M.dP[n];
      v1[0] += M.rP[n] * M.rP[n];
    }
    ens_sum<1>(c, v1);
    rw = rwn;
    const double rr = v1[0];
    ++it;
    outer += 1;
    go = it < prm.max_outer;
    if (!isfinite(rr)) { status = 2; go = false; }
    if (outer >= ENS_OUTER_BUDGET && status == 0) status = 3;
    if (status != 0) go = false;
    if (rr <= red * red * rr0) go = false;
  }
}

// FP64 residual (RV, RP) = (f, h) - [K G; G^T 0](V, P) and its norm over bnorm
MW_D double ens_true_residual(EnsCtx& c, const double* V, const double* P, double bnorm, double* rv) {
  const EnsMember& M = *c.M;
  ApplyArgs<double> a;
  memset(&a, 0, sizeof(a));
  a.u = V; a.p = P; a.eta = M.eta64; a.fix = M.fixV; a.diag = M.diag64;
  a.yV = M.RV; a.yP = M.RP; a.bV = M.f; a.bP = M.h;
  ens_apply<double, AM_RESID>(c, M.g, a);
  const int64_t nv = 2LL * M.g.nnx * M.g.nnz, np = (int64_t)(M.g.nx + 1) * (M.g.nz + 1);
  double v2[2] = {0.0, 0.0};
  for (int64_t i = c.t0; i < nv; i += ENS_NT) v2[0] += M.RV[i] * M.RV[i];
  for (int64_t i = c.t0; i < np; i += ENS_NT) v2[1] += M.RP[i] * M.RP[i];
  ens_sum<2>(c, v2);
  rv[0] = v2[0];
  rv[1] = v2[1];
  return sqrt(v2[0] + v2[1]) / bnorm;
}

template <typename T>
MW_D void ens_stage(T* dst, const T* src) {         // a struct copied by the CTA's threads, 8 bytes each
  static_assert(sizeof(T) % 8 == 0, "8-byte words");
  for (int i = threadIdx.x; i < (int)(sizeof(T) / 8); i += blockDim.x)
    reinterpret_cast<uint64_t*>(dst)[i] = reinterpret_cast<const uint64_t*>(src)[i];
}

__global__ void __cluster_dims__(ENS_CLUSTER, 1, 1) __launch_bounds__(ENS_THREADS, MW_ENS_MINB)
k_ens_stokes(const EnsMember* __restrict__ members, const int* __restrict__ order, int n_members, EnsParams prm) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char ens_dyn[];
  __shared__ __align__(16) EnsMember sM;
  __shared__ double swarp[ENS_WARPS * 4], sred[8], gx[36], gz[36], Me[16];
  const int cid = blockIdx.x / ENS_CLUSTER;
  if (cid >= n_members) return;                      // whole clusters only (the grid is a multiple)
  ens_stage(&sM, &members[order[cid]]);
  if (threadIdx.x < 36) {
    gx[threadIdx.x] = c_ref.GX[threadIdx.x];
    gz[threadIdx.x] = c_ref.GZ[threadIdx.x];
  }
  __syncthreads();
  if (threadIdx.x < 16) Me[threadIdx.x] = mass_entry(sM.g, threadIdx.x / 4, threadIdx.x % 4);
  EnsCtx c;
  c.tile = reinterpret_cast<EnsApplySmem*>(ens_dyn);
  c.swarp = swarp; c.sred = sred; c.gx = gx; c.gz = gz; c.Me = Me; c.M = &sM;
  c.rank = (int)cluster_rank();
  c.t0 = c.rank * ENS_THREADS + threadIdx.x;
  c.phase = 0;
  const EnsMember& M = sM;
  float* xs[MAXLEV];
  float* ts[MAXLEV];
  for (int l = 0; l < M.nlev; ++l) { xs[l] = M.L[l].x; ts[l] = M.L[l].t; }
  const int64_t nv = 2LL * M.g.nnx * M.g.nnz, np = (int64_t)(M.g.nx + 1) * (M.g.nz + 1);
  if (!prm.use_guess) {
    for (int64_t i = c.t0; i < nv; i += ENS_NT) M.V[i] = 0.0;
    for (int64_t i = c.t0; i < np; i += ENS_NT) M.P[i] = 0.0;
  }
  double v2[2] = {0.0, 0.0};
  for (int64_t i = c.t0; i < nv; i += ENS_NT) v2[0] += M.f[i] * M.f[i];
  for (int64_t i = c.t0; i < np; i += ENS_NT) v2[1] += M.h[i] * M.h[i];
  ens_sum<2>(c, v2);                                 // (also orders the zeroing and the Me tables)
  const double bnorm = sqrt(v2[0] + v2[1]);
  double inner = 0, outer = 0, nref = 0, trv[2];
  int status = 0;
  double rel = ens_true_residual(c, M.V, M.P, bnorm, trv);
  const double rel0 = rel;
  bool go = isfinite(rel) && rel > prm.tol && prm.max_refine > 0;
  while (go) {                                       // refinement sweeps on the FP64 residual
    for (int64_t i = c.t0; i < nv; i += ENS_NT) { M.fr[i] = M.RV[i]; M.cV[i] = 0.0; }
    for (int64_t i = c.t0; i < np; i += ENS_NT) { M.hr[i] = M.RP[i]; M.cP[i] = 0.0; }
    cluster_barrier();
    const double red = sweep_target_reduction(prm.sweep_reduction, prm.sweep_target, prm.tol, rel);
    ens_uzawa(c, prm, xs, ts, M.fr, M.hr, M.cV, M.cP, red, inner, outer, status);
    for (int64_t i = c.t0; i < nv; i += ENS_NT) M.V[i] = M.V[i] + 1.0 * M.cV[i];
    for (int64_t i = c.t0; i < np; i += ENS_NT) M.P[i] = M.P[i] + 1.0 * M.cP[i];
    cluster_barrier();
    rel = ens_true_residual(c, M.V, M.P, bnorm, trv);
    nref += 1;
    go = isfinite(rel) && rel > prm.tol && nref < (double)prm.max_refine && status == 0;
  }
  // no CTA leaves while another may still read its shared memory (the last ens_sum's remote loads)
  cluster_barrier();
  if (c.rank == 0 && threadIdx.x == 0) {
    double* sc = M.sc;
    sc[S_BB] = v2[0]; sc[S_BH] = v2[1]; sc[S_BNORM] = bnorm;
    sc[T_RV] = trv[0]; sc[T_RP] = trv[1]; sc[T_REL] = rel; sc[S_REL0] = rel0;
    sc[S_NREF] = nref; sc[I_OUTER] = outer; sc[I_INNER] = inner; sc[I_STATUS] = status;
  }
}

}  // namespace mw

// ---------------------------------------------------------------- C ABI
struct mw_stokes_ensemble {
  int n = 0;
  std::vector<mw_stokes*> solvers;   // to refuse a solve while a model's hierarchy is out of date
  mw::EnsMember* d_members = nullptr;
  int* d_order = nullptr;
  ~mw_stokes_ensemble() {
    if (d_members) cudaFree(d_members);
    if (d_order) cudaFree(d_order);
  }
};

extern "C" {

int mw_stokes_ensemble_create(mw_stokes* const* S, const double* const* f, const double* const* h,
                              double* const* V, double* const* P, int32_t n, mw_stokes_ensemble** out) {
  using namespace mw;
  if (!S || !f || !h || !V || !P || !out || n <= 0) return MW_ERR_BAD_ARG;
  *out = nullptr;
  std::vector<EnsMember> mem(n);
  std::vector<std::pair<int64_t, int>> size(n);
  for (int i = 0; i < n; ++i) {
    mw_stokes* s = S[i];
    if (!s || !s->has32 || !f[i] || !h[i] || !V[i] || !P[i]) return MW_ERR_BAD_ARG;
    if (((uintptr_t)f[i] % 16) || ((uintptr_t)V[i] % 16)) return MW_ERR_BAD_ARG;
    EnsMember& m = mem[i];
    memset(&m, 0, sizeof(m));
    const Hierarchy<float>& H = s->H32;
    m.nlev = H.nlev; m.dense = H.dense ? 1 : 0; m.nd = H.nd; m.Ainv = H.Ainv;
    for (int l = 0; l < H.nlev; ++l) {
      const Level<float>& L = H.L[l];
      m.L[l] = TailLevel<float>{L.g, L.eta, L.fix, L.diag, L.x, L.t, L.b, L.r, L.d, L.cheb, L.deg};
    }
    m.xr = s->pc32[0]; m.r = s->pc32[1]; m.p = s->pc32[3]; m.Ap = s->pc32[4];
    m.g = s->fine; m.fixV = s->fixV;
    m.eta64 = s->etaq64; m.diag64 = s->diag64; m.etae_w = s->etae_w; m.mdiag = s->mdiag; m.medi = s->medi;
    m.f = f[i]; m.h = h[i]; m.V = V[i]; m.P = P[i];
    m.fr = s->f; m.hr = s->h; m.cV = s->cV; m.cP = s->cP; m.z = s->z; m.rP = s->rP; m.wP = s->wP; m.dP = s->dP;
    m.Gd = s->Gd; m.GTz = s->GTz; m.RV = s->RV; m.RP = s->RP; m.tP = s->tP; m.tP2 = s->tP2;
    m.sc = s->sc;
    size[i] = {-(int64_t)s->fine.nx * s->fine.nz, i};
  }
  std::sort(size.begin(), size.end());              // largest models first
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = size[i].second;
  auto* E = new mw_stokes_ensemble();
  E->n = n;
  E->solvers.assign(S, S + n);
  if (cudaMalloc(&E->d_members, sizeof(EnsMember) * n) != cudaSuccess ||
      cudaMalloc(&E->d_order, sizeof(int) * n) != cudaSuccess ||
      cudaMemcpy(E->d_members, mem.data(), sizeof(EnsMember) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(E->d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    delete E;
    return MW_ERR_CUDA;
  }
  *out = E;
  return MW_OK;
}

int mw_stokes_ensemble_destroy(mw_stokes_ensemble* E) {
  delete E;
  return MW_OK;
}

int mw_stokes_prepare(mw_stokes* S, int32_t precision, void* stream) {
  if (!S) return MW_ERR_BAD_ARG;
  return mw::ensure_hierarchy(S, precision == MW_F64 ? MW_F64 : MW_F32, (cudaStream_t)stream);
}

int mw_stokes_ensemble_solve(mw_stokes_ensemble* E, mw_solve_params sp, void* stream) {
  using namespace mw;
  if (!E || sp.precision != MW_F32 || sp.history) return MW_ERR_BAD_ARG;
  for (const mw_stokes* s : E->solvers)            // viscosity set but hierarchy not prepared
    if (s->dirty32) return MW_ERR_BAD_ARG;
  EnsParams p;
  p.tol = sp.tol; p.inner_rtol = sp.inner_rtol; p.sweep_reduction = sp.sweep_reduction; p.sweep_target = sp.sweep_target;
  p.max_inner = sp.max_inner; p.max_outer = sp.max_outer; p.max_refine = sp.max_refine;
  p.mass_iters = sp.mass_iters; p.use_guess = sp.use_guess; p.weighted = sp.scheme == MW_SCHEME_UZAWA3 ? 0 : 1;
  const size_t smem = sizeof(EnsApplySmem);
  pdl_launch(k_ens_stokes, E->n * ENS_CLUSTER, ENS_THREADS, smem, (cudaStream_t)stream,
             (const EnsMember*)E->d_members, (const int*)E->d_order, E->n, p);
  return cudaGetLastError() == cudaSuccess ? MW_OK : MW_ERR_CUDA;
}

}  // extern "C"
