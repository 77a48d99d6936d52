// Particle-in-cell kernels for the Cartesian box (sm_100a).
//
// Reference: pic_functions.py (locate :108-137, interpolate :85-101 and :18-37, advect :180-292,
// element projection :603-650, nodal projections :659-1053) and the material hooks
// experiment0.py:230-264 / experiment1.py:91-113.
//
// Layout: particles are SoA (x, z, r, t: f64; iel: i32; active: u8), one thread per particle,
// grid-stride loops sized to a multiple of the SM count.  Projections are atomic-free and
// deterministic: particles are binned by element (counting sort, each bin sorted by particle
// index), so every element and node sums its particles in particle-index order -- the order of
// the reference's sequential loops.  This file is compiled with -fmad=false so the basis and
// weight arithmetic rounds exactly as the reference's unfused double-precision code.
#include <cstdlib>

#include "common.cuh"

namespace mw {

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("MW_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

int grid_for(int64_t n, int threads, int waves) {
  int64_t need = (n + threads - 1) / threads;
  int64_t cap = (int64_t)num_sms() * waves;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

// Element containing point (x, z): pic_functions.py:29-31 (int() truncates toward zero).
// Returns false when the truncated quotient does not fit an int (the reference would index
// out of bounds there).
MW_D bool element_of(const mw_box& b, double x, double z, int64_t* e) {
  double qx = x / b.hx, qz = z / b.hz;
  if (!(qx > -2147483648.0 && qx < 2147483647.0 && qz > -2147483648.0 && qz < 2147483647.0)) return false;
  int ielx = (int)qx, ielz = (int)qz;
  *e = (int64_t)b.nelx * ielz + ielx;
  return true;
}

// x_V / z_V of local node 0 of element e: build_velocity_mesh.py:116-117 computes i*hx/2.
MW_D double xv0(const mw_box& b, int ex) { return ((double)(2 * ex) * b.hx) / 2; }
MW_D double zv0(const mw_box& b, int ez) { return ((double)(2 * ez) * b.hz) / 2; }

template <typename F>
MW_D double q2_dot(const double* N, const F& nodal, int ex, int ez, int nnx) {
  double acc = N[0] * nodal(q2_node(ex, ez, 0, nnx));
  for (int k = 1; k < 9; ++k) acc = acc + N[k] * nodal(q2_node(ex, ez, k, nnx));
  return acc;
}

// ------------------------------------------------------------------------------------------
__global__ void k_locate(mw_box b, int64_t n, const uint8_t* __restrict__ active,
                         const double* __restrict__ x, const double* __restrict__ z,
                         double* __restrict__ r, double* __restrict__ t, int32_t* __restrict__ iel,
                         int32_t* err) {
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!active[i]) { r[i] = 0.0; t[i] = 0.0; iel[i] = 0; continue; }
    double xi = x[i], zi = z[i];
    int64_t e;
    if (!element_of(b, xi, zi, &e) || e < 0 || e >= nel) {
      set_flag(err, MW_FLAG_ELEMENT_RANGE);
      r[i] = 0.0; t[i] = 0.0; iel[i] = -1;
      continue;
    }
    int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
    double rr = ((xi - xv0(b, ex)) / b.hx - 0.5) * 2;
    double tt = ((zi - zv0(b, ez)) / b.hz - 0.5) * 2;
    if (rr < -1.0 || rr > 1.0) set_flag(err, MW_FLAG_R_OUT_OF_BOUNDS);
    if (tt < -1.0 || tt > 1.0) set_flag(err, MW_FLAG_T_OUT_OF_BOUNDS);
    r[i] = rr; t[i] = tt; iel[i] = (int32_t)e;
  }
}

// ------------------------------------------------------------------------------------------
struct FieldSet {
  const double* in[MW_MAX_FIELDS];
  double* out[MW_MAX_FIELDS];
  int n;
};

__global__ void k_interp(mw_box b, int64_t n, const uint8_t* __restrict__ active, const double* __restrict__ r,
                         const double* __restrict__ t, const int32_t* __restrict__ iel, FieldSet fs) {
  const int nnx = 2 * b.nelx + 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!active[i]) {
      for (int f = 0; f < fs.n; ++f) fs.out[f][i] = 0.0;
      continue;
    }
    double N[9];
    q2_basis<double>(r[i], t[i], N);
    int e = iel[i];
    int ex = e % b.nelx, ez = e / b.nelx;
    for (int f = 0; f < fs.n; ++f) {
      const double* phi = fs.in[f];
      fs.out[f][i] = q2_dot(N, [&](int64_t j) { return __ldg(phi + j); }, ex, ez, nnx);
    }
  }
}

// Interpolation of the five nodal fields the time loop needs (meeuuw.py:1118-1125) fused with
// the material model (experiment0.py:254-264 / experiment1.py:104-111).
__global__ void k_interp_material(mw_box b, int64_t n, const uint8_t* __restrict__ active,
                                  const double* __restrict__ r, const double* __restrict__ t,
                                  const int32_t* __restrict__ iel, const int8_t* __restrict__ mat,
                                  mw_nodal5 nodal, mw_material m, mw_swarm_props out) {
  const int nnx = 2 * b.nelx + 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[5] = {0, 0, 0, 0, 0};
    bool act = active[i] != 0;
    if (act) {
      double N[9];
      q2_basis<double>(r[i], t[i], N);
      int e = iel[i];
      int ex = e % b.nelx, ez = e / b.nelx;
      const double* fl[5] = {nodal.exx, nodal.ezz, nodal.exz, nodal.q, nodal.T};
      for (int f = 0; f < 5; ++f) {
        if (fl[f] == nullptr) continue;
        const double* phi = fl[f];
        v[f] = q2_dot(N, [&](int64_t j) { return __ldg(phi + j); }, ex, ez, nnx);
      }
    }
    if (out.exx) out.exx[i] = v[0];
    if (out.ezz) out.ezz[i] = v[1];
    if (out.exz) out.exz[i] = v[2];
    if (out.p) out.p[i] = v[3];
    if (out.T) out.T[i] = v[4];
    double rho, eta, hcond, hcapa, hprod, alpha;
    if (m.kind == MW_MATERIAL_TWO) {
      int id = mat ? (int)mat[i] : 0;
      id = id < 0 ? 0 : (id > 7 ? 7 : id);
      rho = act ? m.mat_rho[id] : 0.0;
      eta = act ? m.mat_eta[id] : 0.0;
      hcond = hcapa = hprod = alpha = 0.0;
    } else {
      double T = v[4];
      rho = m.rho0 * (1 - m.alphaT * T);
      eta = m.fk_gamma != 0.0 ? exp(-m.fk_gamma * T) : m.eta0;
      hcond = m.hcond; hcapa = m.hcapa; hprod = m.hprod; alpha = m.alphaT;
    }
    out.rho[i] = rho;
    out.eta[i] = eta;
    if (out.hcond) out.hcond[i] = hcond;
    if (out.hcapa) out.hcapa[i] = hcapa;
    if (out.hprod) out.hprod[i] = hprod;
    if (out.alpha) out.alpha[i] = alpha;
  }
}

// ------------------------------------------------------------------------------------------
// Velocity at a point: pic_functions.py:18-37.  The element index is the reference's, including
// the case x == Lx that wraps into the next row; indices outside the mesh set a flag.
MW_D bool vel_at(const mw_box& b, int64_t nel, int nnx, double xp, double zp, const double* __restrict__ u,
                 const double* __restrict__ w, double* up, double* wp, int32_t* err) {
  int64_t e;
  if (!element_of(b, xp, zp, &e) || e < 0 || e >= nel) {
    set_flag(err, MW_FLAG_ELEMENT_RANGE);
    *up = 0.0; *wp = 0.0;
    return false;
  }
  int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
  double rp = ((xp - xv0(b, ex)) / b.hx - 0.5) * 2;
  double tp = ((zp - zv0(b, ez)) / b.hz - 0.5) * 2;
  double N[9];
  q2_basis<double>(rp, tp, N);
  *up = q2_dot(N, [&](int64_t j) { return __ldg(u + j); }, ex, ez, nnx);
  *wp = q2_dot(N, [&](int64_t j) { return __ldg(w + j); }, ex, ez, nnx);
  return true;
}

MW_D bool outside(const mw_box& b, double x, double z) { return x < 0 || x > b.Lx || z < 0 || z > b.Lz; }

__global__ void k_advect(mw_box b, int rk, double dt_host, const double* __restrict__ dt_dev, int64_t n, double* __restrict__ x, double* __restrict__ z,
                         uint8_t* __restrict__ active, const double* __restrict__ u, const double* __restrict__ w,
                         double* __restrict__ up_out, double* __restrict__ wp_out, int32_t* err) {
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  const int nnx = 2 * b.nelx + 1;
  const double dt = dt_dev ? *dt_dev : dt_host;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double su = 0.0, sw = 0.0;
    bool act = active[i] != 0;
    if (act) {
      double xA = x[i], zA = z[i], uA, wA;
      vel_at(b, nel, nnx, xA, zA, u, w, &uA, &wA, err);
      if (rk == 1) {                                                  // :220-231
        su = uA; sw = wA;
        double xn = xA + uA * dt, zn = zA + wA * dt;
        x[i] = xn; z[i] = zn;
        if (outside(b, xn, zn)) act = false;
      } else {
        double xB = xA + uA * dt / 2.0, zB = zA + wA * dt / 2.0;      // :239-240
        if (outside(b, xB, zB)) {
          act = false;
        } else {
          double uB, wB;
          vel_at(b, nel, nnx, xB, zB, u, w, &uB, &wB, err);
          if (rk == 2) {                                              // :244-248
            x[i] = xA + uB * dt; z[i] = zA + wB * dt;
            su = uB; sw = wB;
          } else {
            double xC = xA + uB * dt / 2.0, zC = zA + wB * dt / 2.0;  // :265-266
            if (outside(b, xC, zC)) {
              act = false;
            } else {
              double uC, wC;
              vel_at(b, nel, nnx, xC, zC, u, w, &uC, &wC, err);
              double xD = xA + uC * dt, zD = zA + wC * dt;            // :271-272
              if (outside(b, xD, zD)) {
                act = false;
              } else {
                double uD, wD;
                vel_at(b, nel, nnx, xD, zD, u, w, &uD, &wD, err);
                su = (uA + 2 * uB + 2 * uC + uD) / 6;                 // :277-280
                sw = (wA + 2 * wB + 2 * wC + wD) / 6;
                x[i] = xA + su * dt; z[i] = zA + sw * dt;
              }
            }
          }
        }
      }
      if (!act) active[i] = 0;
    }
    if (!act) { x[i] = 0.0; z[i] = 0.0; }                              // :287-290
    if (up_out) up_out[i] = su;
    if (wp_out) wp_out[i] = sw;
  }
}

// ------------------------------------------------------------------------------------------
// Binning: counts -> exclusive scan -> scatter -> per-bin sort by particle index.
__global__ void k_count(int64_t n, int32_t nel, const uint8_t* __restrict__ active, const int32_t* __restrict__ iel,
                        int32_t* __restrict__ counts, int32_t* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!active[i]) continue;
    int e = iel[i];
    if (e < 0 || e >= nel) { set_flag(err, MW_FLAG_ELEMENT_RANGE); continue; }
    atomicAdd(counts + e, 1);
  }
}

// Block-level exclusive scan of int32 (1024 items per block), writing block totals.
__global__ void k_scan_block(const int32_t* __restrict__ in, int32_t* __restrict__ out, int32_t* __restrict__ block_sums,
                             int64_t n) {
  __shared__ int32_t warp_sums[32];
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int32_t v = i < n ? in[i] : 0;
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    int32_t s = lane < nw ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  int32_t base = wid > 0 ? warp_sums[wid - 1] : 0;
  if (i < n) out[i] = base + incl - v;
  if (threadIdx.x == blockDim.x - 1 && block_sums) block_sums[blockIdx.x] = base + incl;
}

__global__ void k_scan_add(int32_t* __restrict__ out, const int32_t* __restrict__ block_prefix, int64_t n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] += block_prefix[blockIdx.x];
}

__global__ void k_scatter(int64_t n, int32_t nel, const uint8_t* __restrict__ active, const int32_t* __restrict__ iel,
                          const int32_t* __restrict__ offsets, int32_t* __restrict__ cursor, int32_t* __restrict__ order) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!active[i]) continue;
    int e = iel[i];
    if (e < 0 || e >= nel) continue;
    int pos = offsets[e] + atomicAdd(cursor + e, 1);
    order[pos] = (int32_t)i;
  }
}

// Sort each bin by particle index (bins hold ~16-25 particles; insertion sort in registers/L1).
__global__ void k_sort_bins(int32_t nel, const int32_t* __restrict__ offsets, int32_t* __restrict__ order) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    int b0 = offsets[e], b1 = offsets[e + 1];
    for (int i = b0 + 1; i < b1; ++i) {
      int v = order[i];
      int j = i - 1;
      while (j >= b0 && order[j] > v) { order[j + 1] = order[j]; --j; }
      order[j + 1] = v;
    }
  }
}

// offsets[0..n) = exclusive prefix sum of counts[0..n); n <= 1024*1024 (two scan levels).
static int scan_exclusive(const int32_t* in, int32_t* out, int64_t n, int32_t* scratch, size_t scratch_ints,
                          cudaStream_t s) {
  const int T = 1024;
  int64_t nb = (n + T - 1) / T;
  if (nb > T || (size_t)(2 * nb) > scratch_ints) return MW_ERR_WORKSPACE;
  int32_t* bsum = scratch;
  int32_t* bpre = scratch + nb;
  k_scan_block<<<(unsigned)nb, T, 0, s>>>(in, out, bsum, n);
  MW_CHECK_LAUNCH();
  k_scan_block<<<1, T, 0, s>>>(bsum, bpre, nullptr, nb);
  MW_CHECK_LAUNCH();
  k_scan_add<<<(unsigned)nb, T, 0, s>>>(out, bpre, n);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

__global__ void k_total(const int32_t* counts, int32_t* offsets, int64_t n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) offsets[n] = n > 0 ? offsets[n - 1] + counts[n - 1] : 0;
}

// ------------------------------------------------------------------------------------------
MW_D double avg_transform(int averaging, double v) {
  if (averaging == MW_AVG_GEOMETRIC) return log10(v);
  if (averaging == MW_AVG_HARMONIC) return 1.0 / v;
  return v;
}

// pic_functions.py:603-650 over the sorted bins.
__global__ void k_project_elements(int32_t nel, const int32_t* __restrict__ offsets, const int32_t* __restrict__ order,
                                   const double* __restrict__ rho, const double* __restrict__ eta, int averaging,
                                   double* __restrict__ rho_e, double* __restrict__ eta_e, int32_t* err) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    int b0 = offsets[e], b1 = offsets[e + 1];
    double sr = 0.0, se = 0.0;
    for (int j = b0; j < b1; ++j) {
      int p = order[j];
      sr = sr + rho[p];
      se = se + avg_transform(averaging, eta[p]);
    }
    double c = (double)(b1 - b0);
    if (b1 == b0) set_flag(err, MW_FLAG_EMPTY_ELEMENT);
    rho_e[e] = sr / c;
    if (averaging == MW_AVG_GEOMETRIC) eta_e[e] = pow(10.0, se / c);
    else if (averaging == MW_AVG_HARMONIC) eta_e[e] = c / se;
    else eta_e[e] = se / c;
  }
}

// Corner-node projection (pic_functions.py:659-1053): node (2i, 2j) sums the particles of its
// (up to) four incident elements, merged in particle-index order.
struct ProjFields {
  const double* phi[MW_MAX_FIELDS];
  double* out[MW_MAX_FIELDS];
  int averaging[MW_MAX_FIELDS];
  int n;
};

MW_D void corner_weight(int flavour, int k, double r, double t, bool* use, double* w) {
  if (flavour == 1) { *use = true; *w = 1.0; return; }
  if (flavour == 2) {
    *use = true;
    if (k == 0) *w = 0.25 * (1 - r) * (1 - t);
    else if (k == 1) *w = 0.25 * (1 + r) * (1 - t);
    else if (k == 2) *w = 0.25 * (1 + r) * (1 + t);
    else *w = 0.25 * (1 - r) * (1 + t);
    return;
  }
  bool u;
  if (k == 0) u = (r <= 0 && t <= 0);
  else if (k == 1) u = (r >= 0 && t <= 0);
  else if (k == 2) u = (r >= 0 && t >= 0);
  else u = (r <= 0 && t >= 0);
  *use = u;
  if (flavour == 3) { *w = 1.0; return; }
  if (k == 0) *w = -r * -t;
  else if (k == 1) *w = (1 - r) * -t;
  else if (k == 2) *w = (1 - r) * (1 - t);
  else *w = -r * (1 - t);
}

__global__ void k_project_corners(mw_box b, int flavour, const int32_t* __restrict__ offsets,
                                  const int32_t* __restrict__ order, const double* __restrict__ r,
                                  const double* __restrict__ t, ProjFields pf) {
  const int ncx = b.nelx + 1, ncz = b.nelz + 1;
  const int nnx = 2 * b.nelx + 1;
  const int64_t ncorner = (int64_t)ncx * ncz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncorner; c += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(c % ncx), j = (int)(c / ncx);
    // incident elements and this node's local corner index in each
    int pos[4], end[4], kk[4];
    int ne = 0;
    const int ex[4] = {i, i - 1, i - 1, i};
    const int ez[4] = {j, j, j - 1, j - 1};
    for (int k = 0; k < 4; ++k) {
      if (ex[k] < 0 || ex[k] >= b.nelx || ez[k] < 0 || ez[k] >= b.nelz) continue;
      int e = ez[k] * b.nelx + ex[k];
      pos[ne] = offsets[e]; end[ne] = offsets[e + 1]; kk[ne] = k; ++ne;
    }
    double acc[MW_MAX_FIELDS];
    double cnt = 0.0;
    for (int f = 0; f < pf.n; ++f) acc[f] = 0.0;
    while (true) {
      int best = -1, bp = 0x7fffffff;
      for (int s = 0; s < ne; ++s)
        if (pos[s] < end[s]) { int p = order[pos[s]]; if (p < bp) { bp = p; best = s; } }
      if (best < 0) break;
      ++pos[best];
      bool use; double w;
      corner_weight(flavour, kk[best], r[bp], t[bp], &use, &w);
      if (!use) continue;
      if (flavour == 1 || flavour == 3) cnt = cnt + 1.0;
      else cnt = cnt + 1 * w;
      for (int f = 0; f < pf.n; ++f) {
        double v = avg_transform(pf.averaging[f], pf.phi[f][bp]);
        acc[f] = (flavour == 1 || flavour == 3) ? acc[f] + v : acc[f] + v * w;
      }
    }
    int64_t node = (int64_t)(2 * j) * nnx + 2 * i;
    for (int f = 0; f < pf.n; ++f) {
      double v;
      if (pf.averaging[f] == MW_AVG_GEOMETRIC) v = pow(10.0, acc[f] / cnt);
      else if (pf.averaging[f] == MW_AVG_HARMONIC) v = cnt / acc[f];
      else v = acc[f] / cnt;
      pf.out[f][node] = v;
    }
  }
}

// Faster form of the same projection: each element sums its particles (in particle-index order)
// per corner into partials (nel x 4 x (nfield+1) doubles), then each corner node adds the partials
// of its incident elements in ascending element order and applies the averaging.  The sums agree
// with the reference's particle-ordered sums to rounding (different association).
__global__ void k_project_elem_partials(mw_box b, int flavour, const int32_t* __restrict__ offsets,
                                        const int32_t* __restrict__ order, const double* __restrict__ r,
                                        const double* __restrict__ t, ProjFields pf, double* __restrict__ part) {
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  const int nf1 = pf.n + 1;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    double acc[4][MW_MAX_FIELDS + 1];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int f = 0; f <= MW_MAX_FIELDS; ++f) acc[k][f] = 0.0;
    const int b0 = offsets[e], b1 = offsets[e + 1];
    for (int j = b0; j < b1; ++j) {
      const int p = order[j];
      const double rp = r[p], tp = t[p];
      double v[MW_MAX_FIELDS];
#pragma unroll
      for (int f = 0; f < MW_MAX_FIELDS; ++f)
        if (f < pf.n) v[f] = avg_transform(pf.averaging[f], pf.phi[f][p]);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        bool use; double w;
        corner_weight(flavour, k, rp, tp, &use, &w);
        if (!use) continue;
        const bool plain = (flavour == 1 || flavour == 3);
        acc[k][MW_MAX_FIELDS] = plain ? acc[k][MW_MAX_FIELDS] + 1.0 : acc[k][MW_MAX_FIELDS] + 1 * w;
#pragma unroll
        for (int f = 0; f < MW_MAX_FIELDS; ++f)
          if (f < pf.n) acc[k][f] = plain ? acc[k][f] + v[f] : acc[k][f] + v[f] * w;
      }
    }
    double* o = part + e * 4 * nf1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      for (int f = 0; f < pf.n; ++f) o[k * nf1 + f] = acc[k][f];
      o[k * nf1 + pf.n] = acc[k][MW_MAX_FIELDS];
    }
  }
}

__global__ void k_project_corner_finish(mw_box b, ProjFields pf, const double* __restrict__ part) {
  const int ncx = b.nelx + 1, ncz = b.nelz + 1;
  const int nnx = 2 * b.nelx + 1;
  const int nf1 = pf.n + 1;
  const int64_t ncorner = (int64_t)ncx * ncz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncorner; c += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % ncx), j = (int)(c / ncx);
    double acc[MW_MAX_FIELDS + 1];
    for (int f = 0; f <= pf.n; ++f) acc[f] = 0.0;
    // ascending element order: (j-1,i-1) corner 2, (j-1,i) corner 3, (j,i-1) corner 1, (j,i) corner 0
    for (int s2 = 0; s2 < 4; ++s2) {
      const int ex = (s2 & 1) ? i : i - 1, ez = (s2 & 2) ? j : j - 1;
      if (ex < 0 || ex >= b.nelx || ez < 0 || ez >= b.nelz) continue;
      const int k = s2 == 0 ? 2 : (s2 == 1 ? 3 : (s2 == 2 ? 1 : 0));
      const double* o = part + ((int64_t)ez * b.nelx + ex) * 4 * nf1 + k * nf1;
      for (int f = 0; f <= pf.n; ++f) acc[f] += o[f];
    }
    const double cnt = acc[pf.n];
    const int64_t node = (int64_t)(2 * j) * nnx + 2 * i;
    for (int f = 0; f < pf.n; ++f) {
      double v;
      if (pf.averaging[f] == MW_AVG_GEOMETRIC) v = pow(10.0, acc[f] / cnt);
      else if (pf.averaging[f] == MW_AVG_HARMONIC) v = cnt / acc[f];
      else v = acc[f] / cnt;
      pf.out[f][node] = v;
    }
  }
}

// Edge and centre nodes from the corners: pic_functions.py:801-809.
__global__ void k_fill_q2(mw_box b, ProjFields pf) {
  const int nnx = 2 * b.nelx + 1, nnz = 2 * b.nelz + 1;
  const int64_t nn = (int64_t)nnx * nnz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    int ix = (int)(n % nnx), iz = (int)(n / nnx);
    bool ox = ix & 1, oz = iz & 1;
    if (!ox && !oz) continue;
    for (int f = 0; f < pf.n; ++f) {
      double* o = pf.out[f];
      double v;
      if (ox && !oz) v = 0.50 * (o[n - 1] + o[n + 1]);
      else if (!ox && oz) v = 0.50 * (o[n - nnx] + o[n + nnx]);
      else v = 0.25 * (((o[n - nnx - 1] + o[n - nnx + 1]) + o[n + nnx + 1]) + o[n + nnx - 1]);
      o[n] = v;
    }
  }
}

// ------------------------------------------------------------------------------------------
// phiq[e, q] = sum_k N[q, k] phi[node_k(e)]: project_nodal_field_onto_qpoints.py:12-62.
__global__ void k_nodal_to_q(mw_box b, int space, const double* __restrict__ Ntab, const double* __restrict__ phi,
                             double* __restrict__ phiq) {
  __shared__ double Ns[81];
  int m = (space == MW_SPACE_Q2) ? 9 : 4;
  for (int i = threadIdx.x; i < 9 * m; i += blockDim.x) Ns[i] = Ntab[i];
  __syncthreads();
  const int64_t nq = (int64_t)b.nelx * b.nelz * 9;
  const int nnx = 2 * b.nelx + 1;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nq; g += (int64_t)gridDim.x * blockDim.x) {
    int64_t e = g / 9;
    int q = (int)(g % 9);
    int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
    double acc;
    if (space == MW_SPACE_Q2) {
      acc = Ns[q * 9] * phi[q2_node(ex, ez, 0, nnx)];
      for (int k = 1; k < 9; ++k) acc = acc + Ns[q * 9 + k] * phi[q2_node(ex, ez, k, nnx)];
    } else if (space == MW_SPACE_Q1_ON_V) {
      acc = Ns[q * 4] * phi[q2_node(ex, ez, 0, nnx)];
      for (int k = 1; k < 4; ++k) acc = acc + Ns[q * 4 + k] * phi[q2_node(ex, ez, k, nnx)];
    } else {
      acc = Ns[q * 4] * phi[q1_node(ex, ez, 0, b.nelx)];
      for (int k = 1; k < 4; ++k) acc = acc + Ns[q * 4 + k] * phi[q1_node(ex, ez, k, b.nelx)];
    }
    phiq[g] = acc;
  }
}

}  // namespace mw

using namespace mw;

static bool box_ok(const mw_box& b) { return b.nelx > 0 && b.nelz > 0 && b.hx > 0 && b.hz > 0; }

extern "C" {

int mw_locate_box(mw_box box, int64_t n, const uint8_t* active, const double* x, const double* z, double* r,
                  double* t, int32_t* iel, int32_t* err, void* stream) {
  if (!box_ok(box) || n < 0) return MW_ERR_BAD_ARG;
  if (n == 0) return MW_OK;
  k_locate<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(box, n, active, x, z, r, t, iel, err);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_interp_q2(mw_box box, int64_t n, const uint8_t* active, const double* r, const double* t, const int32_t* iel,
                 int32_t nfield, const double* const* fields, double* const* out, void* stream) {
  if (!box_ok(box) || n < 0 || nfield < 1 || nfield > MW_MAX_FIELDS) return MW_ERR_BAD_ARG;
  if (n == 0) return MW_OK;
  FieldSet fs;
  fs.n = nfield;
  for (int f = 0; f < nfield; ++f) { fs.in[f] = fields[f]; fs.out[f] = out[f]; }
  k_interp<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(box, n, active, r, t, iel, fs);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_interp_material(mw_box box, int64_t n, const uint8_t* active, const double* r, const double* t,
                       const int32_t* iel, const int8_t* mat, mw_nodal5 nodal, mw_material m, mw_swarm_props out,
                       void* stream) {
  if (!box_ok(box) || n < 0 || !out.rho || !out.eta) return MW_ERR_BAD_ARG;
  if (n == 0) return MW_OK;
  k_interp_material<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(box, n, active, r, t, iel, mat, nodal, m, out);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_advect_box(mw_box box, int32_t rk, double dt, const double* dt_dev, int64_t n, double* x, double* z,
                  uint8_t* active, const double* u, const double* w, double* up, double* wp, int32_t* err,
                  void* stream) {
  if (!box_ok(box) || n < 0 || !(rk == 1 || rk == 2 || rk == 4)) return MW_ERR_BAD_ARG;
  if (n == 0) return MW_OK;
  k_advect<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(box, rk, dt, dt_dev, n, x, z, active, u, w, up, wp, err);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

size_t mw_bin_workspace_bytes(int32_t nel) {
  int64_t nb = ((int64_t)nel + 1 + 1023) / 1024;
  return (size_t)((int64_t)nel + 2 * nb + 16) * sizeof(int32_t);
}

int mw_bin_particles(int32_t nel, int64_t n, const uint8_t* active, const int32_t* iel, int32_t* counts,
                     int32_t* offsets, int32_t* order, void* work, size_t work_bytes, int32_t* err, void* stream) {
  if (nel <= 0 || n < 0 || (int64_t)nel > 1024LL * 1024LL) return MW_ERR_BAD_ARG;
  if (work_bytes < mw_bin_workspace_bytes(nel)) return MW_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  int32_t* cursor = (int32_t*)work;
  int32_t* scratch = cursor + nel;
  size_t scratch_ints = work_bytes / sizeof(int32_t) - nel;
  if (cudaMemsetAsync(counts, 0, sizeof(int32_t) * nel, s) != cudaSuccess) return MW_ERR_CUDA;
  if (cudaMemsetAsync(cursor, 0, sizeof(int32_t) * nel, s) != cudaSuccess) return MW_ERR_CUDA;
  if (n > 0) {
    k_count<<<grid_for(n, 256), 256, 0, s>>>(n, nel, active, iel, counts, err);
    MW_CHECK_LAUNCH();
  }
  int rc = scan_exclusive(counts, offsets, nel, scratch, scratch_ints, s);
  if (rc) return rc;
  k_total<<<1, 32, 0, s>>>(counts, offsets, nel);
  MW_CHECK_LAUNCH();
  if (n > 0) {
    k_scatter<<<grid_for(n, 256), 256, 0, s>>>(n, nel, active, iel, offsets, cursor, order);
    MW_CHECK_LAUNCH();
    k_sort_bins<<<grid_for(nel, 128), 128, 0, s>>>(nel, offsets, order);
    MW_CHECK_LAUNCH();
  }
  return MW_OK;
}

int mw_project_elements(int32_t nel, const int32_t* offsets, const int32_t* order, const double* rho,
                        const double* eta, int32_t averaging, double* rho_e, double* eta_e, int32_t* err,
                        void* stream) {
  if (nel <= 0 || averaging < 0 || averaging > 2) return MW_ERR_BAD_ARG;
  k_project_elements<<<grid_for(nel, 128), 128, 0, (cudaStream_t)stream>>>(nel, offsets, order, rho, eta, averaging,
                                                                             rho_e, eta_e, err);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

size_t mw_project_nodes_workspace_bytes(mw_box box, int32_t nfield) {
  return (size_t)box.nelx * box.nelz * 4 * (nfield + 1) * sizeof(double);
}

int mw_project_nodes(mw_box box, int32_t flavour, int32_t nfield, const int32_t* averaging, const int32_t* offsets,
                     const int32_t* order, const double* r, const double* t, const double* const* phi,
                     double* const* phi_nodal, void* work, size_t work_bytes, void* stream) {
  if (!box_ok(box) || flavour < 1 || flavour > 4 || nfield < 1 || nfield > MW_MAX_FIELDS) return MW_ERR_BAD_ARG;
  ProjFields pf;
  pf.n = nfield;
  for (int f = 0; f < nfield; ++f) {
    if (averaging[f] < 0 || averaging[f] > 2) return MW_ERR_BAD_ARG;
    pf.phi[f] = phi[f]; pf.out[f] = phi_nodal[f]; pf.averaging[f] = averaging[f];
  }
  cudaStream_t s = (cudaStream_t)stream;
  int64_t nc = (int64_t)(box.nelx + 1) * (box.nelz + 1);
  if (work && work_bytes >= mw_project_nodes_workspace_bytes(box, nfield)) {
    int64_t nel = (int64_t)box.nelx * box.nelz;
    k_project_elem_partials<<<grid_for(nel, 128), 128, 0, s>>>(box, flavour, offsets, order, r, t, pf, (double*)work);
    MW_CHECK_LAUNCH();
    k_project_corner_finish<<<grid_for(nc, 256), 256, 0, s>>>(box, pf, (const double*)work);
  } else {
    // no workspace: per-node merge of the incident elements' particles in particle-index order
    k_project_corners<<<grid_for(nc, 128), 128, 0, s>>>(box, flavour, offsets, order, r, t, pf);
  }
  MW_CHECK_LAUNCH();
  int64_t nn = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1);
  k_fill_q2<<<grid_for(nn, 256), 256, 0, s>>>(box, pf);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_nodal_to_qpoints(mw_box box, int32_t space, const double* N, const double* phi, double* phiq, void* stream) {
  if (!box_ok(box) || space < 0 || space > 2) return MW_ERR_BAD_ARG;
  int64_t nq = (int64_t)box.nelx * box.nelz * 9;
  k_nodal_to_q<<<grid_for(nq, 256), 256, 0, (cudaStream_t)stream>>>(box, space, N, phi, phiq);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

}  // extern "C"
