// Particle-in-cell kernels for the Cartesian box (sm_100a).
//
// Reference: pic_functions.py (locate :108-137, element projection :603-650, nodal projections
// :659-1053, least squares :1061-1285, population control :1621-1812).  Interpolation and
// advection are in advect.cu.
//
// Layout: particles are SoA (x, z, r, t: f64; iel: i32; active: u8), one thread per particle,
// grid-stride loops sized to a multiple of the SM count.  Projections are atomic-free and
// deterministic: particles are binned by element (counting sort, each bin sorted by particle
// index), so every element and node sums its particles in particle-index order -- the order of
// the reference's sequential loops.  This file is compiled with -fmad=false so the basis and
// weight arithmetic rounds exactly as the reference's unfused double-precision code.
#include <cstdlib>

#include "common.cuh"
#include "pic_common.cuh"

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
// NF: register capacity for the fields (pf.n <= NF), so that the accumulators of the usual two- or
// four-field projections do not occupy the registers of eight.
template <int NF>
__global__ void k_project_elem_partials(mw_box b, int flavour, const int32_t* __restrict__ offsets,
                                        const int32_t* __restrict__ order, const double* __restrict__ r,
                                        const double* __restrict__ t, ProjFields pf, double* __restrict__ part) {
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  const int nf1 = pf.n + 1;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    double acc[4][NF + 1];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int f = 0; f <= NF; ++f) acc[k][f] = 0.0;
    const int b0 = offsets[e], b1 = offsets[e + 1];
    for (int j = b0; j < b1; ++j) {
      const int p = order[j];
      const double rp = r[p], tp = t[p];
      double v[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f)
        if (f < pf.n) v[f] = avg_transform(pf.averaging[f], pf.phi[f][p]);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        bool use; double w;
        corner_weight(flavour, k, rp, tp, &use, &w);
        if (!use) continue;
        const bool plain = (flavour == 1 || flavour == 3);
        acc[k][NF] = plain ? acc[k][NF] + 1.0 : acc[k][NF] + 1 * w;
#pragma unroll
        for (int f = 0; f < NF; ++f)
          if (f < pf.n) acc[k][f] = plain ? acc[k][f] + v[f] : acc[k][f] + v[f] * w;
      }
    }
    double* o = part + e * 4 * nf1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
      for (int f = 0; f < NF; ++f)
        if (f < pf.n) o[k * nf1 + f] = acc[k][f];
      o[k * nf1 + pf.n] = acc[k][NF];
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

// ------------------------------------------------------------------------------------------
// Least-squares particle fits (pic_functions.py:1098-1285) and their slope limiter
// (pic_functions.py:1068-1089).  One thread per element sums the normal equations over the
// element's bin in particle-index order -- each accumulator in the reference's order, products
// formed as the reference writes them ((sx*sx)*sz, sx*(sz*sz), (v*sx)*sz) -- then solves them by
// Gaussian elimination with partial pivoting (the reference calls LAPACK's solve).
struct LsFields {
  const double* phi[MW_MAX_FIELDS];
  double* coef[MW_MAX_FIELDS];
  double* fmin[MW_MAX_FIELDS];
  double* fmax[MW_MAX_FIELDS];
  int n;
};

// Python's min(a, b): a unless b < a
MW_D double py_min(double a, double b) { return b < a ? b : a; }
MW_D double py_sign(double v) { return v < 0 ? -1.0 : 1.0; }

// limiter(c_0, c_1, c_2, S, L, h), pic_functions.py:1068-1089
MW_D void ls_limiter(double c0, double& c1, double& c2, double S, double L, double h) {
  const double k_u = py_min(c0 - S, L - c0);
  double k_l = (fabs(c1) + fabs(c2)) * h / 2;
  if (k_l > k_u) {
    const double c_max = k_u * 2 / h;
    c1 = py_sign(c1) * py_min(fabs(c1), c_max);
    c2 = py_sign(c2) * py_min(fabs(c2), c_max);
  }
  k_l = (fabs(c1) + fabs(c2)) * h / 2;
  if (k_l > k_u) {
    const double c_change = (k_l - k_u) / h;
    c1 = py_sign(c1) * (fabs(c1) - c_change);
    c2 = py_sign(c2) * (fabs(c2) - c_change);
  }
}

// Solve A x = b in place (b -> x) for the NC x NC system: Gaussian elimination, partial pivoting
// (first largest magnitude in the column).  Returns false on a zero pivot.
template <int NC>
MW_D bool small_solve(double (&A)[NC][NC], double (&b)[NC]) {
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    int piv = k;
    double best = fabs(A[k][k]);
#pragma unroll
    for (int i = k + 1; i < NC; ++i)
      if (fabs(A[i][k]) > best) { best = fabs(A[i][k]); piv = i; }
    if (best == 0.0) return false;
    if (piv != k) {
#pragma unroll
      for (int j = 0; j < NC; ++j) { double tmp = A[k][j]; A[k][j] = A[piv][j]; A[piv][j] = tmp; }
      double tmp = b[k]; b[k] = b[piv]; b[piv] = tmp;
    }
#pragma unroll
    for (int i = k + 1; i < NC; ++i) {
      const double l = A[i][k] / A[k][k];
#pragma unroll
      for (int j = k + 1; j < NC; ++j) A[i][j] = A[i][j] - l * A[k][j];
      b[i] = b[i] - l * b[k];
    }
  }
#pragma unroll
  for (int k = NC - 1; k >= 0; --k) {
    double s = b[k];
#pragma unroll
    for (int j = k + 1; j < NC; ++j) s = s - A[k][j] * b[j];
    b[k] = s / A[k][k];
  }
  return true;
}

// element centre x_V[icon_V[8, iel]] = i hx / 2 with i = 2 ex + 1 (build_velocity_mesh.py:116-117)
MW_D double x_centre(const mw_box& b, int ex) { return ((double)(2 * ex + 1) * b.hx) / 2; }
MW_D double z_centre(const mw_box& b, int ez) { return ((double)(2 * ez + 1) * b.hz) / 2; }

template <int NC>
__global__ void k_ls_fit(mw_box b, const int32_t* __restrict__ offsets, const int32_t* __restrict__ order,
                         const double* __restrict__ x, const double* __restrict__ z, LsFields f, double limit_h,
                         int32_t* err) {
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    const int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
    const double xe = x_centre(b, ex), ze = z_centre(b, ez);
    const int b0 = offsets[e], b1 = offsets[e + 1];
    if (b1 == b0) { set_flag(err, MW_FLAG_EMPTY_ELEMENT); continue; }
    double A[NC][NC];
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) A[i][j] = 0.0;
    A[0][0] = (double)(b1 - b0);
    for (int j = b0; j < b1; ++j) {                       // pic_functions.py:1134-1146 / :1226-1246
      const int p = order[j];
      const double sx = x[p] - xe, sz = z[p] - ze;
      A[0][1] += sx;
      A[0][2] += sz;
      if (NC == 4) A[0][3] += sx * sz;
      A[1][1] += sx * sx;
      A[1][2] += sx * sz;
      if (NC == 4) A[1][3] += (sx * sx) * sz;
      A[2][2] += sz * sz;
      if (NC == 4) {
        A[2][3] += sx * (sz * sz);
        A[3][3] += (sx * sx) * (sz * sz);
      }
    }
#pragma unroll
    for (int i = 1; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < i; ++j) A[i][j] = A[j][i];
    for (int fi = 0; fi < f.n; ++fi) {
      const double* phi = f.phi[fi];
      double rhs[NC];
#pragma unroll
      for (int i = 0; i < NC; ++i) rhs[i] = 0.0;
      double vmin = 0.0, vmax = 0.0;
      for (int j = b0; j < b1; ++j) {
        const int p = order[j];
        const double sx = x[p] - xe, sz = z[p] - ze, v = phi[p];
        rhs[0] += v;
        rhs[1] += v * sx;
        rhs[2] += v * sz;
        if (NC == 4) rhs[3] += (v * sx) * sz;
        if (j == b0 || v < vmin) vmin = v;                 // np.min / np.max (:1164-1167)
        if (j == b0 || v > vmax) vmax = v;
      }
      double M[NC][NC];
#pragma unroll
      for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) M[i][j] = A[i][j];
      if (!small_solve<NC>(M, rhs)) set_flag(err, MW_FLAG_NONFINITE);
      if (NC == 3 && limit_h > 0.0) ls_limiter(rhs[0], rhs[1], rhs[2], vmin, vmax, limit_h);   // meeuuw.py:1241-1248
#pragma unroll
      for (int i = 0; i < NC; ++i) f.coef[fi][e * NC + i] = rhs[i];
      if (f.fmin[fi]) f.fmin[fi][e] = vmin;
      if (f.fmax[fi]) f.fmax[fi][e] = vmax;
    }
  }
}

// a + b (xq - x_e) + c (zq - z_e) [+ d (xq - x_e)(zq - z_e)] at every qpoint (meeuuw.py:1517-1532)
template <int NC>
__global__ void k_ls_q(mw_box b, const double* __restrict__ coef, const double* __restrict__ xq,
                       const double* __restrict__ zq, double* __restrict__ phiq) {
  const int64_t nq = (int64_t)b.nelx * b.nelz * 9;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nq; g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = g / 9;
    const int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
    const double* c = coef + e * NC;
    const double dx = xq[g] - x_centre(b, ex), dz = zq[g] - z_centre(b, ez);
    double v = c[0] + c[1] * dx + c[2] * dz;
    if (NC == 4) v = v + c[3] * dx * dz;
    phiq[g] = v;
  }
}

// ------------------------------------------------------------------------------------------
// Population control (pic_functions.py:1621-1812).
//
// numpy's pairwise summation of a float64 array (np.add.reduce, so np.mean / np.average): < 8
// values sequentially from 0; up to 128 in eight interleaved partial sums combined as a tree,
// then the remainder; longer arrays split at an 8-aligned half.  v(k) is the k-th value.
template <typename V>
MW_D double np_pairwise(const V& v, int k0, int n) {
  if (n < 8) {
    double res = 0.0;
    for (int i = 0; i < n; ++i) res += v(k0 + i);
    return res;
  }
  if (n <= 128) {
    double r[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = v(k0 + j);
    int i = 8;
    for (; i < n - (n % 8); i += 8)
#pragma unroll
      for (int j = 0; j < 8; ++j) r[j] += v(k0 + i + j);
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) res += v(k0 + i);
    return res;
  }
  int n2 = n / 2;
  n2 -= n2 % 8;
  return np_pairwise(v, k0, n2) + np_pairwise(v, k0 + n2, n - n2);
}

// counter-based uniform [0, 1) numbers (SplitMix64 finaliser, 53-bit mantissa)
MW_D double splitmix_u01(uint64_t seed, uint64_t k) {
  uint64_t zz = seed + (k + 1) * 0x9E3779B97F4A7C15ull;
  zz = (zz ^ (zz >> 30)) * 0xBF58476D1CE4E5B9ull;
  zz = (zz ^ (zz >> 27)) * 0x94D049BB133111EBull;
  zz ^= zz >> 31;
  return (double)(zz >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void k_pc_need(int32_t nel, int32_t nmin, const int32_t* __restrict__ counts, int32_t* __restrict__ need) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t d = nmin - counts[e];
    need[e] = d > 0 ? d : 0;                                      // :1655-1657
  }
}

__global__ void k_pc_flag(int64_t n, const uint8_t* __restrict__ active, int32_t* __restrict__ flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = active[i] ? 0 : 1;
}

__global__ void k_pc_list(int64_t n, const int32_t* __restrict__ flag, const int32_t* __restrict__ off,
                          int32_t* __restrict__ avail) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (flag[i]) avail[off[i]] = (int32_t)i;                     // :1680-1688, index order
}

// totals: need_off[nel] (particles needed), avail_off[n] (inactive particles)
__global__ void k_pc_check(const int32_t* __restrict__ need_total, const int32_t* __restrict__ avail_total,
                           int64_t max_new, int32_t* __restrict__ added, int32_t* err) {
  if (threadIdx.x || blockIdx.x) return;
  const int32_t need = *need_total, avail = *avail_total;
  int32_t a = need;
  if (need > avail) { set_flag(err, MW_FLAG_POP_UNAVAILABLE); a = 0; }      // :1722-1733
  else if ((int64_t)need > max_new) { set_flag(err, MW_FLAG_POP_DRAWS); a = 0; }
  *added = a;
}

struct PcFields {
  double* f[MW_MAX_FIELDS];
  int n;
};

// One thread per added particle j: its element (need_off[e] <= j < need_off[e + 1]), its particle
// (avail[j]), its position from two uniform numbers, the nearest particle's material and the
// element particles' means of the `avg` fields (eta, u, w on the box path; :1739-1799).  The
// element's particles are its step-start bin filtered by the current active flags, read before any
// flag changes (k_pc_commit sets them); added particles are inactive, so no thread reads a value
// another one writes.
__global__ void k_pc_fill(mw_box b, const int32_t* __restrict__ need_off, const int32_t* __restrict__ offsets,
                          const int32_t* __restrict__ order, const int32_t* __restrict__ avail,
                          const int32_t* __restrict__ added, const uint8_t* __restrict__ active, int32_t* iel,
                          double* r, double* t, double* x, double* z, int8_t* mat, int32_t* source, PcFields avg,
                          const double* __restrict__ draws, uint64_t seed, int64_t max_new, int32_t* err) {
  const int32_t total = *added;
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  const int nnx = 2 * b.nelx + 1;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < max_new && j < total;
       j += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = nel - 1;                                // last e with need_off[e] <= j
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) / 2;
      if (need_off[mid] <= j) lo = mid; else hi = mid - 1;
    }
    const int64_t e = lo;
    const int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
    const int b0 = offsets[e], b1 = offsets[e + 1];
    int m = 0;
    for (int k = b0; k < b1; ++k) m += active[order[k]] ? 1 : 0;
    if (m == 0) { set_flag(err, MW_FLAG_POP_MASK_EMPTY); continue; }      // :1747-1748
    const int pid = avail[j];
    const double lo_ = -0.95, hi_ = 0.95;                       // random.uniform(-0.95, 0.95)
    const double u0 = draws ? draws[2 * j] : splitmix_u01(seed, 2 * (uint64_t)j);
    const double u1 = draws ? draws[2 * j + 1] : splitmix_u01(seed, 2 * (uint64_t)j + 1);
    const double rr = lo_ + (hi_ - lo_) * u0, tt = lo_ + (hi_ - lo_) * u1;
    double N[9];
    q2_basis<double>(rr, tt, N);
    double xn = 0.0, zn = 0.0;
    for (int k = 0; k < 9; ++k) {                                 // np.dot(N, x_V[icon_V[:, iel]])
      const int64_t nd = q2_node(ex, ez, k, nnx);
      const int ix = (int)(nd % nnx), iz = (int)(nd / nnx);
      xn = xn + N[k] * (((double)ix * b.hx) / 2);
      zn = zn + N[k] * (((double)iz * b.hz) / 2);
    }
    // nearest particle (the first in index order on ties, as np.argmin)
    double best = 0.0;
    int bi = -1;
    for (int k = b0; k < b1; ++k) {
      const int q = order[k];
      if (!active[q]) continue;
      const double dx = x[q] - xn, dz = z[q] - zn;
      const double d = dx * dx + dz * dz;
      if (bi < 0 || d < best) { best = d; bi = q; }
    }
    auto nth = [&](int kk) -> int {                              // the kk-th particle of the mask
      int c = 0;
      for (int k = b0; k < b1; ++k) {
        const int q = order[k];
        if (!active[q]) continue;
        if (c == kk) return q;
        ++c;
      }
      return order[b0];
    };
    for (int fi = 0; fi < avg.n; ++fi) {                          // np.average(field[mask])
      double* fld = avg.f[fi];
      const double sm = np_pairwise([&](int kk) { return fld[nth(kk)]; }, 0, m);
      fld[pid] = sm / m;
    }
    iel[pid] = (int32_t)e;
    r[pid] = rr;
    t[pid] = tt;
    x[pid] = xn;
    z[pid] = zn;
    if (mat) mat[pid] = mat[bi];
    if (source) source[pid] = bi;
  }
}

__global__ void k_pc_commit(const int32_t* __restrict__ avail, const int32_t* __restrict__ added, int64_t max_new,
                            uint8_t* __restrict__ active) {
  const int32_t total = *added;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < max_new && j < total;
       j += (int64_t)gridDim.x * blockDim.x)
    active[avail[j]] = 1;
}

// Exclusive scan of any length (block scans, recursively over the block totals).
static int scan_any(const int32_t* in, int32_t* out, int64_t n, int32_t* scratch, size_t scratch_ints,
                    cudaStream_t s) {
  const int T = 1024;
  const int64_t nb = (n + T - 1) / T;
  if (nb <= 1) {
    k_scan_block<<<1, T, 0, s>>>(in, out, nullptr, n);
    MW_CHECK_LAUNCH();
    return MW_OK;
  }
  if ((size_t)(2 * nb) > scratch_ints) return MW_ERR_WORKSPACE;
  int32_t* bsum = scratch;
  int32_t* bpre = scratch + nb;
  k_scan_block<<<(unsigned)nb, T, 0, s>>>(in, out, bsum, n);
  MW_CHECK_LAUNCH();
  int rc = scan_any(bsum, bpre, nb, scratch + 2 * nb, scratch_ints - 2 * nb, s);
  if (rc) return rc;
  k_scan_add<<<(unsigned)nb, T, 0, s>>>(out, bpre, n);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

static size_t scan_any_ints(int64_t n) {
  size_t s = 0;
  for (int64_t m = (n + 1023) / 1024; m > 1; m = (m + 1023) / 1024) s += 2 * m;
  return s + 64;
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
    if (nfield <= 2)
      k_project_elem_partials<2><<<grid_for(nel, 128), 128, 0, s>>>(box, flavour, offsets, order, r, t, pf, (double*)work);
    else if (nfield <= 4)
      k_project_elem_partials<4><<<grid_for(nel, 128), 128, 0, s>>>(box, flavour, offsets, order, r, t, pf, (double*)work);
    else
      k_project_elem_partials<MW_MAX_FIELDS><<<grid_for(nel, 128), 128, 0, s>>>(box, flavour, offsets, order, r, t, pf,
                                                                               (double*)work);
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

int mw_ls_fit(mw_box box, int32_t ncoef, const int32_t* offsets, const int32_t* order, const double* x,
              const double* z, mw_ls_fields fields, double limit_h, int32_t* err, void* stream) {
  if (!box_ok(box) || !(ncoef == 3 || ncoef == 4) || fields.n < 1 || fields.n > MW_MAX_FIELDS || !offsets ||
      !order || !x || !z)
    return MW_ERR_BAD_ARG;
  if (ncoef == 4 && limit_h > 0.0) return MW_ERR_BAD_ARG;       // the reference limits P1 fits only
  LsFields f;
  f.n = fields.n;
  for (int i = 0; i < fields.n; ++i) {
    if (!fields.phi[i] || !fields.coef[i]) return MW_ERR_BAD_ARG;
    f.phi[i] = fields.phi[i]; f.coef[i] = fields.coef[i]; f.fmin[i] = fields.fmin[i]; f.fmax[i] = fields.fmax[i];
  }
  const int64_t nel = (int64_t)box.nelx * box.nelz;
  cudaStream_t s = (cudaStream_t)stream;
  if (ncoef == 3) k_ls_fit<3><<<grid_for(nel, 128), 128, 0, s>>>(box, offsets, order, x, z, f, limit_h, err);
  else k_ls_fit<4><<<grid_for(nel, 128), 128, 0, s>>>(box, offsets, order, x, z, f, 0.0, err);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_ls_to_qpoints(mw_box box, int32_t ncoef, const double* coef, const double* xq, const double* zq,
                     double* phiq, void* stream) {
  if (!box_ok(box) || !(ncoef == 3 || ncoef == 4) || !coef || !xq || !zq || !phiq) return MW_ERR_BAD_ARG;
  const int64_t nq = (int64_t)box.nelx * box.nelz * 9;
  cudaStream_t s = (cudaStream_t)stream;
  if (ncoef == 3) k_ls_q<3><<<grid_for(nq, 256), 256, 0, s>>>(box, coef, xq, zq, phiq);
  else k_ls_q<4><<<grid_for(nq, 256), 256, 0, s>>>(box, coef, xq, zq, phiq);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

size_t mw_population_workspace_bytes(int32_t nel, int64_t nparticle) {
  const size_t ints = (size_t)2 * (nel + 1) + (size_t)3 * (nparticle + 1) + scan_any_ints(nel + 1) +
                      scan_any_ints(nparticle + 1) + 64;
  return ints * sizeof(int32_t);
}

int mw_population_control(mw_box box, int32_t nparticle_min, int64_t nparticle, const int32_t* counts,
                          const int32_t* offsets, const int32_t* order, uint8_t* active, int32_t* iel, double* r,
                          double* t, double* x, double* z, int8_t* mat, int32_t* source, mw_pc_fields avg,
                          const double* draws, int64_t max_new, uint64_t seed, int32_t* added, void* work,
                          size_t work_bytes, int32_t* err, void* stream) {
  if (!box_ok(box) || nparticle < 1 || nparticle > INT32_MAX - 1 || !counts || !offsets || !order || !active ||
      !iel || !r || !t || !x || !z || !added || !work || avg.n < 0 || avg.n > MW_MAX_FIELDS)
    return MW_ERR_BAD_ARG;
  PcFields pf;
  pf.n = avg.n;
  for (int i = 0; i < avg.n; ++i) {
    if (!avg.f[i]) return MW_ERR_BAD_ARG;
    pf.f[i] = avg.f[i];
  }
  const int32_t nel = box.nelx * box.nelz;
  if (work_bytes < mw_population_workspace_bytes(nel, nparticle)) return MW_ERR_WORKSPACE;
  if (!draws) max_new = nparticle;                 // the device draws as many numbers as it needs
  if (max_new < 0) return MW_ERR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int32_t* need = (int32_t*)work;
  int32_t* need_off = need + (nel + 1);
  int32_t* flag = need_off + (nel + 1);
  int32_t* avail_off = flag + (nparticle + 1);
  int32_t* avail = avail_off + (nparticle + 1);
  int32_t* scratch = avail + (nparticle + 1);
  const size_t scratch_ints = work_bytes / sizeof(int32_t) - (size_t)(scratch - need);
  k_pc_need<<<grid_for(nel, 256), 256, 0, s>>>(nel, nparticle_min, counts, need);
  MW_CHECK_LAUNCH();
  int rc = scan_any(need, need_off, nel, scratch, scratch_ints, s);
  if (rc) return rc;
  k_total<<<1, 32, 0, s>>>(need, need_off, nel);
  MW_CHECK_LAUNCH();
  k_pc_flag<<<grid_for(nparticle, 256), 256, 0, s>>>(nparticle, active, flag);
  MW_CHECK_LAUNCH();
  rc = scan_any(flag, avail_off, nparticle, scratch, scratch_ints, s);
  if (rc) return rc;
  k_total<<<1, 32, 0, s>>>(flag, avail_off, nparticle);
  MW_CHECK_LAUNCH();
  k_pc_list<<<grid_for(nparticle, 256), 256, 0, s>>>(nparticle, flag, avail_off, avail);
  MW_CHECK_LAUNCH();
  k_pc_check<<<1, 32, 0, s>>>(need_off + nel, avail_off + nparticle, max_new, added, err);
  MW_CHECK_LAUNCH();
  if (max_new > 0) {
    k_pc_fill<<<grid_for(max_new, 128), 128, 0, s>>>(box, need_off, offsets, order, avail, added, active, iel, r, t,
                                                     x, z, mat, source, pf, draws, seed, max_new, err);
    MW_CHECK_LAUNCH();
    k_pc_commit<<<grid_for(max_new, 256), 256, 0, s>>>(avail, added, max_new, active);
    MW_CHECK_LAUNCH();
  }
  return MW_OK;
}

}  // extern "C"
