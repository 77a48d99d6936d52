// Particle interpolation and advection for the Cartesian box (sm_100a).
//
// Reference: pic_functions.py (interpolate :85-101, velocity at a point :18-37, advect :180-292)
// and the material hooks experiment0.py:230-264 / experiment1.py:91-113.
//
// Unlike pic.cu (locate, binning and element means, which must round exactly as the reference),
// this file is compiled with FMA contraction: the basis and dot-product arithmetic agrees with the
// reference's unfused arithmetic to a few ulp, and the element index of a velocity evaluation comes
// from the reciprocal of the spacing, falling back to the division wherever the quotient is close
// enough to an integer for its truncation to depend on the last bits -- so the element (and the
// reference's wrap of x == Lx into the next row) is the reference's.
#include "pic_common.cuh"

namespace mw {

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
// x / h from the reciprocal ih = 1/h (within a few ulp of the rounded quotient); where that lies
// within 2^-48 (relative) of an integer -- close enough for its truncation to depend on the last
// bits -- the quotient itself, so the truncated value is always the reference's int(x / h).
MW_D double quotient(double x, double h, double ih) {
  const double q = x * ih;
  return fabs(q - rint(q)) <= fabs(q) * 0x1p-48 ? x / h : q;
}

// Velocity at a point: pic_functions.py:18-37.  The element index is the reference's, including
// the case x == Lx that wraps into the next row; indices outside the mesh set a flag.  ihx, ihz:
// the reciprocals of the spacings.
MW_D bool vel_at(const mw_box& b, double ihx, double ihz, int64_t nel, int nnx, double xp, double zp,
                 const double* __restrict__ u, const double* __restrict__ w, double* up, double* wp, int32_t* err) {
  const double qx = quotient(xp, b.hx, ihx), qz = quotient(zp, b.hz, ihz);
  int ex, ez;
  bool ok = qx > -2147483648.0 && qx < 2147483647.0 && qz > -2147483648.0 && qz < 2147483647.0;
  if (ok) {
    ex = (int)qx; ez = (int)qz;
    const int64_t e = (int64_t)b.nelx * ez + ex;
    ok = e >= 0 && e < nel;
    if (ok && (ex < 0 || ex >= b.nelx)) { ex = (int)(e % b.nelx); ez = (int)(e / b.nelx); }   // row wrap
  }
  if (!ok) {
    set_flag(err, MW_FLAG_ELEMENT_RANGE);
    *up = 0.0; *wp = 0.0;
    return false;
  }
  const double rp = ((xp - xv0(b, ex)) * ihx - 0.5) * 2;
  const double tp = ((zp - zv0(b, ez)) * ihz - 0.5) * 2;
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
  const double ihx = 1.0 / b.hx, ihz = 1.0 / b.hz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double su = 0.0, sw = 0.0;
    bool act = active[i] != 0;
    if (act) {
      double xA = x[i], zA = z[i], uA, wA;
      vel_at(b, ihx, ihz, nel, nnx, xA, zA, u, w, &uA, &wA, err);
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
          vel_at(b, ihx, ihz, nel, nnx, xB, zB, u, w, &uB, &wB, err);
          if (rk == 2) {                                              // :244-248
            x[i] = xA + uB * dt; z[i] = zA + wB * dt;
            su = uB; sw = wB;
          } else {
            double xC = xA + uB * dt / 2.0, zC = zA + wB * dt / 2.0;  // :265-266
            if (outside(b, xC, zC)) {
              act = false;
            } else {
              double uC, wC;
              vel_at(b, ihx, ihz, nel, nnx, xC, zC, u, w, &uC, &wC, err);
              double xD = xA + uC * dt, zD = zA + wC * dt;            // :271-272
              if (outside(b, xD, zD)) {
                act = false;
              } else {
                double uD, wD;
                vel_at(b, ihx, ihz, nel, nnx, xD, zD, u, w, &uD, &wD, err);
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

}  // namespace mw

using namespace mw;

static bool box_ok(const mw_box& b) { return b.nelx > 0 && b.nelz > 0 && b.hx > 0 && b.hz > 0; }

extern "C" {

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

}  // extern "C"
