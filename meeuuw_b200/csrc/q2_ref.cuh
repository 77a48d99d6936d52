// Reference-element values of the Q2xQ1 element at the 3x3 Gauss points, shared by the operator
// kernels (stokes.cu, energy.cu): host-computed tables for the constant bank, and the same values
// as compile-time expressions that decide which terms vanish.
#pragma once

#include <cmath>

#include "common.cuh"

namespace mw {

struct RefTables {
  double dr[81], dt[81];   // d N_V / d r, d t at the 9 Gauss points  [q*9+k]
  double NV[81];           // N_V at the Gauss points
  double NP[36];           // N_P at the Gauss points   [q*4+k]
  double wq[9];            // Gauss weights
  double GX[36], GZ[36];   // sum_q w_q dN_V/dr (q, k) N_P(q, j) and the same with dN_V/dt  [k*4+j]
};

// The same reference-element values as compile-time expressions for the operator kernels: inside
// fully unrolled loops they fold into immediates, and the terms whose basis value vanishes at a
// Gauss point (a third of them: the 1D Q2 functions are 0 or 1 at the middle point) disappear.
// Gauss point q = 3 i + j sits at (r, s) = (g_i, g_j), g = (-sqrt(3/5), 0, sqrt(3/5)).
constexpr double GQ = 0.77459666924148337704;      // sqrt(3/5)
MW_HD constexpr double gpt(int i) { return i == 0 ? -GQ : (i == 1 ? 0.0 : GQ); }
MW_HD constexpr double gwt(int i) { return i == 1 ? 8.0 / 9.0 : 5.0 / 9.0; }
// 1D Q2 Lagrange functions on nodes -1, 0, 1 (a = 0, 1, 2) and their derivatives
MW_HD constexpr double lq(int a, double x) { return a == 0 ? 0.5 * x * (x - 1.0) : (a == 1 ? 1.0 - x * x : 0.5 * x * (x + 1.0)); }
MW_HD constexpr double dlq(int a, double x) { return a == 0 ? x - 0.5 : (a == 1 ? -2.0 * x : x + 0.5); }
MW_HD constexpr int kdx(int k) { return (k == 0 || k == 3 || k == 7) ? 0 : ((k == 1 || k == 2 || k == 5) ? 2 : 1); }
MW_HD constexpr int kdz(int k) { return (k == 0 || k == 1 || k == 4) ? 0 : ((k == 2 || k == 3 || k == 6) ? 2 : 1); }
MW_HD constexpr double ref_dr(int q, int k) { return dlq(kdx(k), gpt(q / 3)) * lq(kdz(k), gpt(q % 3)); }
MW_HD constexpr double ref_dt(int q, int k) { return lq(kdx(k), gpt(q / 3)) * dlq(kdz(k), gpt(q % 3)); }
MW_HD constexpr double ref_np(int q, int k) {
  return 0.25 * (k == 0 || k == 3 ? 1.0 - gpt(q / 3) : 1.0 + gpt(q / 3)) *
         (k == 0 || k == 1 ? 1.0 - gpt(q % 3) : 1.0 + gpt(q % 3));
}
MW_HD constexpr double ref_wq(int q) { return gwt(q / 3) * gwt(q % 3); }
// N_V at Gauss point q: the product of the 1D functions (used for which terms vanish)
MW_HD constexpr double ref_nv(int q, int k) { return lq(kdx(k), gpt(q / 3)) * lq(kdz(k), gpt(q % 3)); }

inline void host_ref_tables(RefTables* T) {
  const double qc[3] = {-std::sqrt(3.0 / 5.0), 0.0, std::sqrt(3.0 / 5.0)};
  const double qw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  int q = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j, ++q) {
      double r = qc[i], s = qc[j];
      T->wq[q] = qw[i] * qw[j];
      double N[9];
      q2_basis<double>(r, s, N);
      for (int k = 0; k < 9; ++k) T->NV[q * 9 + k] = N[k];
      double dr[9] = {0.5 * (2.0 * r - 1.0) * 0.5 * s * (s - 1), 0.5 * (2.0 * r + 1.0) * 0.5 * s * (s - 1),
                      0.5 * (2.0 * r + 1.0) * 0.5 * s * (s + 1), 0.5 * (2.0 * r - 1.0) * 0.5 * s * (s + 1),
                      (-2.0 * r) * 0.5 * s * (s - 1), 0.5 * (2.0 * r + 1.0) * (1.0 - s * s),
                      (-2.0 * r) * 0.5 * s * (s + 1), 0.5 * (2.0 * r - 1.0) * (1.0 - s * s), (-2.0 * r) * (1.0 - s * s)};
      double dt[9] = {0.5 * r * (r - 1.0) * 0.5 * (2.0 * s - 1.0), 0.5 * r * (r + 1.0) * 0.5 * (2.0 * s - 1.0),
                      0.5 * r * (r + 1.0) * 0.5 * (2.0 * s + 1.0), 0.5 * r * (r - 1.0) * 0.5 * (2.0 * s + 1.0),
                      (1.0 - r * r) * 0.5 * (2.0 * s - 1.0), 0.5 * r * (r + 1.0) * (-2.0 * s),
                      (1.0 - r * r) * 0.5 * (2.0 * s + 1.0), 0.5 * r * (r - 1.0) * (-2.0 * s), (1.0 - r * r) * (-2.0 * s)};
      for (int k = 0; k < 9; ++k) { T->dr[q * 9 + k] = dr[k]; T->dt[q * 9 + k] = dt[k]; }
      T->NP[q * 4 + 0] = 0.25 * (1 - r) * (1 - s);
      T->NP[q * 4 + 1] = 0.25 * (1 + r) * (1 - s);
      T->NP[q * 4 + 2] = 0.25 * (1 + r) * (1 + s);
      T->NP[q * 4 + 3] = 0.25 * (1 - r) * (1 + s);
    }
  for (int k = 0; k < 9; ++k)              // the pressure-gradient element matrix on the reference element
    for (int j = 0; j < 4; ++j) {
      double gx = 0.0, gz = 0.0;
      for (int q2 = 0; q2 < 9; ++q2) {
        gx += T->wq[q2] * T->dr[q2 * 9 + k] * T->NP[q2 * 4 + j];
        gz += T->wq[q2] * T->dt[q2 * 9 + k] * T->NP[q2 * 4 + j];
      }
      T->GX[k * 4 + j] = gx;
      T->GZ[k * 4 + j] = gz;
    }
}

}  // namespace mw
