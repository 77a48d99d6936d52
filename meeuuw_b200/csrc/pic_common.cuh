// Particle-in-cell helpers shared by the bit-exact kernels (pic.cu: locate, binning,
// projections) and the FMA-contracted ones (advect.cu: interpolation, advection).
#pragma once

#include "common.cuh"

namespace mw {

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

}  // namespace mw
