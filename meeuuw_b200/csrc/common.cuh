// Shared definitions for the meeuuw_b200 sm_100a kernels.
//
// Mesh convention: the reference's uniform Cartesian box (build_velocity_mesh.py:113-145,
// build_velocity_connectivity.py:63-92, build_pressure_connectivity.py).  Q2 velocity/temperature
// nodes form a (2*nelx+1) x (2*nelz+1) lattice numbered x-fastest; element e = nelx*ez + ex;
// its 9 nodes in the reference's local order 3--6--2 / 7 8 5 / 0--4--1 are computed from (ex, ez)
// instead of being read from icon_V, and its 4 Q1 pressure nodes likewise from (ex, ez).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "../../include/meeuuw_b200.h"

#define MW_HD __host__ __device__ __forceinline__
#define MW_D __device__ __forceinline__

namespace mw {

// local node k of a Q2 element -> (dx, dz) offset on the Q2 node lattice
MW_HD int q2_dx(int k) { return (k == 0 || k == 3 || k == 7) ? 0 : ((k == 1 || k == 2 || k == 5) ? 2 : 1); }
MW_HD int q2_dz(int k) { return (k == 0 || k == 1 || k == 4) ? 0 : ((k == 2 || k == 3 || k == 6) ? 2 : 1); }
// local node k of a Q1 element -> (dx, dz) in {0,1}
MW_HD int q1_dx(int k) { return (k == 1 || k == 2) ? 1 : 0; }
MW_HD int q1_dz(int k) { return (k == 2 || k == 3) ? 1 : 0; }

MW_HD int64_t q2_node(int ex, int ez, int k, int nnx) {
  return (int64_t)(2 * ez + q2_dz(k)) * nnx + (2 * ex + q2_dx(k));
}
MW_HD int64_t q1_node(int ex, int ez, int k, int nelx) {
  return (int64_t)(ez + q1_dz(k)) * (nelx + 1) + (ex + q1_dx(k));
}

// Q2 basis in the reference's operation order (basis_functions.py:20-30).  Files that need the
// reference's exact rounding are compiled with -fmad=false so no product/sum pair is fused.
template <typename R>
MW_HD void q2_basis(R r, R s, R* N) {
  N[0] = R(0.5) * r * (r - R(1.0)) * R(0.5) * s * (s - R(1.0));
  N[1] = R(0.5) * r * (r + R(1.0)) * R(0.5) * s * (s - R(1.0));
  N[2] = R(0.5) * r * (r + R(1.0)) * R(0.5) * s * (s + R(1.0));
  N[3] = R(0.5) * r * (r - R(1.0)) * R(0.5) * s * (s + R(1.0));
  N[4] = (R(1.0) - r * r) * R(0.5) * s * (s - R(1.0));
  N[5] = R(0.5) * r * (r + R(1.0)) * (R(1.0) - s * s);
  N[6] = (R(1.0) - r * r) * R(0.5) * s * (s + R(1.0));
  N[7] = R(0.5) * r * (r - R(1.0)) * (R(1.0) - s * s);
  N[8] = (R(1.0) - r * r) * (R(1.0) - s * s);
}

MW_D void set_flag(int32_t* err, int32_t bit) {
  if (err) atomicOr(err, bit);
}

// Grid size: enough CTAs to cover n work items, capped at a multiple of the SM count.
int grid_for(int64_t n, int threads, int waves = 8);
int num_sms();

// Programmatic dependent launch.  The solver loops are long chains of short kernels on one stream;
// launched through pdl_launch(), a kernel's CTAs are scheduled while its predecessor is still
// running, so the launch latency between the two is hidden.  Every kernel started this way runs
// pdl_entry() before touching global memory: it waits until every prerequisite grid has completed
// and its writes are visible, then allows the next kernel to be scheduled (for a kernel started the
// ordinary way both instructions return at once).  Because each kernel waits for the complete
// predecessor before its first access, the stream order of all reads and writes is unchanged, and
// at most one waiting grid is resident beside the running one.
MW_D void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

bool pdl_enabled();        // false when the environment sets MW_PDL=0

template <typename... KArgs, typename... Args>
inline void pdl_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = (s != nullptr && pdl_enabled()) ? 1 : 0;     // not on the legacy default stream
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace mw

#define MW_CHECK_LAUNCH()                              \
  do {                                                 \
    cudaError_t e__ = cudaGetLastError();              \
    if (e__ != cudaSuccess) return MW_ERR_CUDA;        \
  } while (0)
