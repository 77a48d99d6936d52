/* meeuuw_b200 -- C ABI of the B200 (sm_100a) implementation of meeuuw's per-timestep hot path.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t passed as void*,
 * launches stream-ordered work and returns an int status (MW_OK = 0).  Nothing allocates device
 * memory: callers pass outputs and, where a routine needs scratch, a workspace whose size a
 * *_workspace_bytes() query returns.  Problems a kernel detects (a particle outside [-1,1], an
 * element without particles, ...) are OR-ed into an optional device int32 flag word `err`
 * (MW_FLAG_*), which the caller reads when it needs the reference's exit semantics.
 *
 * Mesh: the reference's uniform Cartesian box (build_velocity_mesh.py:113-145,
 * build_velocity_connectivity.py:63-92, build_pressure_connectivity.py).  Connectivity (icon_V,
 * icon_P, local_to_globalV) is implied by mw_box and computed in the kernels.
 *
 * Each declaration names the reference function it replaces (file:line in cedrict/meeuuw).
 */
#ifndef MEEUUW_B200_H
#define MEEUUW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (return values) ---- */
#define MW_OK 0
#define MW_ERR_BAD_ARG 1
#define MW_ERR_CUDA 2
#define MW_ERR_NOT_CONVERGED 3
#define MW_ERR_WORKSPACE 4
#define MW_ERR_DEVICE_FLAG 5
#define MW_ERR_TOO_LARGE 6   /* the problem exceeds a fixed-capacity entry point's static scratch */

/* ---- device flag bits (err word) ---- */
#define MW_FLAG_R_OUT_OF_BOUNDS 1   /* locate_particles.py:61-62 "r value out of bounds" */
#define MW_FLAG_T_OUT_OF_BOUNDS 2   /* locate_particles.py:63-64 "t value out of bounds" */
#define MW_FLAG_ELEMENT_RANGE 4     /* a point maps to an element index outside the mesh */
#define MW_FLAG_EMPTY_ELEMENT 8     /* meeuuw.py:1198-1199 "an element contains no particle" */
#define MW_FLAG_NONFINITE 16        /* NaN/Inf met in a solver reduction */
#define MW_FLAG_ITER_LIMIT 32       /* a bounded device loop gave up */
#define MW_FLAG_POP_UNAVAILABLE 64  /* pic_functions.py:1722-1733 "population_control: not available yet" */
#define MW_FLAG_POP_MASK_EMPTY 128  /* pic_functions.py:1747-1748 "population_control: mask empty" */
#define MW_FLAG_POP_DRAWS 256       /* population control needs more uniform numbers than were passed */

#define MW_MAX_FIELDS 8

#define MW_AVG_ARITHMETIC 0
#define MW_AVG_GEOMETRIC 1
#define MW_AVG_HARMONIC 2

#define MW_SPACE_Q2 0        /* N_V on the 9 Q2 nodes (icon_V)          */
#define MW_SPACE_Q1_ON_V 1   /* N_P on the 4 corner V nodes (icon_V[0:4]) */
#define MW_SPACE_Q1 2        /* N_P on the 4 pressure nodes (icon_P)       */

#define MW_MATERIAL_BOUSSINESQ 0 /* experiment0.py:254-264: rho0(1-alpha T), eta=exp(-gamma T) or eta0 */
#define MW_MATERIAL_TWO 1        /* experiment1.py:104-111: rho, eta by particle material id          */

typedef struct {
  int32_t nelx, nelz;
  double Lx, Lz, hx, hz; /* hx = Lx/nelx, hz = Lz/nelz as build_velocity_mesh.py:19-20 */
} mw_box;

typedef struct {
  int32_t kind;
  double rho0, alphaT, fk_gamma, eta0, hcond, hcapa, hprod;
  double mat_rho[8], mat_eta[8];
} mw_material;

typedef struct { /* nodal (nn_V) fields interpolated onto particles; NULL entries are skipped */
  const double *exx, *ezz, *exz, *q, *T;
} mw_nodal5;

typedef struct { /* per-particle outputs; NULL entries are not written (rho, eta required) */
  double *exx, *ezz, *exz, *p, *T, *rho, *eta, *hcond, *hcapa, *hprod, *alpha;
} mw_swarm_props;

/* ======================= particle-in-cell (pic_functions.py) ======================= */

/* locate_particles___box, pic_functions.py:108-137 (+ bounds check locate_particles.py:61-64).
 * Inactive particles get r=t=0, iel=0. */
int mw_locate_box(mw_box box, int64_t nparticle, const uint8_t* active, const double* x, const double* z,
                  double* r, double* t, int32_t* iel, int32_t* err, void* stream);

/* interpolate_field_on_particles, pic_functions.py:85-101, for nfield (<= MW_MAX_FIELDS) nodal
 * fields at once; `fields` and `out` are HOST arrays of device pointers. */
int mw_interp_q2(mw_box box, int64_t nparticle, const uint8_t* active, const double* r, const double* t,
                 const int32_t* iel, int32_t nfield, const double* const* fields, double* const* out,
                 void* stream);

/* The five interpolations of meeuuw.py:1118-1125 fused with material_model (meeuuw.py:1154;
 * experiment0.py:230-264 and experiment1.py:91-113).  `mat` is the int8 material id (may be NULL
 * for MW_MATERIAL_BOUSSINESQ). */
int mw_interp_material(mw_box box, int64_t nparticle, const uint8_t* active, const double* r, const double* t,
                       const int32_t* iel, const int8_t* mat, mw_nodal5 nodal, mw_material m,
                       mw_swarm_props out, void* stream);

/* advect_particles___box, pic_functions.py:180-292 (RK 1, 2, 4).  x, z, active are updated in
 * place; up/wp receive the particle velocities (may be NULL).  If dt_dev is not NULL the time step
 * is read from that device scalar instead of `dt`. */
int mw_advect_box(mw_box box, int32_t rk, double dt, const double* dt_dev, int64_t nparticle, double* x, double* z,
                  uint8_t* active, const double* u, const double* w, double* up, double* wp, int32_t* err,
                  void* stream);

/* Counting sort of the active particles by element (no reference counterpart: it is the data
 * structure behind the atomic-free projections below).  counts[nel], offsets[nel+1],
 * order[nparticle]; bins are sorted by particle index. */
size_t mw_bin_workspace_bytes(int32_t nel);
int mw_bin_particles(int32_t nel, int64_t nparticle, const uint8_t* active, const int32_t* iel, int32_t* counts,
                     int32_t* offsets, int32_t* order, void* work, size_t work_bytes, int32_t* err, void* stream);

/* project_particles_on_elements, pic_functions.py:603-650 (nparticle_per_element = counts from
 * mw_bin_particles).  Empty elements set MW_FLAG_EMPTY_ELEMENT. */
int mw_project_elements(int32_t nel, const int32_t* offsets, const int32_t* order, const double* rho,
                        const double* eta, int32_t averaging, double* rho_e, double* eta_e, int32_t* err,
                        void* stream);

/* project_particle_field_on_nodes_{1,2,3,4}, pic_functions.py:659-1053, for nfield fields at once
 * (each with its own averaging); `averaging`, `phi`, `phi_nodal` are HOST arrays.  With a
 * workspace of mw_project_nodes_workspace_bytes() the sums go through per-element partials (fast);
 * with work == NULL each node merges its elements' particles in particle-index order (the
 * reference's exact summation order, slower). */
size_t mw_project_nodes_workspace_bytes(mw_box box, int32_t nfield);
int mw_project_nodes(mw_box box, int32_t flavour, int32_t nfield, const int32_t* averaging, const int32_t* offsets,
                     const int32_t* order, const double* r, const double* t, const double* const* phi,
                     double* const* phi_nodal, void* work, size_t work_bytes, void* stream);

/* project_nodal_{V,P,T}field_onto_qpoints, project_nodal_field_onto_qpoints.py:12-62.
 * N is the device (9 x m) basis table (N_V for MW_SPACE_Q2, N_P otherwise); phiq is (nel, 9). */
int mw_nodal_to_qpoints(mw_box box, int32_t space, const double* N, const double* phi, double* phiq, void* stream);

/* ======================= least-squares projections, population control ======================= */

/* compute_ls_coefficients_P1 (ncoef 3: a + b dx + c dz) and compute_ls_coefficients_Q1 (ncoef 4:
 * + d dx dz), pic_functions.py:1098-1285, for up to MW_MAX_FIELDS particle fields at once, with
 * dx, dz measured from the element centre (node 8).  offsets/order must bin EVERY particle
 * (mw_bin_particles with an all-ones active array): the reference's mask swarm_iel == iel takes
 * inactive particles, which locate leaves at iel 0, into element 0's fit.  Per element the normal
 * equations are summed particle by particle in index order, each sum as the reference forms it,
 * and solved by Gaussian elimination with partial pivoting (the reference calls LAPACK's solve).
 * coef[f]: (nel, ncoef) row-major; fmin[f], fmax[f] (may be NULL): the particle extrema per element
 * (pic_functions.py:1164-1167).  limit_h > 0 (P1 only) limits the slopes as the driver does:
 * limiter(), pic_functions.py:1068-1089, called with h = hx at meeuuw.py:1241-1248.  Elements
 * without particles set MW_FLAG_EMPTY_ELEMENT (the driver aborts before, meeuuw.py:1198). */
typedef struct {
  const double* phi[MW_MAX_FIELDS];
  double* coef[MW_MAX_FIELDS];
  double* fmin[MW_MAX_FIELDS];
  double* fmax[MW_MAX_FIELDS];
  int32_t n;
} mw_ls_fields;
int mw_ls_fit(mw_box box, int32_t ncoef, const int32_t* offsets, const int32_t* order, const double* x,
              const double* z, mw_ls_fields fields, double limit_h, int32_t* err, void* stream);

/* The fits at the quadrature points, meeuuw.py:1517-1532 (particle_rho/eta_projection
 * "least_squares_P1/Q1"): phiq[e, q] = a + b (xq - x_e) + c (zq - z_e) [+ d (xq - x_e)(zq - z_e)].
 * coef (nel, ncoef); xq, zq, phiq (nel, 9). */
int mw_ls_to_qpoints(mw_box box, int32_t ncoef, const double* coef, const double* xq, const double* zq,
                     double* phiq, void* stream);

/* population_control, pic_functions.py:1621-1812, on the box path's particle arrays (an int8
 * material id in place of the weight fractions).  Called where the driver calls it
 * (meeuuw.py:2846-2850): after advection, before locate.  counts, offsets and order are the step's
 * binning (mw_bin_particles over the step-start active flags and element indices); active, x, z are
 * the values after advection.  Each element with fewer than nparticle_min particles receives
 * inactive particles, taken in index order, at reduced coordinates r, t = -0.95 + 1.9 u (the
 * reference's random.uniform(-0.95, 0.95), r first); each takes the material id of the nearest
 * particle of its element (the first in index order on a tie, as np.argmin; that particle's index
 * goes to source[pid], if source is not NULL, so a caller can copy other per-particle data such as
 * weight fractions) and, for every field in `avg`, the mean of the element's particles
 * (np.average: numpy's pairwise summation order; eta, u, w on the box path, strain or melt
 * fraction where a caller carries them).  draws: 2 * max_new uniform [0, 1) numbers, two per added
 * particle in the order the reference consumes them; or NULL: the numbers come from a
 * counter-based generator keyed by `seed`.  The number of particles added is written to *added
 * (device int32).  Errors set device flags (no particle is added): MW_FLAG_POP_UNAVAILABLE when more
 * particles are needed than are inactive, MW_FLAG_POP_DRAWS when more than max_new are needed;
 * MW_FLAG_POP_MASK_EMPTY marks a flagged element without active particles.  mat and source may be
 * NULL. */
typedef struct { double* f[MW_MAX_FIELDS]; int32_t n; } mw_pc_fields;
size_t mw_population_workspace_bytes(int32_t nel, int64_t nparticle);
int mw_population_control(mw_box box, int32_t nparticle_min, int64_t nparticle, const int32_t* counts,
                          const int32_t* offsets, const int32_t* order, uint8_t* active, int32_t* iel, double* r,
                          double* t, double* x, double* z, int8_t* mat, int32_t* source, mw_pc_fields avg,
                          const double* draws, int64_t max_new, uint64_t seed, int32_t* added, void* work,
                          size_t work_bytes, int32_t* err, void* stream);

/* ======================= element assembly ======================= */

#define MW_F64 0
#define MW_F32 1

typedef struct { /* inputs of build_matrix_stokes (build_matrix_stokes.py:18-64), device pointers */
  const double *rhoq, *etaq, *JxWq, *jcbi00q, *jcbi01q, *jcbi10q, *jcbi11q, *gxq, *gzq; /* (nel, 9) */
  const double* eta_e;                                                             /* (nel)    */
  const double *N_V, *N_P, *dNdr_V, *dNdt_V, *dNdr_P, *dNdt_P; /* (9,9) / (9,4) basis tables     */
  const uint8_t* bc_fix_V;                                     /* (Nfem_V)                       */
  const double* bc_val_V;                                      /* (Nfem_V)                       */
  double eta_ref, L_ref;
} mw_stokes_in;

typedef struct { /* outputs; VV arrays are float or double per `precision`; rhs always double */
  void *VV_Stokes, *VV_K, *VV_G, *VV_GT, *VV_M, *VV_M_eta, *VV_H;
  double *rhs_f, *rhs_h;
} mw_stokes_out;

/* build_matrix_stokes, build_matrix_stokes.py:18-278 (box, plane strain).  blocks=0 writes the
 * full layout VV_Stokes (nel*468, :267-276), blocks=1 the K/G/GT/M/M_eta/H blocks (:235-265).
 * Matches the COO index arrays II/JJ of meeuuw.py:884-1017.  With all VV pointers NULL only
 * rhs_f and rhs_h are produced (the matrix-free solver needs no stored matrix). */
size_t mw_assemble_stokes_workspace_bytes(mw_box box);
int mw_assemble_stokes(mw_box box, int32_t blocks, int32_t precision, mw_stokes_in in, mw_stokes_out out, void* work,
                       size_t work_bytes, void* stream);

/* rhs_f, rhs_h of build_matrix_stokes (build_matrix_stokes.py:141-143, :206-229) for the case
 * where every Dirichlet value bc_val_V is zero: body force only, fixed rows 0, rhs_h = 0.
 * Workspace: mw_assemble_stokes_workspace_bytes(box). */
int mw_stokes_rhs_body(mw_box box, const double* rhoq, const double* gxq, const double* gzq, const double* JxWq,
                       const double* N_V, const uint8_t* bc_fix_V, double* rhs_f, double* rhs_h, void* work,
                       size_t work_bytes, void* stream);

typedef struct { /* inputs of build_matrix_energy (build_matrix_energy.py:12-47) */
  const double* T; /* (nn_V) previous-step temperature, T_mem */
  const double *rhoq, *etaq, *Tq, *uq, *wq, *hcondq, *hcapaq, *alphaq, *hprodq, *exxq, *ezzq, *exzq, *JxWq;
  const double *jcbi00q, *jcbi01q, *jcbi10q, *jcbi11q;
  const double *N_T, *dNdr_T, *dNds_T;
  const uint8_t* bc_fix_T;
  const double* bc_val_T;
  double dt, rho0;
  const double* dt_dev; /* if not NULL, dt is read from this device scalar */
  int32_t formulation;  /* 0 = "BA", 1 = "EBA" */
} mw_energy_in;

/* build_matrix_energy, build_matrix_energy.py:12-141: VV_T (nel*81, float or double) and rhs. */
size_t mw_assemble_energy_workspace_bytes(mw_box box);
int mw_assemble_energy(mw_box box, int32_t precision, mw_energy_in in, void* VV_T, double* rhs, void* work,
                       size_t work_bytes, void* stream);

/* ======================= FP64 derived fields and reductions ======================= */

#define MW_PNORM_NONE 0
#define MW_PNORM_SURFACE 1
#define MW_PNORM_VOLUME 2

typedef struct { double c[3], w[3]; } mw_gauss3; /* qcoords, qweights (quadrature_setup.py:13-15) */

typedef struct {
  double CFLnb, hx, hz, dt_max;
  int32_t solve_T;
} mw_dt_params;

/* Scratch for the reductions below (partial sums). */
size_t mw_post_workspace_bytes(void);

/* compute_pressure_offset, compute_pressure_offset.py:12-66 (Cartesian): writes the device scalar
 * *offset.  "surface" sums the top edge sequentially in element order as the reference does. */
int mw_pressure_offset(mw_box box, int32_t normalisation, const double* p, const double* N_P, const double* JxWq,
                       double volume, double* offset, void* work, size_t work_bytes, void* stream);

/* p -= offset (meeuuw.py:1977) and compute_nodal_pressure (compute_nodal_pressure.py:8-21):
 * q on V nodes.  offset may be NULL; q may be NULL (only the subtraction is done). */
int mw_nodal_pressure(mw_box box, double* p, const double* offset, int32_t subtract_in_place, const double* N_P_n,
                      double* q, void* stream);

/* compute_nodal_strain_rate, compute_strain_rate.py:51-73.  The jcbi*n (nel, 9) arrays may be NULL
 * for the uniform box (inverse Jacobian diag(2/hx, 2/hz)). */
int mw_nodal_strain_rate(mw_box box, const double* u, const double* w, const double* dNdr_V_n,
                         const double* dNdt_V_n, const double* jcbi00n, const double* jcbi01n, const double* jcbi10n,
                         const double* jcbi11n, double* exx_n, double* ezz_n, double* exz_n, void* stream);

/* compute_nodal_heat_flux, compute_nodal_heat_flux.py:12-40 -> dTdx_n, dTdz_n, qx_n, qz_n. */
int mw_nodal_heat_flux(mw_box box, const double* T, const double* hcond_n, const double* dNdr_T_n,
                       const double* dNdt_T_n, const double* jcbi00, const double* jcbi01, const double* jcbi10,
                       const double* jcbi11, double* dTdx_n, double* dTdz_n, double* qx_n, double* qz_n,
                       void* stream);

/* compute_Nu, postprocessors.py:114-248: out13 = the reference's 13-tuple, Nu last. */
size_t mw_nu_workspace_bytes(mw_box box);
int mw_compute_nu(mw_box box, const double* T, const double* dTdx_n, const double* dTdz_n, const double* hcond_n,
                  mw_gauss3 g, double* out13, void* work, size_t work_bytes, void* stream);

/* Nusselt number without any allocation.  No counterpart in the reference: it exists for callers
 * that hold the temperature and heat-flux arrays on the device but cannot allocate device memory
 * themselves -- for example a diagnostics or monitoring hook that a host code hands read-only
 * device pointers to, with no allocator of its own, and that must not change the memory state of
 * the running simulation (mw_compute_nu needs a caller-allocated workspace).  Its scratch is a
 * fixed file-scope device array sized for at most MW_NU_NOALLOC_MAX_BOUNDARY_ELEMENTS boundary
 * elements, 2*(nelx+nelz) (2.25 MiB, held by every GPU that loads the library until exit);
 * larger meshes return MW_ERR_TOO_LARGE.  The call makes no cudaMalloc/cudaFree and calls no
 * allocating routine.  The first call in a CUDA context does the set-up: it looks up the array's
 * device address (cudaGetSymbolAddress) and, under CUDA's lazy module loading, that lookup loads
 * the library's post-processing module together with the 2.25 MiB array -- so device free memory
 * drops once, at that first call, unless another post-processing entry point ran first.  Make the
 * first call before the simulation's memory state must stay fixed and before any stream capture.
 * The address is cached per context (by its unique id), so a cudaDeviceReset or a different
 * context repeats the set-up.  All calls share the one array and each call writes every slot it
 * reads, so nothing needs clearing between calls; calls that overlap on the GPU (different
 * streams, same device) race and must be serialised by the caller.  Output: the same 13 values as
 * mw_compute_nu. */
#define MW_NU_NOALLOC_MAX_BOUNDARY_ELEMENTS 32768
int mw_compute_nu_noalloc(mw_box box, const double* T, const double* dTdx_n, const double* dTdz_n,
                          const double* hcond_n, mw_gauss3 g, double* out13, void* stream);

/* compute_global_quantities, postprocessors.py:14-83 (the vrms, Tavrg and mass sums):
 * out3 = {vrms, Tavrg, TM}.  Tq, rhoq may be NULL. */
int mw_global_quantities(int64_t nq, const double* uq, const double* wq, const double* Tq, const double* rhoq,
                         const double* JxWq, double volume, double* out3, void* work, size_t work_bytes,
                         void* stream);
/* The whole compute_global_quantities tuple (postprocessors.py:14-83): out9 = {vrms, EK, WAG,
 * TVD, GPE (= 0), ITE, TM, Tavrg, eta_avrg}; eta_avrg is NaN when sum(eII JxW) = 0, where the
 * reference leaves it unassigned.  All arrays (nq = nel*9 qpoint values) are required. */
int mw_global_quantities_full(int64_t nq, const double* uq, const double* wq, const double* Tq, const double* rhoq,
                              const double* hcapaq, const double* etaq, const double* exxq, const double* ezzq,
                              const double* exzq, const double* gxq, const double* gzq, const double* JxWq,
                              double volume, double* out9, void* work, size_t work_bytes, void* stream);

/* Time step, meeuuw.py:2112-2139: state2 = {dt1_mem, dt2_mem} (device, updated),
 * out3 = {dt, dt1, dt2} (device). */
int mw_compute_dt(int64_t nn_V, const double* u, const double* w, int64_t nparticle, const double* swarm_hcond,
                  const double* swarm_hcapa, const double* swarm_rho, mw_dt_params prm, double* state2,
                  double* out3, void* work, size_t work_bytes, void* stream);

/* ======================= matrix-free Stokes operator and solver ======================= */

#define MW_SCHEME_CD_U_ETA 0 /* cd_u_eta.py:13-99: Schur PCG preconditioned by M_eta (Q1 mass / eta_e) */
#define MW_SCHEME_UZAWA3 1   /* uzawa3_solver_L2.py:21-99: Schur PCG preconditioned by M             */

typedef struct mw_stokes mw_stokes; /* opaque host-side handle; device memory is the caller's workspace */

typedef struct {
  double eta_ref, L_ref;  /* G scaling eta_ref/L_ref, build_matrix_stokes.py:157                    */
  int32_t precisions;     /* bit 0: FP64 multigrid hierarchy, bit 1: FP32 hierarchy                */
  int32_t coarse_min;     /* coarsen while both element counts stay >= coarse_min                   */
  int32_t dense_max;      /* coarsest level solved with a dense inverse when its dofs <= dense_max   */
  int32_t cheb_degree;    /* Chebyshev-Jacobi smoothing steps per pre/post sweep                     */
  double cheb_ratio;      /* smoothing interval [lambda_max/ratio, lambda_max]                       */
  double cheb_safety;     /* lambda_max estimate multiplier                                          */
  int32_t power_iters;    /* power iterations for lambda_max(D^-1 K) per level (first viscosity)    */
  int32_t power_iters_warm; /* power iterations on later viscosities, warm-started                   */
  int32_t tail_nel;       /* levels with at most this many elements run each V-cycle as one launch of
                             one cluster (0: a launch per smoothing step, residual and transfer)    */
  int32_t cheb_degree_coarse; /* Chebyshev steps per sweep below the finest level (0: cheb_degree)   */
  int32_t coarsen_odd;    /* 1: an odd element count coarsens to ceil(n/2) elements over the same box
                             (a grid not nested in the fine one, Q2 interpolation as the transfer);
                             0: coarsening stops at the first odd count                           */
  int32_t coarse_dense_max; /* keep coarsening below coarse_min (down to 2 elements a side) while the
                             coarsest level has more unknowns than this (0: off); 168 fits the
                             one-CTA shared-memory inverse                                          */
} mw_stokes_params;

typedef struct {
  int32_t scheme;         /* MW_SCHEME_*                                                             */
  int32_t precision;      /* MW_F64: plain FP64; MW_F32: FP32 inner PCG + FP64 iterative refinement  */
  double tol;             /* FP64 relative true residual ||b - A x|| / ||b|| target (e.g. 1e-8)      */
  int32_t max_outer;      /* Schur-PCG iterations per run (the reference caps at 100)                */
  int32_t max_inner;      /* multigrid-PCG iterations per K solve                                    */
  double inner_rtol;      /* relative tolerance of each K solve                                      */
  int32_t max_refine;     /* refinement sweeps (MW_F32)                                              */
  double sweep_reduction; /* Schur residual reduction per refinement sweep (MW_F32)                  */
  int32_t mass_iters;     /* Chebyshev-Jacobi steps per M / M_eta solve (error 2^(1-iters))          */
  int32_t use_guess;      /* 1: start from the solV/solP passed in (warm start)                      */
  double* history;        /* optional device [4][history_len]: per Schur iteration xiV = ||alpha d||, */
  int32_t history_len;    /* xiP = ||alpha p||, alpha, beta (the reference's array_xiV/xiP/alpha/beta) */
  int32_t host_loops;     /* 0: loops as CUDA-graph conditional nodes (one graph launch per solve, the  */
                          /* default); 1: loops driven by the host (one synchronisation per iteration) */
  double sweep_target;    /* MW_F32: > 0 stops each refinement sweep's Schur iteration at the reduction */
                          /* max(sweep_reduction, sweep_target * tol / current relative residual), so a */
                          /* sweep that starts near tol does only what reaching sweep_target * tol    */
                          /* needs; 0: every sweep reduces by sweep_reduction                          */
} mw_solve_params;

typedef struct {
  int32_t outer_iters, inner_iters, refinements, converged;
  double rel_residual, initial_rel_residual;
} mw_solve_info;

void mw_stokes_default_params(mw_stokes_params* p);
void mw_solve_default_params(mw_solve_params* p);

/* Device workspace the solver needs for this mesh and parameter set. */
size_t mw_stokes_workspace_bytes(mw_box box, mw_stokes_params prm);

/* Create a solver for the box with the velocity Dirichlet mask bc_fix_V (device, Nfem_V bytes,
 * kept by reference).  All device arrays are carved from `work`. */
int mw_stokes_create(mw_box box, mw_stokes_params prm, const uint8_t* bc_fix_V, void* work, size_t work_bytes,
                     mw_stokes** out);
int mw_stokes_destroy(mw_stokes* S);
int mw_stokes_levels(const mw_stokes* S, int32_t precision);

/* New viscosity (etaq (nel,9), eta_e (nel) or NULL): the data build_matrix_stokes.py reads. */
int mw_stokes_set_viscosity(mw_stokes* S, const double* etaq, const double* eta_e, void* stream);

/* Matrix-free y = [K G; G^T 0] (u, p) with the Dirichlet elimination of
 * build_matrix_stokes.py:206-217 -- equal to SpMV with the assembled COO (meeuuw.py:1798).
 * u or p may be NULL (treated as zero); yV or yP may be NULL (not computed). */
int mw_stokes_apply(mw_stokes* S, const double* u, const double* p, double* yV, double* yP, void* stream);
int mw_stokes_apply_f32(mw_stokes* S, const float* u, const float* p, float* yV, float* yP, void* stream);
/* The G and G^T blocks alone (build_matrix_stokes.py:130-157, Dirichlet rows of G zero and fixed
 * entries of u ignored, as the eliminated COO): yV = G p, yP = G^T u, as node stencils of the
 * uniform box's element matrix (what the Schur-complement iterations apply). */
int mw_stokes_grad(mw_stokes* S, const double* p, double* yV, void* stream);
/* One Chebyshev smoothing step of the FP32 multigrid's finest level (the kernel the V-cycle
 * launches most): d = c1 d + c2 D^-1 (b - K x), xo = x + d with the level's coefficient pair
 * `step` (0: the restart step, d not read).  For measurement and tests. */
int mw_stokes_cheb_step_f32(mw_stokes* S, const float* b, const float* x, float* xo, float* d, int32_t step,
                            void* stream);
int mw_stokes_div(mw_stokes* S, const double* u, double* yP, void* stream);

/* One multigrid V-cycle for K (the inner preconditioner); b, x in the given precision. */
int mw_stokes_vcycle(mw_stokes* S, int32_t precision, const void* b, void* x, void* stream);
/* Grid transfer between multigrid levels `level` (fine) and level + 1 (coarse) of the current
 * hierarchy: restrict_dir = 1: out (coarse) = P^T in (fine), fixed coarse dofs zero; 0: out (fine)
 * += P in (coarse) on the free fine dofs.  Element counts of a level: mw_stokes_level_shape. */
int mw_stokes_transfer(mw_stokes* S, int32_t precision, int32_t level, int32_t restrict_dir, const void* in,
                       void* out, void* stream);
int mw_stokes_level_shape(const mw_stokes* S, int32_t precision, int32_t level, int32_t* nx, int32_t* nz);

/* K x = b by multigrid-preconditioned CG (replaces splu(K).solve, uzawa3_solver_L2.py:37-38). */
int mw_stokes_solve_K(mw_stokes* S, int32_t precision, const double* b, double* x, double rtol, int32_t maxit,
                      int32_t* iters, double* relres, void* stream);

/* Result of the last solve from its device scalars (synchronises `stream`).  When mw_stokes_solve is
 * called on a stream that is recording a CUDA graph, the solve is recorded into that graph (its
 * loops as conditional nodes), returns MW_OK with a zeroed info, and this call reads the outcome
 * after a replay; converged = rel_residual <= tol. */
int mw_stokes_device_info(mw_stokes* S, double tol, mw_solve_info* info, void* stream);

/* 1 when this solver has run a solve as one recorded CUDA graph with device-side loops (the
 * default), 0 when it fell back to host-driven loops. */
int mw_stokes_device_loops(const mw_stokes* S);

/* Uzawa residual of a pressure candidate (no reference counterpart: it judges initial guesses for
 * uzawa3_solver_L2 / cd_u_eta, which recompute the velocity from the pressure): V = K^-1 (f - G P)
 * by the multigrid PCG at `precision` to rtol (V may be NULL: internal scratch), then
 * *norm_out = || G^T V - h ||_2 with the mean removed (closed box).  Synchronises. */
int mw_stokes_uzawa_residual(mw_stokes* S, int32_t precision, const double* f, const double* h, const double* P,
                             double rtol, int32_t maxit, double* V, double* norm_out, void* stream);

/* FP64 residual (RV, RP) = (f, h) - A (V, P) and its 2-norm. */
int mw_stokes_residual(mw_stokes* S, const double* V, const double* P, const double* f, const double* h, double* RV,
                       double* RP, double* norm_out, void* stream);

/* uzawa3_solver_L2 (uzawa3_solver_L2.py:21-99) / cd_u_eta (cd_u_eta.py:13-99) on the device: the
 * Schur-complement PCG with K^-1 by multigrid PCG, stopped on the FP64 relative true residual.
 * solV (Nfem_V, interleaved u,w) and solP (Nfem_P) receive the solution (solP is the unscaled
 * Stokes pressure: the caller multiplies by eta_ref/L_ref as meeuuw.py:1848 does). */
int mw_stokes_solve(mw_stokes* S, const double* f, const double* h, double* solV, double* solP, mw_solve_params sp,
                    mw_solve_info* info, void* stream);

/* Ensembles: the Stokes solves of many models in one launch, one thread-block cluster per model
 * running that model's whole mixed-precision solve (MW_F32: FP64 refinement, Schur-complement CG,
 * FP32 multigrid-PCG inner solves) with its own hierarchy, iteration counts and convergence tests.
 * mw_stokes_ensemble_create binds n solvers (each created with the FP32 hierarchy) to their
 * right-hand sides f, h and solutions V, P (device arrays that stay in place; V 16-byte aligned);
 * before each ensemble solve, every model's viscosity is set (mw_stokes_set_viscosity) and its
 * hierarchy prepared (mw_stokes_prepare, on a stream ordered before the solve).  The solve takes
 * precision MW_F32 and no history (MW_ERR_BAD_ARG otherwise, and while any model's viscosity was set
 * after its last mw_stokes_prepare); each model's outcome is read with mw_stokes_device_info.
 * Replaces, for an ensemble, the per-model mw_stokes_solve calls (one per model and step). */
typedef struct mw_stokes_ensemble mw_stokes_ensemble;
int mw_stokes_prepare(mw_stokes* S, int32_t precision, void* stream);
int mw_stokes_ensemble_create(mw_stokes* const* S, const double* const* f, const double* const* h,
                              double* const* V, double* const* P, int32_t n, mw_stokes_ensemble** out);
int mw_stokes_ensemble_solve(mw_stokes_ensemble* E, mw_solve_params sp, void* stream);
int mw_stokes_ensemble_destroy(mw_stokes_ensemble* E);

/* u, w from the interleaved solution and p = solP * scale (meeuuw.py:1846-1851). */
int mw_split_solution(int64_t nn_V, int64_t nn_P, const double* solV, const double* solP, double scale, double* u,
                      double* w, double* p, void* stream);

/* "elemental" qpoint fields (meeuuw.py:1512-1514, :1545-1547): aq[e, :] = a[e] (b, bq optional). */
int mw_elemental_to_qpoints(int64_t nel, const double* a, const double* b, double* aq, double* bq, void* stream);

/* ======================= sparse patterns ======================= */

/* The reference's COO index arrays (meeuuw.py:874-1017) for the uniform box, in its element order:
 * kind 0 the full Stokes matrix (nel*468 entries, pressure indices offset by Nfem_V), 1 K (nel*324),
 * 2 G (nel*72), 3 G^T (nel*72), 4 the Q1 pressure mass matrix M_P (nel*16), 5 the Q2 temperature
 * matrix (nel*81) -- the triplets the assembly's VV layouts pair with. */
#define MW_COO_STOKES 0
#define MW_COO_K 1
#define MW_COO_G 2
#define MW_COO_GT 3
#define MW_COO_MP 4
#define MW_COO_T 5
int64_t mw_coo_length(mw_box box, int32_t kind);
int mw_coo_pattern(mw_box box, int32_t kind, int32_t* II, int32_t* JJ, void* stream);
/* The summed matrix coo_matrix((VV, (II, JJ))).tocsr() of meeuuw.py:1784-1800 / :2232 in CSR form on
 * the device: mw_csr_pattern writes the row pointers (rows + 1, int64) and returns nnz (synchronises;
 * workspace mw_csr_workspace_bytes), mw_csr_columns the sorted column indices (nnz, int32),
 * mw_csr_values the values from a VV of the same kind (duplicates summed in ascending element
 * order).  The pattern is constant: build it once, refresh the values every step. */
int64_t mw_csr_rows(mw_box box, int32_t kind);
size_t mw_csr_workspace_bytes(mw_box box, int32_t kind);
int mw_csr_pattern(mw_box box, int32_t kind, int64_t* row_ptr, int64_t* nnz, void* work, size_t work_bytes,
                   void* stream);
int mw_csr_columns(mw_box box, int32_t kind, const int64_t* row_ptr, int32_t* col, void* stream);
int mw_csr_values(mw_box box, int32_t kind, const double* VV, const int64_t* row_ptr, const int32_t* col, double* val,
                  void* stream);

/* ======================= energy solve ======================= */

/* y = A x with A the summed element matrices VV_T (nel*81, build_matrix_energy.py:133-137). */
int mw_energy_matvec(mw_box box, const double* VV_T, const double* x, double* y, void* stream);

/* Iterations and relative residual of the last energy solve from the device scalars in `work`
 * (synchronises).  When mw_energy_solve is called on a stream that is recording a CUDA graph the
 * solve is recorded into it (a device-side loop) and reports 0 / 0; read the outcome here after a
 * replay. */
int mw_energy_device_info(mw_box box, const void* work, int32_t* iters, double* relres, void* stream);
/* T = A^-1 rhs (replaces spsolve of coo_matrix((VV_T,(II_T,JJ_T))).tocsr(), meeuuw.py:2232-2235):
 * Jacobi-preconditioned BiCGSTAB in FP64 from the initial guess in T, to rtol. */
size_t mw_energy_solve_workspace_bytes(mw_box box);
int mw_energy_solve(mw_box box, const double* VV_T, const double* rhs, double* T, double rtol, int32_t maxit,
                    int32_t* iters, double* relres, void* work, size_t work_bytes, void* stream);

/* Matrix-free form of the same system (no reference counterpart as an interface: it replaces the
 * pair build_matrix_energy, build_matrix_energy.py:12-141, + spsolve, meeuuw.py:2232-2235, where
 * the element matrices are not needed).  mw_energy_op_setup takes build_matrix_energy's inputs and
 * writes into `op` (mw_energy_op_bytes) the Gauss-point coefficients of A = M + (dt/2)(Ka + Kd)
 * (5 x 9 doubles per element), the summed element diagonals and the Dirichlet flags, and writes rhs
 * as build_matrix_energy does (:112-130, to rounding); the box's Jacobian is diagonal, so jcbi01q
 * and jcbi10q are not read and N_T / dNdr_T / dNds_T are the standard Q2 values at the 3x3 Gauss
 * points.  mw_energy_op_apply: y = A x with the reference's Dirichlet elimination.
 * mw_energy_op_solve: mw_energy_solve on the matrix-free operator (same iteration, device info
 * and recording).  The first call on a device loads the reference-element tables (synchronous). */
size_t mw_energy_op_bytes(mw_box box);
int mw_energy_op_setup(mw_box box, mw_energy_in in, void* op, size_t op_bytes, double* rhs, void* stream);
int mw_energy_op_apply(mw_box box, const void* op, const double* x, double* y, void* stream);
size_t mw_energy_op_solve_workspace_bytes(mw_box box);
int mw_energy_op_solve(mw_box box, const void* op, const double* rhs, double* T, double rtol, int32_t maxit,
                       int32_t* iters, double* relres, void* work, size_t work_bytes, void* stream);

/* ======================= learned warm start: tensor-core kernels ======================= */
/* No reference counterpart: the learned warm start is this build's addition to the method. */

#define MW_GEMM_EPI_F32 0   /* out: float, D (+ bias)                      */
#define MW_GEMM_EPI_BF16 1  /* out: bf16, relu?(D + bias)                  */

typedef struct {
  int32_t mode, relu, splits; /* splits > 1: split-K with FP32 partials in `work` (mode F32 only) */
  const float* bias;          /* per output column, may be NULL                                  */
  void* out;                  /* row-major [M, N] with leading dimension ldo                     */
  int64_t ldo;
} mw_gemm_epilogue;

/* D[M, N] = A[M, K] * B[N, K]^T with BF16 operands (row-major, leading dimensions lda, ldb >= K,
 * K a multiple of 64, 16-byte aligned rows) and FP32 accumulation: TMA-fed tcgen05.mma with
 * the accumulator in TMEM.  err (device int32, may be NULL) receives MW_FLAG_ITER_LIMIT if a
 * pipeline wait ever gives up. */
size_t mw_gemm_workspace_bytes(int32_t M, int32_t N, int32_t splits);
int mw_gemm_bf16_tn(int32_t M, int32_t N, int32_t K, const void* A, int64_t lda, const void* B, int64_t ldb,
                    mw_gemm_epilogue epi, void* work, size_t work_bytes, int32_t* err, void* stream);

/* 3x3 'same' convolution of NHWC BF16 activations X [B, H, W, C] as an implicit GEMM:
 * out[B*H*W, N] = im2col(X) * Wt[N, ldw]^T with the im2col layout (K = tap*C + c, tap = 3 dy + dx)
 * never written: each K block's A tile is loaded from X by a 4D TMA box at the tap's offset.  The
 * same K blocks and MMAs in the same order as mw_gemm_bf16_tn on im2col(X), so the outputs are
 * equal.  C a multiple of 32, W <= 128 with 128 % W == 0, H*W a multiple of 128, ldw >= 9 C,
 * splits = 1; otherwise MW_ERR_BAD_ARG (use mw_unet_im2col + mw_gemm_bf16_tn). */
int mw_conv3x3_bf16(int32_t B, int32_t H, int32_t W, int32_t C, const void* X, int32_t N, const void* Wt, int64_t ldw,
                    mw_gemm_epilogue epi, int32_t* err, void* stream);

/* U-Net building blocks (activations NHWC BF16, gradients FP32; conv K index = tap*C + c, zero
 * padded to Kp, a multiple of 64).  transposed=1 writes the im2col matrix as [Kp, ldT] with
 * ldT >= B*H*W and zeros in the columns past B*H*W (ldT ignored otherwise). */
int mw_unet_im2col(int32_t B, int32_t H, int32_t W, int32_t C, int32_t Kp, int32_t transposed, int64_t ldT,
                   const void* X, void* col, void* stream);
int mw_unet_cast_bf16(int64_t n, const float* a, void* b, void* stream);
/* weights of the data-gradient convolution: Wt[ci][tap*Cout+co] = W[co][(8-tap)*Cin+ci] */
int mw_unet_weights_bwd(int32_t Cout, int32_t Cin, int32_t Kp_in, int32_t Kp_out, const float* W, void* Wt,
                        void* stream);
/* dZ = dA * (A > 0) (relu=1) or dA: bf16 [M,C], bf16 transposed [C,ldT] (ldT >= M, columns past
 * M left untouched), fp32 [M,C] */
int mw_unet_relu_grad(int64_t M, int32_t C, int32_t relu, int64_t ldT, const float* dA, const void* A, void* dZ,
                      void* dZT, float* dZ32, void* stream);
int mw_unet_colsum(int64_t M, int32_t C, const float* X, float* out, void* stream);
int mw_unet_avgpool2(int32_t B, int32_t H, int32_t W, int32_t C, const void* X, void* Y, void* stream);
int mw_unet_avgpool2_bwd(int32_t B, int32_t H, int32_t W, int32_t C, const float* dY, float* dX, int32_t accumulate,
                         void* stream);
int mw_unet_upsample2_into(int32_t B, int32_t h, int32_t w, int32_t C, int32_t Ctot, int32_t c0, const void* X,
                           void* Y, void* stream);
int mw_unet_copy_channels(int64_t P, int32_t C, int32_t Ctot, int32_t c0, const void* X, void* Y, void* stream);
int mw_unet_upsample2_bwd(int32_t B, int32_t h, int32_t w, int32_t C, int32_t Ctot, int32_t c0, const float* dY,
                          float* dX, void* stream);
int mw_unet_slice_grad(int64_t P, int32_t C, int32_t Ctot, int32_t c0, const float* dY, float* dX, int32_t accumulate,
                       void* stream);
int mw_unet_mse(int64_t n, const float* y, const float* t, float* dy, double* loss_part, int32_t nparts,
                void* stream);
int mw_unet_adam(int64_t n, float* w, float* m, float* v, const float* g, float lr, float b1, float b2, float eps,
                 float bc1, float bc2, void* w16, void* stream);
/* network input [nelz/f, nelx/f, 2] from T (nodal) and eta_e: (T at element centres,
 * (log10 eta_e - mean)/2.5), each averaged over f x f elements; stats = {mean log10 eta,
 * Ra / 10^mean} (device) */
int mw_unet_features(mw_box box, int32_t f, const double* T, const double* eta_e, double Ra, double* stats, void* X,
                     void* stream);
/* network output [nelz/f, nelx/f, 5] -> Stokes initial guess (solV interleaved on the Q2
 * lattice, solP on Q1 nodes; bilinear in the network-cell centres, fixed dofs 0).  Channels:
 * u/sv, w/sv, (p - hydrostatic)/sp, log10 sv, log10 sp; velocities in units of stats[1], dynamic
 * pressure in units of pscale, the hydrostatic pressure ghyd * (Lz/2 - z) added (ghyd = rho0 |g_z|
 * in the solver's pressure units).  scales (device, 2 doubles) receives the predicted (sv, sp). */
int mw_unet_to_fields(mw_box box, int32_t f, const float* Y, const double* stats, double pscale, double ghyd,
                      double* scales, const uint8_t* bc_fix_V, double* solV, double* solP, void* stream);
/* The same two on a network grid gzp x gxp at least nelz/f x nelx/f (the network needs multiples
 * of 8): the features repeat the last cell row and column, the guess reads the mesh's cells only. */
int mw_unet_features_padded(mw_box box, int32_t f, int32_t gxp, int32_t gzp, const double* T, const double* eta_e,
                            double Ra, double* stats, void* X, void* stream);
int mw_unet_to_fields_padded(mw_box box, int32_t f, int32_t gxp, const float* Y, const double* stats, double pscale,
                             double ghyd, double* scales, const uint8_t* bc_fix_V, double* solV, double* solP,
                             void* stream);
/* training targets [nelz, nelx, 5] from a solution (inverse of mw_unet_to_fields at the element
 * centres); scales (device, 2 doubles) receives the solution's (sv, sp) */
int mw_unet_targets(mw_box box, const double* solV, const double* solP, const double* stats, double pscale,
                    double ghyd, double* scales, float* Y, void* stream);

#ifdef __cplusplus
}
#endif
#endif
