/*
 * C ABI of the B200 (sm_100a) hex8 SIMP topology-optimisation hot path.
 *
 * Every entry point returns an int status (0 = ok, see TF_STATUS_*) and stores
 * a message retrievable with tf_last_error().  Device pointers are raw CUDA
 * pointers owned by the caller; `stream` is a cudaStream_t passed as void*
 * (NULL = legacy default stream).  Dense right-hand-side / solution blocks are
 * column-contiguous: column c of an [ndof x R] block starts at ptr + c * ndof,
 * i.e. a Fortran-ordered NumPy [ndof, R] array, with dof = 3 * node + component
 * and nodes in C order over (nx+1, ny+1, nz+1).
 *
 * The reference interface each function replaces is cited beside it
 * (paths inside the reference project AAPPHH/Deep_Frame).
 */
#ifndef TF_B200_H
#define TF_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define TF_API __attribute__((visibility("default")))
#else
#define TF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  TF_STATUS_OK = 0,
  TF_STATUS_INVALID = 1,        /* bad argument: ValueError in the reference */
  TF_STATUS_CUDA = 2,           /* CUDA runtime failure */
  TF_STATUS_NOT_CONVERGED = 3,  /* PCG did not reach the tolerance */
  TF_STATUS_NUMERIC = 4,        /* breakdown (non-SPD coarsest matrix, non-finite values) */
  TF_STATUS_INTERNAL = 5
};

enum { TF_PRECISION_FLOAT64 = 0, TF_PRECISION_FLOAT32 = 1, TF_PRECISION_BFLOAT16 = 2, TF_PRECISION_FLOAT16 = 3 };
enum { TF_SMOOTHER_JACOBI = 0, TF_SMOOTHER_CHEBYSHEV = 1 };
enum { TF_CYCLE_V = 0, TF_CYCLE_W = 1 };
enum { TF_COARSE_GALERKIN = 0, TF_COARSE_REDISCRETIZE = 1 };

typedef struct tf_handle tf_handle;

/* Structured grid of shape[0] x shape[1] x shape[2] hex8 elements. */
typedef struct tf_grid {
  int64_t shape[3];
  double spacing[3];
} tf_grid;

/* Multigrid settings; same meaning as the reference's MULTIGRID dict
 * (deep_frame/topology_multigrid.py:8-11). */
typedef struct tf_settings {
  int32_t precision;          /* work precision of the V-cycle (TF_PRECISION_*) */
  int32_t smoother;           /* TF_SMOOTHER_* */
  int32_t cycle;              /* TF_CYCLE_* */
  int32_t coarse;             /* TF_COARSE_* */
  int32_t sweeps;             /* Jacobi sweeps on the finest level (x growth^level below) */
  int32_t chebyshev_degree;   /* Chebyshev degree on the finest level (x growth^level below) */
  int32_t max_levels;
  int32_t power_iterations;   /* lambda_max(D^-1 A) power iterations per level */
  int32_t max_iterations;     /* PCG iteration limit */
  int32_t retries;            /* FP64 re-runs of columns that missed the tolerance */
  int32_t batch;              /* columns per PCG launch (0 = all live columns at once) */
  int32_t tensor_cores;       /* 1: FP32 finest-level V-cycle apply on the tensor cores (tcgen05, TF32 operands,
                                 FP32 accumulation); 0: FP32 CUDA-core stencil.  FP64 applies are unaffected. */
  int64_t coarsest_dofs;      /* level count grows until the coarsest grid has <= this many dofs */
  double damping;             /* Jacobi damping */
  double chebyshev_ratio;     /* lambda_max / lambda_min of the Chebyshev interval */
  double growth;              /* smoothing growth factor per level */
  double tolerance;           /* relative residual of the recomputed true residual */
  double dead_ratio;          /* coarse dofs with diag <= dead_ratio * max(diag) are dropped */
  double zero_rhs;            /* columns with norm <= zero_rhs * max norm are skipped */
  double reliable;            /* mixed PCG: the FP64 residual is recomputed once a column's iterated residual fell by this
                                 factor since the last recomputation (0 < reliable < 1) */
  int32_t pcg_precision;      /* TF_PRECISION_FLOAT64: the reference's FP64 PCG.  TF_PRECISION_FLOAT32 (with the FP32 work
                                 precision): FP32 PCG iterations and operator, x in FP64, FP64 true residuals replacing the
                                 iterated one (reliable updates) and deciding convergence; no counterpart in the reference */
  int32_t fine_tz;            /* node-tile height (along z) of the finest-level operator: 7, 8, 9, or 0 = 8 unless 9 pads
                                 at least 15 % fewer threads along z (the 9-high variants spill registers) or, for the
                                 FP32 operator, 7 pads at least 10 % fewer; a tuning choice that never changes results */
} tf_settings;

/* Solve report (deep_frame/topology_multigrid.py:367-373).  Arrays are caller-owned. */
typedef struct tf_report {
  int32_t* iterations;        /* [nrhs] or NULL */
  double* relative_residual;  /* [nrhs] or NULL */
  double* history;            /* [history_capacity] max relative residual per PCG step, or NULL */
  int32_t history_capacity;
  int32_t history_len;
  int32_t converged;
  int32_t batches;
  int32_t retried_columns;
  int32_t zero_rhs_columns;
  int32_t levels;
  int32_t steps;
  int64_t coarsest_dofs;
  double seconds;
  double setup_s;
  double lambda_max[16];
} tf_report;

/* Fill `s` with the library defaults (the reference's MULTIGRID values, with
 * coarsest_dofs sized for a dense coarsest factor). */
TF_API int tf_default_settings(tf_settings* s);

/* GeometricMultigrid.__init__(shape, spacing, ke, settings, me)
 * (deep_frame/topology_multigrid.py:47-79).  ke, me: 24x24 row-major FP64 host
 * arrays (me may be NULL). */
TF_API int tf_create(const tf_grid* grid, const double* ke, const double* me, const tf_settings* settings, tf_handle** out);

/* Level count and padded element shape chosen at creation (topology_multigrid.py:58-63). */
TF_API int tf_levels(const tf_handle* h, int32_t* levels, int64_t padded[3]);

/* GeometricMultigrid.update(moduli) (topology_multigrid.py:97-100): element moduli
 * [nelem] FP64 on the device, C order; drops every cached hierarchy. */
TF_API int tf_update(tf_handle* h, const double* moduli_dev, void* stream);

/* Register the Dirichlet dof set of hierarchy `key` (the `fixed` argument of
 * GeometricMultigrid.solve / .hierarchy, topology_multigrid.py:145,336).  Host
 * array of unpadded dof indices; the hierarchy itself is built lazily by tf_solve. */
TF_API int tf_set_bc(tf_handle* h, uint64_t key, const int64_t* fixed, int64_t count);

/* GeometricMultigrid.solve(key, fixed, forces) (topology_multigrid.py:336-375) for a
 * Dirichlet-supported key: f_dev [nrhs][ndof] in, u_dev [nrhs][ndof] out (device FP64). */
TF_API int tf_solve(tf_handle* h, uint64_t key, const double* f_dev, int32_t nrhs, double* u_dev, tf_report* report,
             void* stream);

/* tf_solve started from an initial guess: u_dev is read as the guess (Dirichlet dofs are
 * masked to zero) and overwritten by the solution.  The reference's _pcg(hierarchy, rhs,
 * initial) (topology_multigrid.py:407-417, used by its retries at :393) starts from
 * r = b - A x0 the same way; zero-force columns still return zero. */
TF_API int tf_solve_guess(tf_handle* h, uint64_t key, const double* f_dev, int32_t nrhs, double* u_dev, tf_report* report,
                          void* stream);

/* tf_solve over `count` independent instances at once: instance i solves hierarchy keys[i] of
 * handles[i] for f_dev[i] [nrhs[i]][ndof_i] into u_dev[i], reports[i] (reports may be NULL).
 * The result of each instance is that of its own tf_solve (the same PCG, convergence test and
 * retries, topology_multigrid.py:336-454); the difference is the schedule: every PCG and V-cycle
 * stage runs as one launch over all instances' blocks, in place of one launch per instance
 * (the reference solves one problem per call, with the columns of one load set batched,
 * topology_multigrid.py:353-362).  Each instance needs its own handle; all share the element
 * stiffness ke and the V-cycle settings, run the FP64 PCG (pcg_precision float64) with V-cycles
 * on the CUDA-core operators, and solve their live columns as one block (settings.batch 0 or at
 * least that count).  One stream for all.  Each report's `seconds` is the whole batch's time. */
TF_API int tf_solve_batch(tf_handle* const* handles, const uint64_t* keys, int32_t count, const double* const* f_dev,
                          const int32_t* nrhs, double* const* u_dev, tf_report* reports, void* stream);

/* Mass operator of GeometricMultigrid.eigenpairs (topology_multigrid.py:491-496): y = mask *
 * (sum_e mass_e M0 (mask u)_e + lumped * u), with M0 the `me` given to tf_create, mass_dev the
 * element masses [nelem] (unpadded, C order), lumped_dev the lumped nodal masses [ndof] (may be
 * NULL) and mask the live-dof mask of hierarchy `key`; u_dev, y_dev are [nrhs][ndof] device FP64. */
TF_API int tf_mass_apply(tf_handle* h, uint64_t key, const double* mass_dev, const double* lumped_dev, const double* u_dev,
                         int32_t nrhs, double* y_dev, void* stream);

/* GeometricMultigrid.hierarchy(key, fixed) (topology_multigrid.py:145-208): build (or reuse)
 * the hierarchy of `key` now and fill the level fields of `report` (levels, coarsest_dofs,
 * setup_s, lambda_max); report may be NULL. */
TF_API int tf_prepare(tf_handle* h, uint64_t key, tf_report* report, void* stream);

/* GeometricMultigrid.precondition (topology_multigrid.py:318-324): z = M^-1 r with one
 * V-cycle of the hierarchy of `key`, the residual scaled by max|r| per column.
 * r_dev, z_dev: [nrhs][ndof] device FP64. */
TF_API int tf_precondition(tf_handle* h, uint64_t key, const double* r_dev, int32_t nrhs, double* z_dev, void* stream);

/* GeometricMultigrid.operator (topology_multigrid.py:105-109) / .product (:455-457):
 * y = K(E) u for nrhs columns; with use_mask != 0 the live mask of `key` is applied
 * to input and output (the reduced operator used by PCG). */
TF_API int tf_apply(tf_handle* h, uint64_t key, int32_t use_mask, const double* u_dev, int32_t nrhs, double* y_dev,
             void* stream);

/* One level operator of the hierarchy of `key` in FP64 (the reference's _apply, topology_multigrid.py:110-117):
 * level 0 the masked finest operator, level l >= 1 the Galerkin operator P^T A_{l-1} P of
 * :145-208 as assembled by this library, y = mask_l * A_l (mask_l * u).  u_dev, y_dev are
 * [nrhs][3 * nodes_l] device FP64 vectors on the PADDED level grid of
 * (padded[0] >> l) x (padded[1] >> l) x (padded[2] >> l) elements (tf_levels gives `padded`). */
TF_API int tf_apply_level(tf_handle* h, uint64_t key, int32_t level, const double* u_dev, int32_t nrhs, double* y_dev,
                          void* stream);

/* GeometricMultigrid.element_energy (topology_multigrid.py:458-459) and the
 * sensitivity sums of HexElasticity._collect (topology_optimization.py:721-734) /
 * InterfaceCovariance.energy (topology_problem.py:647-652):
 *   per_column != 0:  out[c][e] = u_c,e^T K0 u_c,e                 (out is [nrhs][nelem])
 *   otherwise:        out[e] (+)= scale[e] * sum_j coef[j] * w_j,e^T K0 w_j,e
 * with w_j = u_j (comb == NULL, ncomb ignored) or w_j = sum_c comb[c * ncomb + j] u_c.
 * comb, coef, scale are device arrays and may be NULL (coef, scale default to 1). */
TF_API int tf_element_energy(tf_handle* h, const double* u_dev, int32_t nrhs, const double* comb_dev, int32_t ncomb,
                      const double* coef_dev, const double* scale_dev, double* out_dev, int32_t accumulate,
                      int32_t per_column, void* stream);

/* F = A B^T for column blocks A [ra][n] and B [rb][n] (device FP64, ra, rb <= 64): the
 * flexibility P^T U of InterfaceCovariance.matrix (deep_frame/topology_problem.py:639-646).
 * out_dev is [ra][rb]; scratch_dev holds tf_gram_scratch_size(ra, rb) doubles.  The
 * reduction order is fixed, so results are bitwise reproducible. */
TF_API int tf_gram(const double* a_dev, int32_t ra, const double* b_dev, int32_t rb, int64_t n, double* out_dev,
                   double* scratch_dev, void* stream);
TF_API int64_t tf_gram_scratch_size(int32_t ra, int32_t rb);

/* tf_gram without the scratch argument, for callers that cannot allocate device memory
 * when they need F (a host application that owns every device allocation through a
 * fixed budget, or code running inside its callbacks).  No counterpart in the reference.
 * The partials live in a static 4.85 MB device array inside the library (held by every
 * GPU that loads it), which limits ra * rb to 2048 pairs; larger requests return
 * TF_STATUS_INVALID with a message in tf_last_error(NULL).  The first call on a device
 * resolves the array's device address and should come before any stream capture.  All
 * calls share the array: calls that overlap on the GPU race and must be ordered by the
 * caller.  The cached address belongs to the device's primary context (the one the CUDA runtime
 * uses): a caller that makes another driver-API context current, or resets the device, must not
 * call it afterwards in the same process.  Allocates nothing. */
TF_API int tf_gram_static(const double* a_dev, int32_t ra, const double* b_dev, int32_t rb, int64_t n, double* out_dev,
                          void* stream);

/* out[j][i] = sum_c coef[c * ncomb + j] * u[c][i] for column blocks u [nrhs][n] and out [ncomb][n]
 * (device FP64, 1 <= nrhs, ncomb <= 64; coef is a device [nrhs][ncomb] array): the combinations
 * U v of solution columns that the lambda_max sensitivity of InterfaceCovariance.measure needs
 * (deep_frame/topology_problem.py:647-652, 680-683), formed per rank before the all-reduce when the
 * columns are sharded over GPUs. */
TF_API int tf_combine(const double* u_dev, int32_t nrhs, int64_t n, const double* coef_dev, int32_t ncomb, double* out_dev,
                      void* stream);

/* SIMP interpolation (HexElasticity.solve, deep_frame/topology_optimization.py:657-661):
 * moduli = young (eps + (1 - eps) rho^p), derivative = young (1 - eps) p rho^(p-1), both zero
 * where active[c] == 0 (active may be NULL); volume (device scalar, may be NULL) receives
 * sum of rho over the active cells (the volume row of topology_problem.py:345). */
TF_API int tf_simp(const double* rho_dev, int64_t n, double penalization, double min_stiffness_ratio, double young,
                   const uint8_t* active_dev, double* moduli_dev, double* derivative_dev, double* volume_dev, void* stream);

/* ------------------------------------------------------------------------------------
 * Cone density filter (ConeFilter / cone_filter / DensityMap.filtered, .pullback,
 * .project: deep_frame/topology_optimization.py:1082-1178).  Cells are C-ordered over
 * shape; allowed / preserve are host byte masks (preserve may be NULL).  The filter
 * radius may span at most 4 cells per axis.
 * ------------------------------------------------------------------------------------ */
typedef struct tf_filter tf_filter;
TF_API int tf_filter_create(const int64_t shape[3], const double spacing[3], double radius, const uint8_t* allowed,
                            const uint8_t* preserve, tf_filter** out);
/* adjoint == 0: out = allowed * (W (allowed * in * in2)) / sums          (DensityMap.filtered)
 * adjoint != 0: out = free * (W (allowed * in * in2 / sums))             (DensityMap.pullback)
 * in2 is an optional per-cell multiplier (the projection derivative of the pullback). */
TF_API int tf_filter_apply(tf_filter* f, const double* in_dev, const double* in2_dev, double* out_dev, int32_t adjoint, void* stream);
/* Row sums W (allowed) on allowed cells, 1 on forbidden cells (DensityMap.sums). */
TF_API int tf_filter_sums(const tf_filter* f, double* sums_dev, void* stream);
/* Threshold projection with derivative; robust != 0 selects the eroded/dilated form. */
TF_API int tf_filter_project(tf_filter* f, const double* filtered_dev, double beta, double eta, int32_t robust,
                             double* physical_dev, double* derivative_dev, void* stream);
/* DensityMap.volume (topology_optimization.py:1146-1151): *volume_dev = sum(weights *
 * project(filtered(design), eta)) with weights NULL = ones; one fused launch with a
 * deterministic reduction.  Pass the dilated threshold for the robust volume. */
TF_API int tf_filter_volume(tf_filter* f, const double* design_dev, const double* weights_dev, double beta, double eta,
                            int32_t robust, double* volume_dev, void* stream);

/* Optimality-criteria update _oc_update (topology_optimization.py:1197-1233): ratios
 * max(1e-30, -dC/max(dV, 1e-12 max dV)) on the free cells, move-limited bounds, the
 * lowest-design shortcut, multiplier bracketing (x2, at most 100) and bisection (at most
 * 70, relative width 1e-8) against `target` of the volume above evaluated at threshold
 * `eta`.  The search runs on the device; the host reads its state once per 8 rounds.
 * Status TF_NUMERIC with "Invalid OC sensitivities" or "OC could not bracket the volume
 * multiplier" mirrors the reference's RuntimeErrors.  candidate_dev must not alias design_dev. */
typedef struct tf_oc_report {
  double multiplier;   /* accepted multiplier (the bracket's upper end); 0 for the lowest design */
  double lower;        /* lower end of the final bracket */
  double volume;       /* volume of the last evaluated proposal */
  int32_t evaluations; /* volume evaluations */
  int32_t lowest;      /* 1 when the lowest design already exceeded the target */
} tf_oc_report;
TF_API int tf_oc_update(tf_filter* f, const double* design_dev, const double* objective_derivative_dev,
                        const double* volume_derivative_dev, const double* weights_dev, double target, double minimum_density,
                        double move_limit, double beta, double eta, int32_t robust, double* candidate_dev, tf_oc_report* report,
                        void* stream);
TF_API int tf_filter_destroy(tf_filter* f);
/* NULL: the message of this thread's last failed call without a handle (as tf_last_error(NULL)). */
TF_API const char* tf_filter_last_error(const tf_filter* f);

/* ------------------------------------------------------------------------------------
 * Learned initial guess (no counterpart in the reference: the small convolutional
 * network that maps (density, load) to a displacement guess for PCG).  Layers of a 3-D
 * encoder / decoder on channel-major [C][nx][ny][nz] FP32 node grids; every kernel is
 * deterministic.  Errors: tf_nn_last_error().
 * ------------------------------------------------------------------------------------ */
TF_API const char* tf_nn_last_error(void);
/* C = alpha op(A) op(B) + beta C (row-major; op = transpose when trans* != 0), split over K with
 * partial tiles in `work` (>= m * n floats, up to 64 * m * n used) summed in a fixed order. */
TF_API int tf_nn_gemm(int32_t transa, int32_t transb, int32_t m, int32_t n, int32_t k, float alpha, const float* a, int32_t lda,
                      const float* b, int32_t ldb, float beta, float* c, int32_t ldc, float* work, int64_t work_floats, void* stream);
/* Inference form of a 3 x 3 x 3 convolution on the tensor cores (tcgen05 kind::f16, FP16 operands,
 * FP32 accumulation): y[o][v] = act(bias[o] + sum_{c,tap} W[o][c * 27 + tap] x[c][v + offset(tap)])
 * (act = ReLU when relu != 0), x [cin][n] and y [cout][n] FP32 on the node grid `shape`; the
 * weights are packed first by tf_nn_pack16 from FP32 W [cout][27 cin] to FP16 [np][kp] (np a
 * multiple of 16 in [cout, 64], kp a multiple of 64, zero padding).  *err (device int) is set when
 * a bounded wait on the tensor cores timed out. */
TF_API int tf_nn_pack16(const float* w, int32_t cout, int32_t k, void* w16, int32_t np, int32_t kp, void* stream);
TF_API int tf_nn_conv16(const float* x, int32_t cin, const int32_t shape[3], const void* w16, int32_t cout, int32_t np, int32_t kp,
                        const float* bias, int32_t relu, float* y, int32_t* err, void* stream);
/* col[(c * 27 + tap)][v] = in[c][v + offset(tap)], 3 x 3 x 3 taps, zero outside; col2im is its adjoint. */
TF_API int tf_nn_im2col(const float* in, int32_t channels, const int32_t shape[3], float* col, void* stream);
TF_API int tf_nn_col2im(const float* col, int32_t channels, const int32_t shape[3], float* out, void* stream);
/* x = act(x + bias[c]) in place (relu != 0: max(., 0)); act_back: dy *= (y > 0) for relu, dbias (+)= sum over voxels. */
TF_API int tf_nn_bias_act(float* x, const float* bias, int32_t channels, int64_t n, int32_t relu, void* stream);
TF_API int tf_nn_act_back(float* dy, const float* y, int32_t channels, int64_t n, int32_t relu, float* dbias, int32_t accumulate,
                          void* stream);
/* 2 x 2 x 2 average pooling (coarse extent = ceil(fine / 2)); resample mode 0 = nearest upsampling,
 * 1 = pooling adjoint, 2 = upsampling adjoint. */
TF_API int tf_nn_pool(const float* in, int32_t channels, const int32_t fine[3], const int32_t coarse[3], float* out, void* stream);
TF_API int tf_nn_resample(const float* in, int32_t channels, const int32_t fine[3], const int32_t coarse[3], int32_t mode, float* out,
                          void* stream);
/* *loss_dev = sum w (y - t)^2 / count, dy = its gradient (dy may be NULL; w may be NULL = 1); scratch holds
 * tf_nn_mse_scratch_doubles() doubles. */
TF_API int tf_nn_mse(const float* y, const float* target, const float* weight, int64_t n, double count, float* dy, double* scratch,
                     double* loss_dev, void* stream);
TF_API int64_t tf_nn_mse_scratch_doubles(void);
/* Adam with bias correction (step counts from 1). */
TF_API int tf_nn_adam(float* param, const float* grad, float* m, float* v, int64_t n, float lr, float beta1, float beta2, float eps,
                      int32_t step, void* stream);

/* ------------------------------------------------------------------------------------
 * Method of moving asymptotes (mmapy.mmasub as called from
 * deep_frame/topology_optimizers.py:61-63): asymptotes, move limits, convex
 * approximation and the primal-dual interior-point subproblem, n variables on the
 * device, 1 <= m <= TF_MMA_MAX_M constraints.
 * ------------------------------------------------------------------------------------ */
#define TF_MMA_MAX_M 8
typedef struct tf_mma tf_mma;
typedef struct tf_mma_settings {
  double move, asyinit, asydecr, asyincr, asymin, asymax, raa0, albefa, epsimin;
} tf_mma_settings;
TF_API int tf_mma_create(int32_t m, int64_t n, tf_mma** out);
/* Device arrays: xval, xmin, xmax, xold1, xold2, df0dx [n]; dfdx [m][n]; low, upp [n]
 * (in: previous asymptotes, out: new); xnew [n].  Host arrays: fval, a, c, d [m];
 * y_out, lam_out [m] and z_out, newton_iterations may be NULL.  settings NULL = defaults
 * (move 0.5, asyinit 0.5, asydecr 0.7, asyincr 1.2, asymin 0.01, asymax 10, raa0 1e-5,
 * albefa 0.1, epsimin 1e-7). */
TF_API int tf_mma_step(tf_mma* h, int32_t iteration, const double* xval, const double* xmin, const double* xmax,
                       const double* xold1, const double* xold2, const double* df0dx, const double* fval, const double* dfdx,
                       double* low, double* upp, double a0, const double* a, const double* c, const double* d,
                       const tf_mma_settings* settings, double* xnew, double* y_out, double* z_out, double* lam_out,
                       int32_t* newton_iterations, void* stream);
TF_API int tf_mma_destroy(tf_mma* h);
/* NULL: the message of this thread's last failed call without a handle (as tf_last_error(NULL)). */
TF_API const char* tf_mma_last_error(const tf_mma* h);

/* ------------------------------------------------------------------------------------
 * Dense FP64 direct solver of a small SPD system (CudaDirectSolver,
 * deep_frame/topology_optimization.py:80-244; the reference factors with cuDSS).
 * n <= 32768; the matrix arrives as device CSR (int32 indptr [n+1], indices, FP64 data)
 * and is symmetrised; right-hand sides and solutions are [nrhs][n] device blocks.
 * ------------------------------------------------------------------------------------ */
typedef struct tf_chol tf_chol;
TF_API int tf_chol_create(int64_t n, tf_chol** out);
TF_API int tf_chol_factor_csr(tf_chol* h, const int32_t* indptr_dev, const int32_t* indices_dev, const double* data_dev,
                              void* stream);
TF_API int tf_chol_solve(tf_chol* h, const double* b_dev, int32_t nrhs, double* x_dev, void* stream);
/* Frees the handle in every case; a device error seen while waiting for it returns TF_STATUS_CUDA with
 * the message in tf_chol_last_error(NULL) (CudaDirectSolver.close, topology_optimization.py:205-239). */
TF_API int tf_chol_destroy(tf_chol* h);
/* NULL: the message of this thread's last failed call without a handle (as tf_last_error(NULL)). */
TF_API const char* tf_chol_last_error(const tf_chol* h);

/* CUDA-event timing of the kernel classes this handle launches, recorded on the launching
 * stream: 0 FP64 finest operator of the PCG, 1 finest-level smoothing / residual in the work
 * precision, 2 Galerkin-level operators, 3 restriction + prolongation, 4 PCG vector kernels,
 * 5 dense coarsest solve, 6 hierarchy set-up, 7 element energies.  With nclasses > 0 the
 * summed milliseconds and launch counts since the previous call are returned (after
 * synchronising the recorded events) and the record is cleared; `enable` switches recording
 * on or off for the calls that follow. */
TF_API int tf_timers(tf_handle* h, int32_t enable, double* ms, int64_t* counts, int32_t nclasses);

/* Kernels launched by this library in the calling process so far. */
TF_API int64_t tf_launch_count(void);

/* Release the handle and every device buffer it owns (GeometricMultigrid.close,
 * topology_multigrid.py:543-548).  Idempotent for NULL.  The handle is freed in every case; an
 * error the device reports while the destroy waits for it returns TF_STATUS_CUDA with the message
 * in tf_last_error(NULL), so close() can hand it back as the reference's close does. */
TF_API int tf_destroy(tf_handle* h);

/* Message of the last failed call on `h` (or, with h NULL, of the last failed tf_create,
 * tf_filter_create, tf_mma_create, tf_chol_create or tf_gram_static on this thread). */
TF_API const char* tf_last_error(const tf_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* TF_B200_H */
