/*
 * fagra_b200 — C ABI of a B200 (sm_100a) linear-solve and linearization backend
 * for the fagra factor-graph library.
 *
 * Each entry point below replaces one method of fagra's statically dispatched
 * linear-backend trait or one step of its optimizers; the citation beside it
 * names the fagra source it stands in for (paths inside the fagra repository).
 * A Rust `impl LeastSquaresBackend for GpuSchur` binds these symbols 1:1.
 *
 * Conventions
 *  - Every call returns fg_status (0 = FG_OK); no call aborts the process.
 *  - Scalars cross the boundary as double; FG_PRECISION_* selects the device
 *    storage precision of the bulk data (Jacobians, blocks, Krylov vectors).
 *  - A handle owns all of its device and pinned host buffers. Pointers handed
 *    back (the step delta) borrow handle storage and stay valid until the next
 *    call on that handle, as DampedStep<'_> borrows the backend in fagra.
 *  - Calls on one handle are not thread-safe (fagra uses &mut self). All work
 *    of one device runs on one library stream, see fg_device_stream().
 */
#ifndef FAGRA_B200_H
#define FAGRA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#define FG_API extern "C" __attribute__((visibility("default")))
#else
#define FG_API __attribute__((visibility("default")))
#endif

/* src/error.rs:19-76 — SolverError and EvaluationError variants, one code each. */
typedef enum {
  FG_OK = 0,
  FG_DUPLICATE_COVARIANCE_BLOCK = 1, /* SolverError::DuplicateCovarianceBlock */
  FG_SINGULAR_INFORMATION = 2,       /* SolverError::SingularInformation */
  FG_INVALID_INFORMATION = 3,        /* SolverError::InvalidInformation */
  FG_INVALID_RANK_TOLERANCE = 4,     /* SolverError::InvalidRankTolerance */
  FG_BATCH_NOT_EMPTY = 5,            /* SolverError::BatchNotEmpty */
  FG_INVALID_OPTIONS = 6,            /* SolverError::InvalidOptions */
  FG_KEY_ERROR = 7,                  /* SolverError::Key */
  FG_LINEAR_SOLVE_FAILED = 8,        /* SolverError::LinearSolveFailed (LM retries) */
  FG_NO_CONVERGENCE = 9,             /* SolverError::NoConvergence */
  FG_NO_PROGRESS = 10,               /* SolverError::NoProgress */
  FG_INVALID_EVALUATION = 20,        /* EvaluationError::InvalidEvaluation */
  FG_DIMENSION_MISMATCH = 21,        /* EvaluationError::DimensionMismatch */
  FG_INVALID_EMISSION = 22,          /* EvaluationError::InvalidEmission */
  FG_UNSUPPORTED_STRUCTURE = 23,     /* EvaluationError::UnsupportedStructure */
  FG_CUDA_ERROR = 40,                /* a CUDA runtime call failed; see fg_last_error() */
  FG_OUT_OF_MEMORY = 41,             /* device or pinned allocation failed */
  FG_DEVICE_TIMEOUT = 42,            /* a bounded device-side wait gave up */
  FG_NULL_ARGUMENT = 43,             /* a required pointer argument was NULL */
  FG_NO_DEVICE = 44                  /* no CUDA device (the product has no CPU fallback) */
} fg_status;

/* src/schur.rs:31-41 SchurTermination (+ 0 = None) */
typedef enum {
  FG_TERM_NONE = 0,
  FG_TERM_CONVERGED = 1,
  FG_TERM_ITERATION_LIMIT = 2,
  FG_TERM_NOT_POSITIVE_DEFINITE = 3,
  FG_TERM_NONFINITE = 4
} fg_termination;

typedef enum {
  FG_PRECISION_F64 = 0,        /* everything in f64: the reference arithmetic */
  FG_PRECISION_F32_REFINED = 1 /* f32 bulk; f64 dots, norms, cost and refinement residual */
} fg_precision;

typedef enum {
  FG_PRECOND_RETAINED_BLOCKS = 0, /* (B + lambda I) block-Jacobi, src/schur.rs:658-682 */
  FG_PRECOND_SCHUR_DIAGONAL = 1,  /* exact 9x9 diagonal blocks of S (docs/schur-performance.md:155-159) */
  FG_PRECOND_LEARNED = 2          /* block-Jacobi reshaped by an attached fg_gnn, block-Jacobi fallback;
                                     no reference counterpart */
} fg_preconditioner;

/* src/schur.rs:116-143 public fields, plus device-side choices. */
typedef struct {
  size_t max_iterations;     /* CG iteration limit per attempt; default 1000 */
  double relative_tolerance; /* reduced-residual tolerance in [0,1); default max(1e-10, 128 eps) */
  int collect_timings;       /* default 0 */
  int precision;             /* fg_precision; default FG_PRECISION_F64 */
  int preconditioner;        /* fg_preconditioner; default FG_PRECOND_RETAINED_BLOCKS */
  int device;                /* CUDA device ordinal; default 0 */
  double residual_replacement; /* FP32 mode: the recurrence residual is replaced by the FP64
                                  residual b - S x each time it falls by this factor; default 0 =
                                  automatic: the reduction to the relative tolerance split into the
                                  fewest equal factors of at most 1e-4 */
  int operator_variant;        /* FP32 BAL-shaped systems: 0 = autotune (default), 1..4 = force the
                                  reduced-operator variant of fg_schur_operator_info (a variant
                                  that does not apply to the structure falls back to 1) */
  int coarse_correction;       /* 1: two-level PCG, z = M r + W (W^T S W)^-1 W^T r with the coarse
                                  basis W a device problem supplies (BAL: the 7 similarity-gauge
                                  directions of the cameras); 0 (default): the reference's PCG */
  int learned_policy;          /* FG_PRECOND_LEARNED only. 0 (default): the first learned solve is
                                  compared once with a block-Jacobi solve of the same system, and
                                  the network is switched off for this backend when block-Jacobi
                                  needs fewer iterations or less device time; 1: the network
                                  preconditions every solve, block-Jacobi only redoes a solve that
                                  meets non-positive curvature or does not converge */
} fg_schur_options;

/* src/schur.rs:44-60 SchurDiagnostics (has_* = Some) */
typedef struct {
  int termination; /* fg_termination */
  size_t iterations;
  double damping;
  double estimated_relative_residual;
  double reduced_relative_residual;
  double scaled_relative_residual;
  double original_relative_residual;
  int has_estimated, has_reduced, has_scaled, has_original;
  size_t refinements; /* FP32 mode: FP64 residual replacements in this attempt */
  /* FG_PRECOND_LEARNED only (no reference counterpart): the preconditioner
   * whose step was kept, 0 when the learned PCG ran without a fallback, 1
   * when it met non-positive curvature or did not converge, 2 when the
   * block-Jacobi comparison solve needed fewer iterations or less device time
   * than the learned solve plus the network's inference (the learned
   * preconditioner is then switched off for this backend); iteration counts
   * of the two solves of this attempt (0 when not run), and the device
   * seconds of the comparison. `iterations` is their sum. */
  int preconditioner_used, learned_fallback;
  size_t learned_iterations, block_jacobi_iterations;
  double learned_seconds, block_jacobi_seconds;
  size_t coarse_vectors; /* coarse basis size used by this attempt's PCG (0: one-level) */
} fg_schur_diagnostics;

/* src/schur.rs:75-91 SchurTimings, seconds, device event time. */
typedef struct {
  double preparation, factorization, linear_solve, products, preconditioner, verification;
} fg_schur_timings;

typedef struct fg_backend fg_backend;
typedef struct fg_bal_problem fg_bal_problem;
typedef struct fg_gnn fg_gnn;

/* ---- library ---------------------------------------------------------- */
FG_API const char* fg_version(void);
FG_API const char* fg_last_error(void);   /* thread-local text of the last non-FG_OK status */
FG_API fg_status fg_device_count(int* count);
/* The CUDA stream every call on `device` runs on (cudaStream_t as void*). */
FG_API fg_status fg_device_stream(int device, void** stream);
/* Kernel launches issued by this library since load (all devices). */
FG_API uint64_t fg_kernel_launches(void);

/* ---- Schur backend: LeastSquaresBackend (src/optimization.rs:131-169) ---- */
FG_API void fg_schur_default_options(fg_schur_options* out);
/* Schur::new (src/schur.rs:149-178) */
FG_API fg_status fg_schur_create(size_t retained_dimension, size_t retained_block_width,
                                 size_t eliminated_block_width, const fg_schur_options* options,
                                 fg_backend** out);
FG_API void fg_backend_destroy(fg_backend* backend);
/* Update the public fields (max_iterations, relative_tolerance, collect_timings,
 * preconditioner) between calls, as Rust code assigns them (src/schur.rs:117-125). */
FG_API fg_status fg_schur_set_options(fg_backend* backend, const fg_schur_options* options);
/* LeastSquaresBackend::prepare (src/schur.rs:409-431) */
FG_API fg_status fg_backend_prepare(fg_backend* backend, size_t dimension);
/* LeastSquaresBackend::clear (src/schur.rs:432-437) */
FG_API fg_status fg_backend_clear(fg_backend* backend);
/* LeastSquaresBackend::accumulate (src/schur.rs:438-482, src/linear_model.rs:180-210).
 * residual[rows]; block k has column offset cols[k], width widths[k] and its
 * Jacobian element (i,j) at jacobians[k][i*row_strides[k] + j*col_strides[k]]. */
FG_API fg_status fg_backend_accumulate(fg_backend* backend, size_t rows, const double* residual,
                                       size_t nblocks, const size_t* cols, const size_t* widths,
                                       const double* const* jacobians, const ptrdiff_t* row_strides,
                                       const ptrdiff_t* col_strides);
/* LeastSquaresBackend::gradient_norm (src/schur.rs:483-485) */
FG_API fg_status fg_backend_gradient_norm(fg_backend* backend, double* out);
/* LeastSquaresBackend::solve (src/schur.rs:486-489) */
FG_API fg_status fg_backend_solve(fg_backend* backend, const double** delta, size_t* len);
/* LeastSquaresBackend::prepare_damping (src/schur.rs:490-526) */
FG_API fg_status fg_backend_prepare_damping(fg_backend* backend, double min_column_norm);
/* LeastSquaresBackend::solve_damped (src/schur.rs:527-545). On FG_OK, *delta
 * borrows a pinned host copy of the step (len = dimension). */
FG_API fg_status fg_backend_solve_damped(fg_backend* backend, double lambda, const double** delta,
                                         size_t* len, double* predicted_reduction);
/* Device-resident variant: the step stays on the device (*delta_device is a
 * device pointer of `dimension` doubles); no device-to-host copy. */
FG_API fg_status fg_backend_solve_damped_device(fg_backend* backend, double lambda,
                                                const double** delta_device,
                                                double* predicted_reduction);
/* LeastSquaresBackend::linear_solve_work (src/schur.rs:403-408) */
FG_API fg_status fg_backend_linear_solve_work(const fg_backend* backend, size_t* solves,
                                              size_t* iterations, int* available);
/* Schur::diagnostics / Schur::timings (src/schur.rs:183-190) */
FG_API fg_status fg_schur_get_diagnostics(const fg_backend* backend, fg_schur_diagnostics* out);
FG_API fg_status fg_schur_get_timings(const fg_backend* backend, fg_schur_timings* out);

/* Structure export for bit-exact index-map checks: sizes, then the maps in the
 * reference's own layouts — Jacobian blocks {row,col,rows,cols,start}
 * (src/linear_model.rs:12-19), Schur edges {retained,eliminated,
 * retained_jacobian,eliminated_jacobian} (src/schur.rs:93-99), the owner map
 * with first-appearance block ids (src/linear_model/block_factors.rs:52-87) and
 * variable blocks {col,width,start}. Any output pointer may be NULL. */
FG_API fg_status fg_schur_structure_sizes(fg_backend* backend, size_t* nblocks, size_t* nedges,
                                          size_t* nvalues, size_t* nvariables, size_t* rows,
                                          size_t* cols);
FG_API fg_status fg_schur_export_structure(fg_backend* backend, uint64_t* blocks5, uint64_t* edges4,
                                           uint64_t* owners, uint64_t* variables3);
/* Model values in the reference layouts (f64 copies): packed Jacobian values,
 * -r, gradient, column scales, Gram blocks (first-appearance order, column
 * major) and cross blocks cross[(e*pw+p)*cw+c] (src/schur.rs:516). */
FG_API fg_status fg_schur_export_model(fg_backend* backend, double* values, double* negative_residual,
                                       double* gradient, double* scales, double* gram, double* cross);
/* One application of the reduced operator S = lambda I + B - E C^-1 E^T
 * (src/schur.rs:606-652) to a host vector x of length retained_dimension;
 * requires prepare_damping. */
FG_API fg_status fg_schur_reduced_apply(fg_backend* backend, double lambda, const double* x, double* y);

/* ---- LSMR backend: src/lsmr.rs over the same LeastSquaresBackend entry points ----
 * fg_backend_prepare / clear / accumulate / gradient_norm / prepare_damping /
 * solve_damped / solve / linear_solve_work work on an LSMR handle exactly as on
 * a Schur handle; fg_backend_solve is the undamped identity-preconditioned
 * solve of Lsmr::solve (src/lsmr.rs:500-520). The fg_schur_* extras do not
 * apply to it (FG_INVALID_OPTIONS). */

/* src/lsmr.rs:306-337 public fields, plus device-side choices. */
typedef struct {
  size_t max_iterations;        /* inner iterations per solve, > 0; default 1000 */
  double relative_tolerance;    /* in [0,1); default max(1e-10, 128 eps_f64); the reference's
                                   f32 backend defaults to max(1e-10, 128 eps_f32) */
  int diagonal_preconditioning; /* scale by column norms; default 1 */
  int block_preconditioning;    /* variable-block Jacobi (implies scaling); default 0 */
  int collect_timings;          /* default 0 */
  int precision;                /* fg_precision: storage of J and the row vector; default F64 */
  int device;                   /* CUDA device ordinal; default 0 */
} fg_lsmr_options;

/* src/lsmr.rs:68-104 LsmrDiagnostics (has_* = Some). termination uses
 * fg_termination: NONE, CONVERGED, ITERATION_LIMIT or NONFINITE. */
typedef struct {
  int termination;
  size_t iterations;
  int finite_step;
  double estimated_absolute_residual, estimated_relative_residual;
  double original_absolute_residual, original_relative_residual;
  double scaled_absolute_residual, scaled_relative_residual;
  double min_scale, max_scale, damping;
  size_t block_fallbacks;
  int has_estimated, has_original, has_scaled, has_scales, has_damping;
} fg_lsmr_diagnostics;

/* src/lsmr.rs:38-56 LsmrTimings, seconds of device event time. forward covers
 * the row pass, transpose the column-segment pass (with M^T), preconditioner
 * the update pass (with M). */
typedef struct {
  double preparation, factorization, linear_solve, forward, transpose, preconditioner, residual_checks;
} fg_lsmr_timings;

FG_API void fg_lsmr_default_options(fg_lsmr_options* out);
/* Lsmr::default (src/lsmr.rs:339-362) */
FG_API fg_status fg_lsmr_create(const fg_lsmr_options* options, fg_backend** out);
/* Assign the public fields between calls (src/lsmr.rs:306-323); a changed
 * preconditioning mode needs a new prepare_damping before solve_damped. */
FG_API fg_status fg_lsmr_set_options(fg_backend* backend, const fg_lsmr_options* options);
/* Lsmr::diagnostics / Lsmr::timings (src/lsmr.rs:370-383) */
FG_API fg_status fg_lsmr_get_diagnostics(const fg_backend* backend, fg_lsmr_diagnostics* out);
FG_API fg_status fg_lsmr_get_timings(const fg_backend* backend, fg_lsmr_timings* out);
/* The Damped operator of src/lsmr.rs:128-224 on the device at `lambda`:
 * fwd[rows+n] = A x and tr[n] = A^T y with A = [J D^-1; sqrt(lambda) I]
 * (scaled != 0) or [J; sqrt(lambda) D]; host vectors; requires prepare_damping. */
FG_API fg_status fg_lsmr_damped_products(fg_backend* backend, double lambda, int scaled, const double* x,
                                         double* fwd, const double* y, double* tr);
/* Mean device time of one LSMR iteration (row pass, segment pass, update)
 * at `lambda` in the prepared mode, over `repetitions` iterations; bytes_out
 * receives the algorithmic bytes of one iteration (Jacobian values read
 * twice, structure indices, row and column vectors). */
FG_API fg_status fg_lsmr_time_iteration(fg_backend* backend, double lambda, size_t repetitions,
                                        double* seconds_per_iteration, double* bytes_out);

/* ---- Device BAL problem: examples/bal/model.rs Frame + Reprojection ------ */
/* Cameras are 9 doubles [w(3), t(3), f, k1, k2], points 3 doubles; observation
 * i links obs_camera[i] and obs_point[i] with pixel obs_pixel[2i..2i+1].
 * Observations are grouped into one Frame batch per camera in insertion order
 * (src/optimization.rs:367-389), which fixes the emission order. */
FG_API fg_status fg_bal_create(size_t cameras, size_t points, size_t observations,
                               const double* camera_params, const double* point_params,
                               const uint32_t* obs_camera, const uint32_t* obs_point,
                               const double* obs_pixel, int device, fg_bal_problem** out);
/* Same, from device-resident arrays (device pointers on `device`). */
FG_API fg_status fg_bal_create_device(size_t cameras, size_t points, size_t observations,
                                      const double* camera_params, const double* point_params,
                                      const uint32_t* obs_camera, const uint32_t* obs_point,
                                      const double* obs_pixel, int device, fg_bal_problem** out);
FG_API void fg_bal_destroy(fg_bal_problem* problem);
FG_API fg_status fg_bal_set_parameters(fg_bal_problem* problem, const double* camera_params,
                                       const double* point_params);
FG_API fg_status fg_bal_get_parameters(fg_bal_problem* problem, double* camera_params,
                                       double* point_params);
/* Frame::cost summed over frames (examples/bal/model.rs:201-213, src/optimization.rs:419-430) */
FG_API fg_status fg_bal_cost(fg_bal_problem* problem, double* cost);
/* No counterpart in the reference. The BAL objective (as fg_bal_cost) for
 * callers that cannot let the library allocate device memory: every input and
 * the output are caller-owned device pointers on `device`, and the scratch is a
 * fixed file-scope device array (about 2.4 MB per GPU, held until exit).
 * out[0] = cost, out[1] = 1 if any projection was invalid or an observation
 * index was out of range. Enqueued on `stream` (a cudaStream_t, NULL = the
 * legacy default stream); the result is ready when the stream reaches it.
 * At most 16384 cameras (else FG_INVALID_OPTIONS). Calls share the scratch:
 * calls that overlap on the GPU race and must be serialized by the caller. */
FG_API fg_status fg_bal_cost_noalloc(size_t cameras, size_t points, size_t observations,
                                     const double* camera_params, const double* point_params,
                                     const uint32_t* obs_camera, const uint32_t* obs_point,
                                     const double* obs_pixel, double* out, int device, void* stream);
/* A homogeneous batch of factor emissions straight from device memory, for
 * factor families other than BAL (src/optimization.rs:541-612 CheckedSink +
 * src/linear_model.rs:180-210 LinearizedModel::accumulate + src/schur.rs:438-482
 * Schur::accumulate, for `count` emissions at once instead of one host call
 * each). Every emission has `rows` rows (1..16), one retained block (the
 * retained variable retained_variable[k], width = the backend's retained block
 * width) and one eliminated block (eliminated_variable[k], the eliminated
 * width); variables are numbered within their partition (coordinate offset =
 * index x width, eliminated ones after the retained dimension). Device arrays,
 * SoA: residual[i * count + k]; block element (i, j) of emission k at
 * retained_jacobian[(j * rows + i) * count + k] and
 * eliminated_jacobian[(j * rows + i) * count + k]. Batches after the last
 * fg_backend_clear (or prepare) append in call order; they cannot be mixed
 * with fg_backend_accumulate in one linearization. The packed values, index
 * maps (blocks, edges, variables) and emission order equal those of the same
 * emissions passed to fg_backend_accumulate one by one. Errors:
 * FG_INVALID_EMISSION for a variable outside the layout, FG_INVALID_EVALUATION
 * for a nonfinite value, FG_DIMENSION_MISMATCH for rows outside 1..16; the
 * failing batch is dropped. Schur backends only. */
FG_API fg_status fg_schur_accumulate_pairs_device(fg_backend* backend, size_t count, size_t rows,
                                                  const uint32_t* retained_variable,
                                                  const uint32_t* eliminated_variable, const double* residual,
                                                  const double* retained_jacobian,
                                                  const double* eliminated_jacobian);
/* Workspace::linearize for BAL frames (src/optimization.rs:229-265 +
 * examples/bal/model.rs:214-236): residuals and Jacobians straight into the
 * backend's block storage, in emission order. */
FG_API fg_status fg_bal_linearize(fg_bal_problem* problem, fg_backend* backend);

/* ---- Optimizers (src/optimization/levenberg_marquardt.rs, gauss_newton.rs) ---- */
/* src/optimization.rs:40-84 */
typedef struct {
  size_t max_iterations;
  double gradient_tolerance, step_tolerance, cost_tolerance;
} fg_optimize_options;
/* src/optimization/levenberg_marquardt.rs:17-46 */
typedef struct {
  double initial_damping, min_damping, max_damping, min_column_norm, acceptance_threshold;
  size_t max_trials;
} fg_lm_options;
/* src/optimization.rs:86-112; termination: 1 NoVariables, 2 GradientTolerance,
 * 3 StepTolerance, 4 CostTolerance */
typedef struct {
  size_t iterations;
  double initial_cost, final_cost;
  int termination;
} fg_optimize_report;
/* LmStatistics + LmWork (levenberg_marquardt.rs:84-173); last_rejection:
 * 0 None, 1 LinearSolve, 2 Prediction, 3 InvalidEvaluation, 4 PoorAgreement */
typedef struct {
  size_t linearizations, attempts, rejected_steps, accepted_steps, cost_evaluations;
  double damping, cost, gradient_norm, step_norm;
  int has_cost, has_gradient_norm, has_step_norm, last_rejection;
  size_t linear_solves, linear_iterations;
  int linear_work_available;
} fg_lm_statistics;
/* on_accept observer (levenberg_marquardt.rs:208-210) */
typedef void (*fg_accept_callback)(void* user, const fg_lm_statistics* statistics);

FG_API void fg_optimize_default_options(fg_optimize_options* out);
FG_API void fg_lm_default_options(fg_lm_options* out);

/* LevenbergMarquardt::solve_batch_with_outcome on a device BAL problem. */
FG_API fg_status fg_lm_solve_bal(fg_backend* backend, fg_bal_problem* problem,
                                 const fg_optimize_options* options, const fg_lm_options* lm_options,
                                 fg_optimize_report* report, fg_lm_statistics* statistics,
                                 fg_accept_callback on_accept, void* user);
/* Same LM, additionally stopping (termination 5, "CostTarget") as soon as an
 * accepted cost is <= target_cost: the time-to-cost measurement of
 * examples/bal.rs:14-34 (which records when the accepted cost first crosses a
 * fraction of the initial cost) turned into a stop. */
FG_API fg_status fg_lm_solve_bal_to_cost(fg_backend* backend, fg_bal_problem* problem,
                                         const fg_optimize_options* options, const fg_lm_options* lm_options,
                                         double target_cost, fg_optimize_report* report,
                                         fg_lm_statistics* statistics);
/* Reset the device parameters to the values the problem was created with. */
FG_API fg_status fg_bal_restore_initial(fg_bal_problem* problem);
/* Mean device time (CUDA events on the library stream) of one application of
 * the reduced operator at `lambda`, over `repetitions` back-to-back calls;
 * requires prepare_damping. bytes_out receives the algorithmic bytes one
 * application must move (cross blocks, indices, point factors, camera Gram
 * blocks, input and output vectors). */
FG_API fg_status fg_schur_time_operator(fg_backend* backend, double lambda, size_t repetitions,
                                        double* seconds_per_apply, double* bytes_out);
/* The single-pass operator kernel alone (BAL-shaped systems on the fast path):
 * mean device time of one launch over `repetitions` back-to-back launches
 * (CUDA events on the library stream), and the algorithmic bytes it must move (cross blocks and indices,
 * point factors, x in, the camera sums out once; not the camera Gram blocks,
 * which the reduction step reads). FG_UNSUPPORTED_STRUCTURE without the fast
 * path. */
FG_API fg_status fg_schur_time_operator_kernel(fg_backend* backend, double lambda, size_t repetitions,
                                               double* seconds_per_launch, double* bytes_out);

/* The reduced-operator implementation the autotuner chose for the current
 * structure: 0 generic (any widths), 1 per-warp TMA-ring single pass (the only
 * one for more cameras than one SM's shared memory holds, or points with more
 * than 32 observations), 2 direct-load single pass, 3 prefetching direct-load
 * single pass, 4 TMA-staged stage groups; seconds4[v-1] (may be NULL) =
 * measured time per application of variant v (0 if not measured or not
 * applicable). */
FG_API fg_status fg_schur_operator_info(fg_backend* backend, int* variant, double* seconds4);
/* Test hook (no reference counterpart): the number of polls after which the
 * ring operator's consumer wait on a shared-memory slot gives up; the kernel
 * then drains its copies in flight (with the full limit), raises the error
 * flag and the solve returns FG_DEVICE_TIMEOUT. 0 restores the default
 * (4,194,304 polls). */
FG_API fg_status fg_schur_set_poll_limit(fg_backend* backend, unsigned polls);

/* ---- Learned preconditioner (no reference counterpart) ----------------------
 * A message-passing network over the camera covisibility graph of the reduced
 * camera system. Per retained variable c it emits A_c = I + 0.1 tril(O_c) and
 * the preconditioner block M_c = L_c^-T (A_c A_c^T + 1e-3 I) L_c^-1, where
 * L_c L_c^T = B_c + lambda I is the block-Jacobi factor of src/schur.rs:658-682,
 * so M is SPD and an untrained network (zero output layer) is block-Jacobi.
 * Node features: P_c = L_c^-1 (sum_e E_e C_p^-1 E_e^T) L_c^-T (45 entries),
 * degree, coupling, log10(lambda), trace(P_c); covisibility weights
 * s_ij = sqrt(sum_shared p ||G_ip G_jp^T||_F^2), G_e = L_c^-1 E_e L_p^-T,
 * row-normalized. Three layers h_l = h_{l-1} + relu([h_{l-1}, A h_{l-1}] W_l + b_l),
 * hidden width 64; BF16 weights and operands, FP32 accumulation (tensor cores).
 * Training systems are reduced camera systems of an attached Schur backend;
 * the loss is mean ||x - M_hat S_hat x||^2 over Gaussian whitened probes x.
 * Supports retained widths <= 9, eliminated widths <= 4, <= 16384 retained
 * variables. Handles are not thread safe. */
FG_API fg_status fg_gnn_create(uint64_t seed, int device, fg_gnn** out);
FG_API void fg_gnn_destroy(fg_gnn* gnn);
/* Parameters are FP32 masters, flat: W_in (64x64, row = input), b_in (64),
 * {W_l (128x64), b_l (64)} for l = 1..3, W_out (64x64), b_out (64). */
FG_API fg_status fg_gnn_parameter_count(const fg_gnn* gnn, size_t* count);
FG_API fg_status fg_gnn_get_parameters(fg_gnn* gnn, float* out);
/* Replaces the parameters and resets the Adam state. */
FG_API fg_status fg_gnn_set_parameters(fg_gnn* gnn, const float* parameters);
/* Captures the reduced camera system of a Schur backend (after
 * prepare_damping) at `lambda` as a training system with `probes` probe
 * pairs in whitened coordinates: kind 0 draws x Gaussian and applies
 * y = S_hat x; kind 1 draws y Gaussian and solves S_hat x = y with the
 * backend's block-Jacobi PCG (work counters untouched). index receives its
 * position. */
FG_API fg_status fg_schur_capture_system(fg_backend* schur, fg_gnn* gnn, double lambda, size_t probes,
                                         uint64_t seed, int kind, size_t* index);
/* A training system from host arrays: features C x 64, adjacency C x C
 * (rounded to bf16), probes K x C x width for x and y = S_hat x, mask C. */
FG_API fg_status fg_gnn_import_system(fg_gnn* gnn, size_t cameras, size_t width, size_t probes,
                                      const float* features, const float* adjacency, const float* probe_x,
                                      const float* probe_y, const uint8_t* mask, size_t* index);
FG_API fg_status fg_gnn_system_count(const fg_gnn* gnn, size_t* count);
FG_API fg_status fg_gnn_system_size(const fg_gnn* gnn, size_t index, size_t* cameras, size_t* width,
                                    size_t* probes);
/* Copies a system back (any pointer may be NULL); adjacency as float. */
FG_API fg_status fg_gnn_export_system(fg_gnn* gnn, size_t index, float* features, float* adjacency,
                                      float* probe_x, float* probe_y, uint8_t* mask, double* damping);
FG_API fg_status fg_gnn_clear_systems(fg_gnn* gnn);
/* Loss of one system; when gradient (parameter_count floats) is non-NULL also
 * the backward pass, and outputs (C x 64) receives the network output O. */
FG_API fg_status fg_gnn_evaluate(fg_gnn* gnn, size_t index, double* loss, float* gradient, float* outputs);
/* `steps` Adam steps (beta 0.9 / 0.999), one captured system per step in a
 * shuffled cycle; mean_loss = mean loss over the steps (before each update). */
FG_API fg_status fg_gnn_train(fg_gnn* gnn, size_t steps, double learning_rate, double* mean_loss);
/* Attaches (or, with NULL, detaches) the network used by FG_PRECOND_LEARNED.
 * The backend keeps a pointer: the network must outlive the attachment.
 * Attaching re-arms the one-time block-Jacobi comparison. */
FG_API fg_status fg_schur_attach_learned(fg_backend* schur, fg_gnn* gnn);

/* ---- Dense direct backends on the same LeastSquaresBackend entry points ----
 * fg_backend_prepare / clear / accumulate / gradient_norm / prepare_damping /
 * solve_damped / solve and fg_backend_destroy drive them like the sparse
 * backends. Systems are factored by one thread block: they are meant for
 * bounded windows (a few thousand coordinates), as in the reference. */
/* DenseNormalCholesky::default (src/normal.rs:22-63); solve() factors in place
 * (a later prepare_damping needs a fresh model, normal.rs:154-160). */
FG_API fg_status fg_dense_normal_create(int device, fg_backend** out);
/* DenseSchur::new(retained_dimension, eliminated_widths) (src/dense_schur.rs:63-90) */
FG_API fg_status fg_dense_schur_create(size_t retained_dimension, const size_t* eliminated_widths,
                                       size_t count, int device, fg_backend** out);
/* DenseQr { relative_rank_tolerance, .. } (src/qr.rs:24-63) */
FG_API fg_status fg_dense_qr_create(double relative_rank_tolerance, int device, fg_backend** out);
FG_API fg_status fg_dense_qr_set_tolerance(fg_backend* backend, double relative_rank_tolerance);
/* CovarianceBackend::covariance (src/covariance.rs:263-270) + SelectedCovariance
 * (:225-255) for a backend's current model: out (k x k, column-major) = the
 * selected block of the undamped inverse information, columns in selection
 * order; relative_pivot_tolerance is CovarianceOptions' (default 64 eps).
 * DenseSchur accepts retained columns only. Schur and LSMR handles replay their
 * cached Jacobian into a device DenseNormalCholesky first, as both delegate to
 * LinearizedModel::covariance (src/schur.rs:548-556, src/lsmr.rs:598-604,
 * src/linear_model.rs:122-167); that needs the dense n x n normal matrix. */
FG_API fg_status fg_backend_covariance(fg_backend* backend, const size_t* columns, size_t k,
                                       double relative_pivot_tolerance, double* out);

/* ---- Batched pose-graph windows ----------------------------------------
 * Thousands of independent SE(3) windows of uneven size solved in one
 * persistent launch. Window w owns poses [pose_offset[w], pose_offset[w+1])
 * (7 doubles each: qw qx qy qz tx ty tz) and relative-pose factors
 * [rel_offset[w], rel_offset[w+1]) between window-local poses (i, j) with
 * measurement z (7 doubles): r = Log(z^-1 x_i^-1 x_j), Jacobians from
 * examples/slam/geometry.rs (log_jacobian, adjoint). Pose 0 of every window
 * carries an anchor PosePrior (examples/slam.rs:26-56). Each window is solved
 * by LevenbergMarquardt (levenberg_marquardt.rs:330-472) over an all-retained
 * DenseSchur (src/dense_schur.rs) with dense Cholesky, then its oldest
 * `removed_poses` poses are eliminated by the square-root reduction of
 * src/marginalization.rs:458-513 into a prior (A, b, constant) on its
 * separator poses (touched poses >= removed_poses, increasing). */
typedef struct {
  int status;      /* fg_status of the window's LM: FG_OK, FG_NO_PROGRESS, FG_NO_CONVERGENCE, ... */
  int termination; /* when FG_OK: 2 GradientTolerance, 3 StepTolerance, 4 CostTolerance */
  size_t iterations, linearizations, attempts, rejected_steps, cost_evaluations;
  int last_rejection; /* 0 None, 1 LinearSolve, 2 Prediction, 3 InvalidEvaluation, 4 PoorAgreement */
  double initial_cost, final_cost, damping, gradient_norm, step_norm;
  int prior_status; /* fg_status of the elimination */
  size_t prior_rows, eliminated_rank, separator_poses;
  double prior_constant;
} fg_window_report;
typedef struct fg_windows fg_windows;
/* precision: FG_PRECISION_F64 or FG_PRECISION_F32_REFINED (FP32 Cholesky,
 * FP64 normal matrix, gradient, cost and two FP64 refinement passes per solve). */
FG_API fg_status fg_windows_create(size_t windows, const uint64_t* pose_offset, const uint64_t* rel_offset,
                                   const uint32_t* rel_ij, size_t removed_poses, int precision, int device,
                                   fg_windows** out);
FG_API void fg_windows_destroy(fg_windows* batch);
/* Output layout of the priors (windows + 1 entries each): window w's separator
 * poses are separators[separator_offset[w] .. separator_offset[w+1]) (window-
 * local indices); its A is a column-major prior_rows x (6 * separator poses)
 * matrix at a_offset[w] and its b starts at 6 * separator_offset[w]. */
FG_API fg_status fg_windows_prior_layout(const fg_windows* batch, uint64_t* separator_offset,
                                         uint64_t* a_offset, uint32_t* separators);
/* Replace every window's anchor prior by a general prior on its first
 * prior_poses[w] poses (1 to min(64, window poses)) with prior_rows[w] rows
 * (1 to 384): r = b + sum_i A_i Log(ref_i^-1 x_i), J_i = A_i Jr^-1(Log(ref_i^-1
 * x_i)), the prior that Priors::update (src/marginalization.rs:157-231) feeds
 * into the next solve of a chained window. Per window, concatenated in window
 * order: A (prior_rows x 6 prior_poses, column-major — the layout
 * fg_windows_download writes prior_a in, packed to prior_rows rows), b
 * (prior_rows) and refs (7 per prior pose). The anchor is the case s = 1, A = I,
 * b = 0, ref = the anchor pose, with the same results bit for bit. The priors
 * argument of fg_windows_upload / fg_windows_solve is ignored after this call.
 * Rejects nonfinite A or b (FG_INVALID_EVALUATION) and out-of-range shapes
 * (FG_DIMENSION_MISMATCH), keeping the previous priors. */
FG_API fg_status fg_windows_set_priors(fg_windows* batch, const uint32_t* prior_poses, const uint32_t* prior_rows,
                                       const double* A, const double* b, const double* refs);
/* Host -> device inputs, the device-only solve, device -> host results. */
FG_API fg_status fg_windows_upload(fg_windows* batch, const double* poses, const double* priors,
                                   const double* rel_z);
FG_API fg_status fg_windows_run(fg_windows* batch, const fg_optimize_options* options,
                                const fg_lm_options* lm_options);
FG_API fg_status fg_windows_download(fg_windows* batch, double* poses, fg_window_report* reports,
                                     double* prior_a, double* prior_b);
/* upload + run + download; poses are updated in place. */
FG_API fg_status fg_windows_solve(fg_windows* batch, double* poses, const double* priors, const double* rel_z,
                                  const fg_optimize_options* options, const fg_lm_options* lm_options,
                                  fg_window_report* reports, double* prior_a, double* prior_b);
/* The autotuner's choice (panel width 16 or 32, CTAs per SM) and its sample
 * timings in ms for {32/1, 32/2, 16/2, 16/3} (0 = not run or not resident). */
FG_API fg_status fg_windows_tuning(const fg_windows* batch, int* panel, int* ctas_per_sm, double* ms4);
FG_API fg_status fg_windows_stream(const fg_windows* batch, void** stream);

/* GaussNewton::solve_batch on a device BAL problem. */
FG_API fg_status fg_gn_solve_bal(fg_backend* backend, fg_bal_problem* problem,
                                 const fg_optimize_options* options, fg_optimize_report* report);

/* Host-evaluated problems (any factor family): additive real coordinates of
 * the given dimension; the caller evaluates cost at x and emits each residual
 * through fg_backend_accumulate on the backend it is handed. */
typedef struct {
  size_t dimension;
  int (*cost)(void* user, const double* x, double* out);
  int (*linearize)(void* user, const double* x, fg_backend* backend);
} fg_problem_callbacks;
FG_API fg_status fg_lm_optimize(fg_backend* backend, const fg_problem_callbacks* problem, void* user,
                                double* x, const fg_optimize_options* options,
                                const fg_lm_options* lm_options, fg_optimize_report* report,
                                fg_lm_statistics* statistics);
FG_API fg_status fg_gn_optimize(fg_backend* backend, const fg_problem_callbacks* problem, void* user,
                                double* x, const fg_optimize_options* options,
                                fg_optimize_report* report);

#endif /* FAGRA_B200_H */
