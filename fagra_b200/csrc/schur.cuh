// Device Schur backend: the GPU implementation of fagra's `Schur` linear
// backend (src/schur.rs) over a block-sparse linearization (src/linear_model.rs).
#pragma once
#include "common.cuh"
#include <functional>

namespace fg {

// Jacobian block in the reference layout (src/linear_model.rs:12-19).
struct DBlockMeta {
  int64_t row, start, col;
  int32_t rows, cols;
};
// Schur edge (src/schur.rs:93-99) with partition-local variable indices.
struct DEdgeMeta {
  int32_t cam, pt;  // retained / eliminated variable index
  int64_t lblk, rblk;
};
struct HostBlock {
  size_t row, col, rows, cols, start;
};
// Observations of a device BAL problem in emission order: one Frame batch per
// camera (examples/bal/model.rs:187-200), factors in insertion order.
struct BalObservations {
  uint64_t problem_id = 0;
  size_t cameras = 0, points = 0, observations = 0;
  const uint32_t* cam = nullptr;  // device: camera of each emission (nondecreasing)
  const uint32_t* pt = nullptr;   // device: point of each emission
  // Host copies of cam and pt, downloaded on first use.
  std::function<fg_status(const uint32_t**, const uint32_t**)> host;
};
struct HostEdge {
  size_t retained, eliminated, lblk, rblk;  // column offsets (partition local) + block ids
};

// PCG / verification scalars living on the device (one per backend).
struct PcgState {
  double rz, pq, alpha, beta, rr, bnorm, threshold, lambda;
  double rz_new, rr_last, delta2;
  int done, termination;   // done: 0 running, 1 finished, 2 awaiting the FP64 residual verdict
  int replace;             // 1: an FP64 residual replacement is due
  unsigned iterations, max_iterations, replacements;
  unsigned counter0, counter1, counter2, counter3;
  // two-level preconditioner: c = G W^T r of the last z update, pending until
  // k_coarse_add has added W c to z
  double coarse[8];
  int coarse_pending;
  unsigned counter4;
  unsigned trips;  // loop trips of the single-launch PCG graph (k_pcg_continue)
};
struct VerifyState {
  double jd2;        // ||J delta||^2
  double gd;         // g . delta
  double nr2, g2;    // ||normal residual||^2, ||g||^2 (original coordinates)
  double snr2, sg2;  // scaled by 1/D
  double red2, rhs2; // ||S z - b||^2, ||b||^2
  int nonfinite_step;
  unsigned counter0, counter1, pad;
};

// A linearized model on the host in the reference layout (src/linear_model.rs:
// 12-19, 95-105): Jacobian blocks {row, col, rows, cols, start} in emission
// order, column-major values, and -r.
struct HostModel {
  size_t rows = 0, cols = 0;
  std::vector<HostBlock> blocks;
  std::vector<double> values, negres;
};

class Backend {
 public:
  virtual ~Backend() {}
  virtual int kind() const = 0;  // 0 Schur, 1 LSMR
  virtual fg_status prepare(size_t dimension) = 0;
  virtual fg_status clear() = 0;
  virtual fg_status accumulate(size_t rows, const double* r, size_t nb, const size_t* cols, const size_t* widths,
                               const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) = 0;
  virtual fg_status gradient_norm(double* out) = 0;
  virtual fg_status prepare_damping(double floor) = 0;
  virtual fg_status solve_damped(double lambda, double* predicted, bool copy_to_host) = 0;
  // LeastSquaresBackend::solve: Schur runs prepare_damping(1e-6) + solve_damped(0)
  // (src/schur.rs:486-489); LSMR has its own undamped solve.
  virtual fg_status solve_undamped(bool copy_to_host) {
    FG_TRY(prepare_damping(1e-6));
    double p = 0;
    return solve_damped(0.0, &p, copy_to_host);
  }
  virtual fg_status step_norm_inf(double* out) = 0;
  // max |step| and a nonfinite flag written to d_out[0..1] on the device,
  // without a host synchronization (backends that cannot return unsupported)
  virtual fg_status step_norm_async(double* /*d_out*/) { return FG_UNSUPPORTED_STRUCTURE; }
  virtual const double* step_host() const = 0;
  virtual const double* step_device() const = 0;
  virtual size_t dimension() const = 0;
  virtual void work(size_t* solves, size_t* iterations) const = 0;
  // Device BAL path: bind an implicit BAL structure and expose raw model storage.
  virtual fg_status bind_bal(const BalObservations& obs) = 0;
  virtual void* values_device() = 0;   // T*, packed Jacobian values
  virtual double* negres_device() = 0;  // -r
  virtual bool is_f32() const = 0;
  virtual void mark_device_model(size_t rows) = 0;
  virtual int device() const = 0;
  virtual cudaStream_t stream() const = 0;

  // The current linearization as a host model (Schur and LSMR), for the
  // covariance both delegate to LinearizedModel::covariance (src/schur.rs:548-556,
  // src/lsmr.rs:598-604).
  virtual fg_status model_host(HostModel*) {
    set_error("this backend keeps no linearized model");
    return FG_UNSUPPORTED_STRUCTURE;
  }
  // A device problem's coarse basis for two-level PCG (k vectors of the
  // retained length, row j at basis + j * retained, unscaled coordinates);
  // backends that do not use one ignore it.
  virtual fg_status set_coarse_basis(const double*, int) { return FG_OK; }
  // Schur-only extras.
  virtual fg_status set_options(const fg_schur_options&) { return not_schur(); }
  virtual void diagnostics(fg_schur_diagnostics* d) const { *d = fg_schur_diagnostics{}; }
  virtual void timings(fg_schur_timings* t) const { *t = fg_schur_timings{}; }
  virtual fg_status structure_sizes(size_t*, size_t*, size_t*, size_t*, size_t*, size_t*) { return not_schur(); }
  virtual fg_status export_structure(uint64_t*, uint64_t*, uint64_t*, uint64_t*) { return not_schur(); }
  virtual fg_status export_model(double*, double*, double*, double*, double*, double*) { return not_schur(); }
  virtual fg_status reduced_apply(double, const double*, double*) { return not_schur(); }
  virtual fg_status time_operator(double, size_t, double*, double*) { return not_schur(); }
  virtual fg_status time_operator_kernel(double, size_t, double*, double*) { return not_schur(); }
  virtual fg_status attach_learned(fg_gnn*) { return not_schur(); }
  virtual fg_status capture_system(fg_gnn*, double, size_t, uint64_t, int, size_t*) { return not_schur(); }
  virtual void operator_info(int* variant, double* seconds4) const {
    *variant = 0;
    if (seconds4) seconds4[0] = seconds4[1] = seconds4[2] = seconds4[3] = 0;
  }
  virtual fg_status set_poll_limit(unsigned) { return not_schur(); }
  virtual fg_status accumulate_pairs(size_t, size_t, const uint32_t*, const uint32_t*, const double*, const double*,
                                     const double*) {
    return not_schur();
  }
  // LSMR-only extras.
  virtual fg_status set_lsmr_options(const fg_lsmr_options&) { return not_lsmr(); }
  virtual void lsmr_diagnostics(fg_lsmr_diagnostics* d) const { *d = fg_lsmr_diagnostics{}; }
  virtual void lsmr_timings(fg_lsmr_timings* t) const { *t = fg_lsmr_timings{}; }
  virtual fg_status damped_products(double, int, const double*, double*, const double*, double*) {
    return not_lsmr();
  }
  virtual fg_status time_iteration(double, size_t, double*, double*) { return not_lsmr(); }

 protected:
  static fg_status not_schur() {
    set_error("not a Schur backend");
    return FG_INVALID_OPTIONS;
  }
  static fg_status not_lsmr() {
    set_error("not an LSMR backend");
    return FG_INVALID_OPTIONS;
  }
};

fg_status make_schur(size_t retained, size_t cw, size_t pw, const fg_schur_options& o, Backend** out);
fg_status make_lsmr(const fg_lsmr_options& o, Backend** out);

}  // namespace fg

struct fg_backend {
  fg::Backend* impl;
};
