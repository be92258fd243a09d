// Nonlinear optimizer drivers (host) over the backend interface.
#pragma once
#include "common.cuh"
#include "schur.cuh"
#include "bal.cuh"

namespace fg {

// What the optimizers need from a problem: the Layout dimension, cost at the
// accepted or staged state, linearization into the backend, and the
// Stage/Accept/Reject transaction (src/optimization.rs:419-487).
struct ProblemAdapter {
  virtual ~ProblemAdapter() {}
  virtual size_t dimension() = 0;
  virtual fg_status cost(bool trial, double* out) = 0;
  virtual fg_status linearize(Backend* b) = 0;
  virtual bool device_steps() const = 0;  // stage() takes a device pointer
  virtual fg_status stage(const double* delta) = 0;
  virtual void accept() = 0;
  virtual void reject() = 0;
  // Device trials: stage the device step and evaluate the trial cost without
  // a host round trip, leaving [cost, invalid flag] at *result (device).
  virtual bool device_trials() const { return false; }
  virtual fg_status stage_and_cost_device(const double*, const double** result) {
    *result = nullptr;
    return FG_UNSUPPORTED_STRUCTURE;
  }
};

// One LM trial decided on the device (levenberg_marquardt.rs:388-467): the
// step's infinity norm, the trial cost, the gain ratio, acceptance, the
// stagnation test and the damping update, read back by the host in one copy.
struct LmTrialState {
  double current, lambda, growth, predicted;  // in (predicted from the backend's verification)
  double norm, value, actual, ratio;          // step norm, trial cost
  int norm_bad, accepted, rejection, stalled, stop;
};

fg_status lm_optimize(Backend* b, ProblemAdapter& pb, const fg_optimize_options& opt, const fg_lm_options& lo,
                      fg_optimize_report* rep, fg_lm_statistics* st, fg_accept_callback on_accept, void* user,
                      double target_cost = -1.0);
fg_status gn_optimize(Backend* b, ProblemAdapter& pb, const fg_optimize_options& opt, fg_optimize_report* rep);
fg_status lm_solve_bal(Backend* b, BalProblem* p, const fg_optimize_options& o, const fg_lm_options& lo,
                       fg_optimize_report* rep, fg_lm_statistics* st, fg_accept_callback cb, void* user,
                       double target_cost = -1.0);
fg_status gn_solve_bal(Backend* b, BalProblem* p, const fg_optimize_options& o, fg_optimize_report* rep);
fg_status lm_callbacks(Backend* b, const fg_problem_callbacks* cb, void* user, double* x,
                       const fg_optimize_options& o, const fg_lm_options& lo, fg_optimize_report* rep,
                       fg_lm_statistics* st);
fg_status gn_callbacks(Backend* b, const fg_problem_callbacks* cb, void* user, double* x,
                       const fg_optimize_options& o, fg_optimize_report* rep);

}  // namespace fg
