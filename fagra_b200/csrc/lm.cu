// Levenberg–Marquardt and Gauss–Newton drivers over the device backend.
// They restate src/optimization/levenberg_marquardt.rs:330-472 and
// src/optimization/gauss_newton.rs:101-176 statement for statement; the
// problem side is either the device BAL problem or host callbacks.
#include "lm.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

namespace fg {

namespace {

fg_status validate(const fg_optimize_options& o) {  // src/optimization.rs:69-84
  double v[3] = {o.gradient_tolerance, o.step_tolerance, o.cost_tolerance};
  if (o.max_iterations == 0) return FG_INVALID_OPTIONS;
  for (double x : v)
    if (!std::isfinite(x) || x < 0) return FG_INVALID_OPTIONS;
  return FG_OK;
}
fg_status validate(const fg_lm_options& o) {  // levenberg_marquardt.rs:47-67
  double v[5] = {o.initial_damping, o.min_damping, o.max_damping, o.min_column_norm, o.acceptance_threshold};
  if (o.max_trials == 0) return FG_INVALID_OPTIONS;
  for (double x : v)
    if (!std::isfinite(x) || x <= 0) return FG_INVALID_OPTIONS;
  if (o.min_damping > o.initial_damping || o.initial_damping > o.max_damping || o.acceptance_threshold >= 1)
    return FG_INVALID_OPTIONS;
  return FG_OK;
}

// Device BAL problem adapter.
struct BalAdapter : ProblemAdapter {
  BalProblem* p;
  explicit BalAdapter(BalProblem* pr) : p(pr) {}
  size_t dimension() override { return p->dimension(); }
  fg_status cost(bool trial, double* out) override { return p->cost(trial, out); }
  fg_status linearize(Backend* b) override { return p->linearize(b); }
  bool device_steps() const override { return true; }
  fg_status stage(const double* delta) override { return p->stage(delta); }
  void accept() override { p->accept(); }
  void reject() override { p->reject(); }
  bool device_trials() const override { return true; }
  fg_status stage_and_cost_device(const double* d_delta, const double** result) override {
    FG_TRY(p->stage_and_cost_device(d_delta));
    *result = p->result.get();
    return FG_OK;
  }
};

// The decision of one LM trial on the device, statement for statement as the
// host loop below (levenberg_marquardt.rs:406-467): gain ratio clamped at 2,
// acceptance, stagnation, Nielsen's damping update, or the growth after a
// rejection. Products are rounded one at a time (no fused multiply-add), so
// the damping sequence is the host loop's bit for bit.
__global__ void k_lm_decide(LmTrialState* s, const double* norm, const double* result, fg_lm_options lo,
                            double step_tolerance, double cost_tolerance, int undamped) {
  LmTrialState t = *s;
  t.norm = norm[0];
  t.norm_bad = norm[1] != 0 || !isfinite(norm[0]);
  t.accepted = t.rejection = t.stalled = t.stop = 0;
  if (t.norm_bad) {
    *s = t;
    return;
  }
  if (!isfinite(t.predicted) || t.predicted <= 0) {
    t.rejection = 2;
  } else {
    t.value = result[0];
    if (result[1] != 0 || !isfinite(t.value) || t.value < 0) {  // checked_cost
      t.rejection = 3;
    } else {
      t.actual = __dsub_rn(t.current, t.value);
      t.ratio = fmin(__ddiv_rn(t.actual, t.predicted), 2.0);
      if (t.actual > 0 && t.ratio >= lo.acceptance_threshold) {
        t.accepted = 1;
        t.stalled = step_tolerance > 0 && t.norm <= step_tolerance &&
                    (cost_tolerance == 0 || __ddiv_rn(t.actual, fmax(t.current, 1.0)) <= cost_tolerance);
        const double c = __dsub_rn(__dmul_rn(2.0, fmin(t.ratio, 1.0)), 1.0);
        const double update = fmax(__dsub_rn(1.0, __dmul_rn(__dmul_rn(c, c), c)), 1.0 / 3.0);
        t.lambda = fmin(fmax(__dmul_rn(t.lambda, update), lo.min_damping), lo.max_damping);
        t.current = t.value;
      } else {
        t.rejection = 4;
      }
    }
  }
  if (!t.accepted) {
    if (undamped || t.lambda == lo.max_damping) {
      t.stop = 1;
    } else {
      t.lambda = fmin(__dmul_rn(t.lambda, t.growth), lo.max_damping);
      t.growth = fmin(__dmul_rn(t.growth, 2.0), fmax(lo.max_damping, 2.0));
    }
  }
  *s = t;
}

// Host callback adapter: additive coordinates owned by the caller.
struct CallbackAdapter : ProblemAdapter {
  const fg_problem_callbacks* cb;
  void* user;
  double* x;
  std::vector<double> tx;
  bool trial = false;
  fg_backend handle{nullptr};
  size_t dimension() override { return cb->dimension; }
  fg_status cost(bool t, double* out) override {
    double c = 0;
    int s = cb->cost(user, t ? tx.data() : x, &c);
    if (s) return (fg_status)s;
    if (!std::isfinite(c) || c < 0) return FG_INVALID_EVALUATION;  // checked_cost
    *out = c;
    return FG_OK;
  }
  fg_status linearize(Backend* b) override {
    FG_TRY(b->clear());
    handle.impl = b;
    return (fg_status)cb->linearize(user, x, &handle);
  }
  bool device_steps() const override { return false; }
  fg_status stage(const double* d) override {
    tx.resize(cb->dimension);
    for (size_t i = 0; i < cb->dimension; ++i) tx[i] = x[i] + d[i];
    trial = true;
    return FG_OK;
  }
  void accept() override {
    if (trial) {
      std::copy(tx.begin(), tx.end(), x);
      trial = false;
    }
  }
  void reject() override { trial = false; }
};

void record_work(Backend* b, fg_lm_statistics* st) {
  size_t s = 0, i = 0;
  b->work(&s, &i);
  st->linear_solves = s;
  st->linear_iterations = i;
  st->linear_work_available = 1;
}

}  // namespace

fg_status lm_optimize(Backend* b, ProblemAdapter& pb, const fg_optimize_options& opt, const fg_lm_options& lo,
                      fg_optimize_report* rep, fg_lm_statistics* st, fg_accept_callback on_accept, void* user,
                      double target_cost) {
  *st = fg_lm_statistics{};
  st->linear_work_available = 1;
  FG_TRY(validate(opt));
  FG_TRY(validate(lo));
  double lambda = lo.initial_damping;
  st->damping = lambda;
  FG_TRY(b->prepare(pb.dimension()));
  st->cost_evaluations += 1;
  double initial;
  FG_TRY(pb.cost(false, &initial));
  st->cost = initial;
  st->has_cost = 1;
  double current = initial;
  bool stalled = false, tried_undamped = false;
  rep->initial_cost = initial;
  auto finish = [&](int term) {
    rep->final_cost = current;
    rep->iterations = st->accepted_steps;
    rep->termination = term;
    record_work(b, st);
    return FG_OK;
  };
  auto fail = [&](fg_status s) {
    record_work(b, st);
    return s;
  };
  const bool dev = pb.device_steps();
  // device trials: a device problem and a backend that reduces its step norm
  // on the device; the state lives in the problem's buffers
  constexpr size_t LMW = (sizeof(LmTrialState) + sizeof(double) - 1) / sizeof(double);
  double* d_lm = nullptr;
  LmTrialState* h_lm = nullptr;
  BalProblem* bp = nullptr;
  if (pb.device_trials()) {
    bp = static_cast<BalAdapter&>(pb).p;
    FG_TRY(bp->lm_state.resize(LMW + 2));
    FG_TRY(bp->h_lm_state.resize(LMW));
    d_lm = bp->lm_state.get();
    h_lm = reinterpret_cast<LmTrialState*>(bp->h_lm_state.get());
  }
  for (;;) {
    if (pb.dimension() == 0) return finish(1);
    st->linearizations += 1;
    fg_status s = pb.linearize(b);
    if (s) return fail(s);
    double g;
    if ((s = b->gradient_norm(&g))) return fail(s);
    st->gradient_norm = g;
    st->has_gradient_norm = 1;
    if (g <= opt.gradient_tolerance) return finish(2);
    if (stalled && (tried_undamped || st->accepted_steps == opt.max_iterations)) return fail(FG_NO_PROGRESS);
    if (st->accepted_steps == opt.max_iterations) return fail(FG_NO_CONVERGENCE);
    if ((s = b->prepare_damping(lo.min_column_norm))) return fail(s);
    bool undamped = stalled;
    tried_undamped |= undamped;
    double growth = 2.0;
    bool accepted = false;
    for (size_t t = 0; t < lo.max_trials; ++t) {
      st->attempts += 1;
      double damping = undamped ? 0.0 : lambda;
      st->damping = damping;
      double predicted = 0;
      int rejection = 0;
      fg_status r = b->solve_damped(damping, &predicted, !dev);
      fg_status na = FG_UNSUPPORTED_STRUCTURE;
      if (r == FG_OK && d_lm) na = b->step_norm_async(d_lm + LMW);
      if (r == FG_LINEAR_SOLVE_FAILED) {
        rejection = 1;
      } else if (r) {
        return fail(r);
      } else if (na == FG_OK) {
        // the whole trial on the device, one read back
        LmTrialState in{};
        in.current = current;
        in.lambda = lambda;
        in.growth = growth;
        in.predicted = predicted;
        *h_lm = in;
        const bool costed = std::isfinite(predicted) && predicted > 0;
        FG_CUDA(cudaMemcpyAsync(d_lm, h_lm, sizeof(LmTrialState), cudaMemcpyHostToDevice, bp->st));
        const double* d_result = nullptr;
        if (costed) {
          if ((s = pb.stage_and_cost_device(b->step_device(), &d_result))) return fail(s);
        } else {
          d_result = bp->result.get();  // not read: the decision rejects on the prediction
        }
        FG_LAUNCH(k_lm_decide, 1, 1, 0, bp->st, reinterpret_cast<LmTrialState*>(d_lm), d_lm + LMW, d_result, lo,
                  opt.step_tolerance, opt.cost_tolerance, (int)undamped);
        FG_CUDA(cudaMemcpyAsync(h_lm, d_lm, sizeof(LmTrialState), cudaMemcpyDeviceToHost, bp->st));
        FG_CUDA(cudaStreamSynchronize(bp->st));
        const LmTrialState& o = *h_lm;
        if (o.norm_bad) return fail(FG_LINEAR_SOLVE_FAILED);
        st->step_norm = o.norm;
        st->has_step_norm = 1;
        if (costed) st->cost_evaluations += 1;
        if (o.accepted) {
          pb.accept();
          st->accepted_steps += 1;
          st->cost = o.value;
          st->has_cost = 1;
          stalled = o.stalled != 0;
          current = o.current;
          lambda = o.lambda;
          accepted = true;
          record_work(b, st);
          if (on_accept) on_accept(user, st);
          if (o.value <= target_cost) return finish(5);
          break;
        }
        if (costed) pb.reject();
        st->rejected_steps += 1;
        st->last_rejection = o.rejection;
        if (o.stop) break;
        lambda = o.lambda;
        growth = o.growth;
        continue;
      } else {
        double norm;
        if (b->step_norm_inf(&norm) != FG_OK) return fail(FG_LINEAR_SOLVE_FAILED);
        st->step_norm = norm;
        st->has_step_norm = 1;
        if (!std::isfinite(predicted) || predicted <= 0) {
          rejection = 2;
        } else {
          pb.stage(dev ? b->step_device() : b->step_host());
          st->cost_evaluations += 1;
          double value;
          fg_status ce = pb.cost(true, &value);
          if (ce == FG_INVALID_EVALUATION) {
            pb.reject();
            rejection = 3;
          } else if (ce) {
            pb.reject();
            return fail(ce);
          } else {
            double actual = current - value;
            double ratio = std::min(actual / predicted, 2.0);
            if (actual > 0 && ratio >= lo.acceptance_threshold) {
              pb.accept();
              st->accepted_steps += 1;
              st->cost = value;
              st->has_cost = 1;
              stalled = opt.step_tolerance > 0 && norm <= opt.step_tolerance &&
                        (opt.cost_tolerance == 0 || actual / std::max(current, 1.0) <= opt.cost_tolerance);
              current = value;
              // Nielsen's update; the ratio is clamped before cubing.
              double c = 2.0 * std::min(ratio, 1.0) - 1.0;
              double update = std::max(1.0 - c * c * c, 1.0 / 3.0);
              lambda = std::min(std::max(lambda * update, lo.min_damping), lo.max_damping);
              accepted = true;
              record_work(b, st);
              if (on_accept) on_accept(user, st);
              if (value <= target_cost) return finish(5);
              break;
            }
            pb.reject();
            rejection = 4;
          }
        }
      }
      st->rejected_steps += 1;
      st->last_rejection = rejection;
      if (undamped || lambda == lo.max_damping) break;
      lambda = std::min(lambda * growth, lo.max_damping);
      growth = std::min(growth * 2.0, std::max(lo.max_damping, 2.0));
    }
    if (!accepted) return fail(FG_NO_PROGRESS);
  }
}

fg_status gn_optimize(Backend* b, ProblemAdapter& pb, const fg_optimize_options& opt, fg_optimize_report* rep) {
  FG_TRY(validate(opt));
  FG_TRY(b->prepare(pb.dimension()));
  double initial;
  FG_TRY(pb.cost(false, &initial));
  double current = initial;
  size_t its = 0;
  rep->initial_cost = initial;
  auto report = [&](int term) {
    rep->final_cost = current;
    rep->iterations = its;
    rep->termination = term;
    return FG_OK;
  };
  if (pb.dimension() == 0) return report(1);
  const bool dev = pb.device_steps();
  for (;;) {
    FG_TRY(pb.linearize(b));
    double g;
    FG_TRY(b->gradient_norm(&g));
    if (g <= opt.gradient_tolerance) return report(2);
    if (its == opt.max_iterations) return FG_NO_CONVERGENCE;
    // LeastSquaresBackend::solve (gauss_newton.rs:134).
    FG_TRY(b->solve_undamped(!dev));
    double norm;
    if (b->step_norm_inf(&norm) != FG_OK) return FG_LINEAR_SOLVE_FAILED;
    if (norm <= opt.step_tolerance) return report(3);
    pb.stage(dev ? b->step_device() : b->step_host());
    double tc;
    fg_status s = pb.cost(true, &tc);
    if (s) {
      pb.reject();
      return s;
    }
    pb.accept();
    ++its;
    double dec = current - tc;
    bool conv = tc == 0 || (dec >= 0 && dec / std::max(current, 1.0) <= opt.cost_tolerance);
    current = tc;
    if (conv) return report(4);
  }
}

fg_status lm_solve_bal(Backend* b, BalProblem* p, const fg_optimize_options& o, const fg_lm_options& lo,
                       fg_optimize_report* rep, fg_lm_statistics* st, fg_accept_callback cb, void* user,
                       double target_cost) {
  BalAdapter a(p);
  return lm_optimize(b, a, o, lo, rep, st, cb, user, target_cost);
}
fg_status gn_solve_bal(Backend* b, BalProblem* p, const fg_optimize_options& o, fg_optimize_report* rep) {
  BalAdapter a(p);
  return gn_optimize(b, a, o, rep);
}
fg_status lm_callbacks(Backend* b, const fg_problem_callbacks* cb, void* user, double* x,
                       const fg_optimize_options& o, const fg_lm_options& lo, fg_optimize_report* rep,
                       fg_lm_statistics* st) {
  CallbackAdapter a;
  a.cb = cb;
  a.user = user;
  a.x = x;
  return lm_optimize(b, a, o, lo, rep, st, nullptr, nullptr);
}
fg_status gn_callbacks(Backend* b, const fg_problem_callbacks* cb, void* user, double* x,
                       const fg_optimize_options& o, fg_optimize_report* rep) {
  CallbackAdapter a;
  a.cb = cb;
  a.user = user;
  a.x = x;
  return gn_optimize(b, a, o, rep);
}

}  // namespace fg
