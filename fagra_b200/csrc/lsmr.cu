// Device LSMR backend: fagra's `Lsmr` (src/lsmr.rs, src/lsmr/preconditioner.rs)
// behind the same LeastSquaresBackend entry points as the Schur backend.
//
// Host side: accumulate packs emissions exactly as LinearizedModel::accumulate
// (src/linear_model.rs:180-210) and accumulates the gradient in the same
// order, so gradient_norm matches the reference bit for bit. The structure
// (emission table, column segments and their pieces) is built once per
// distinct emission pattern and reused across linearizations.
//
// Device side (lsmr_kernels.cuh): the LSMR iteration of faer 0.24.4 (restated
// from Fong & Saunders 2011, Algorithm 1: zero start, right preconditioner,
// stopping test ||(A M)^T r|| <= rel_tol ||(A M)^T b|| made before each
// iteration) as three kernels per iteration, replayed from CUDA graphs; the
// step recovery and the explicit verification of recover_and_verify
// (src/lsmr.rs:418-456) run on the device as well.
#include "common.cuh"
#include "schur.cuh"
#include "lsmr_kernels.cuh"
#include <algorithm>
#include <climits>
#include <cstdlib>

namespace fg {

namespace {
enum { MODE_NONE = -1, MODE_IDENTITY = 0, MODE_DIAGONAL = 1, MODE_BLOCK = 2 };
// CUDA graph variants: undamped (no bottom rows, unscaled), identity damped,
// diagonal, block-Jacobi.
enum { GRAPH_UNDAMPED = 0, GRAPH_IDENTITY = 1, GRAPH_DIAGONAL = 2, GRAPH_BLOCK = 3 };
constexpr int LSMR_GRAPH_ITERS = 8;
constexpr int LSMR_COND_ITERS = 2;  // iterations per trip of the single-launch graph

// The loop condition of the single-launch LSMR graph (a WHILE node whose body
// is LSMR_COND_ITERS iterations): continue until the device's stopping rules
// set stop, and for fewer trips than the polled loop's bound allows
// (max_iterations + 2 x 8 launched iterations), so the loop always ends.
__global__ void k_lsmr_continue(cudaGraphConditionalHandle h, LsmrState* st) {
  const unsigned trips = ++st->trips;
  const unsigned long long limit =
      ((unsigned long long)st->max_iterations + 2 * LSMR_GRAPH_ITERS + LSMR_COND_ITERS - 1) / LSMR_COND_ITERS;
  cudaGraphSetConditional(h, !st->stop && trips < limit ? 1u : 0u);
}

int width_class(int64_t w) { return w <= 4 ? 4 : w <= 8 ? 8 : w <= 16 ? 16 : 32; }
}  // namespace

#define LSMR_DISPATCH(W, ...)                     \
  switch (W) {                                    \
    case 4: {                                     \
      constexpr int MW_ = 4;                      \
      __VA_ARGS__;                                \
    } break;                                      \
    case 8: {                                     \
      constexpr int MW_ = 8;                      \
      __VA_ARGS__;                                \
    } break;                                      \
    case 16: {                                    \
      constexpr int MW_ = 16;                     \
      __VA_ARGS__;                                \
    } break;                                      \
    default: {                                    \
      constexpr int MW_ = 32;                     \
      __VA_ARGS__;                                \
    } break;                                      \
  }

template <class TS>
class LsmrImpl final : public Backend {
 public:
  explicit LsmrImpl(const fg_lsmr_options& o) : opt(o), dev(o.device) {}
  ~LsmrImpl() override { drop_graphs(); }

  fg_status init() {
    FG_TRY(select_device(dev));
    FG_TRY(device_stream(dev, &st));
    // FAGRA_B200_POLLED_GRAPHS set when the backend is created: the polled
    // graphs instead of the single-launch conditional graph (the fallback
    // path, selectable so that it stays tested)
    cond_failed = std::getenv("FAGRA_B200_POLLED_GRAPHS") != nullptr;
    FG_TRY(d_state.resize(1));
    FG_TRY(h_state.resize(1));
    FG_TRY(d_ver.resize(1));
    FG_TRY(h_ver.resize(1));
    FG_TRY(d_fallbacks.resize(1));
    FG_TRY(d_norm.resize(2));
    FG_TRY(h_norm.resize(2));
    FG_TRY(d_counter.resize(1));
    FG_CUDA(cudaMemsetAsync(d_state.get(), 0, sizeof(LsmrState), st));
    FG_CUDA(cudaMemsetAsync(d_ver.get(), 0, sizeof(LsmrVerify), st));
    FG_CUDA(cudaMemsetAsync(d_counter.get(), 0, sizeof(unsigned), st));
    h_erow.assign(1, 0);
    h_eblk.assign(1, 0);
    return FG_OK;
  }

  int kind() const override { return 1; }

  fg_status set_lsmr_options(const fg_lsmr_options& o) override {
    int keep = dev, keep_precision = opt.precision;
    opt = o;
    opt.device = keep;
    opt.precision = keep_precision;
    return FG_OK;
  }

  // ------------------------------------------------------------------ trait
  fg_status prepare(size_t dimension) override {  // src/lsmr.rs:469-480
    solves = iterations = 0;
    diag = fg_lsmr_diagnostics{};
    tim = fg_lsmr_timings{};
    prepared_mode = MODE_NONE;
    if (opt.max_iterations == 0 || !(opt.relative_tolerance >= 0 && opt.relative_tolerance < 1)) {
      set_error("LSMR prepare: max_iterations must be positive and relative_tolerance in [0, 1)");
      return FG_INVALID_OPTIONS;
    }
    FG_TRY(select_device(dev));
    if (dimension != dim) structure_built = false;
    dim = dimension;
    h_grad.assign(dim, 0.0);
    FG_TRY(h_step.resize(std::max<size_t>(dim, 1)));
    FG_TRY(resize_columns());
    return clear();
  }

  fg_status clear() override {  // src/lsmr.rs:482-485
    prepared_mode = MODE_NONE;
    h_erow.assign(1, 0);
    h_eblk.assign(1, 0);
    h_eval.clear();
    h_bcol.clear();
    h_bcols.clear();
    h_values.clear();
    h_negres.clear();
    std::fill(h_grad.begin(), h_grad.end(), 0.0);
    rows = 0;
    source = HOST;
    model_current = false;
    gradient_current = false;
    return FG_OK;
  }

  fg_status accumulate(size_t nrows, const double* r, size_t nb, const size_t* bcols, const size_t* widths,
                       const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) override {
    // LinearizedModel::accumulate (src/linear_model.rs:180-210).
    prepared_mode = MODE_NONE;
    if (source != HOST) clear();
    if (nrows && !r) return FG_NULL_ARGUMENT;
    if (nb && (!bcols || !widths || !jac || !rs || !cs)) return FG_NULL_ARGUMENT;
    for (size_t i = 0; i < nb; ++i) {
      size_t end = bcols[i] + widths[i];
      if (end < bcols[i] || end > dim) {
        set_error("Jacobian block outside the prepared dimension");
        return FG_DIMENSION_MISMATCH;
      }
      if (widths[i] && nrows && !jac[i]) return FG_NULL_ARGUMENT;
    }
    if (rows + nrows < rows) return FG_DIMENSION_MISMATCH;
    const size_t row = rows;
    h_eval.push_back((int64_t)h_values.size());
    for (size_t i = 0; i < nrows; ++i) h_negres.push_back(-r[i]);
    for (size_t b = 0; b < nb; ++b) {
      h_bcol.push_back((int64_t)bcols[b]);
      h_bcols.push_back((int32_t)widths[b]);
      for (size_t j = 0; j < widths[b]; ++j) {
        double g = 0;
        for (size_t i = 0; i < nrows; ++i) {
          double v = jac[b][(ptrdiff_t)i * rs[b] + (ptrdiff_t)j * cs[b]];
          h_values.push_back(v);
          g += v * r[i];
        }
        h_grad[bcols[b] + j] += g;
      }
    }
    rows = row + nrows;
    h_erow.push_back((int64_t)rows);
    h_eblk.push_back((int64_t)h_bcol.size());
    model_current = false;
    gradient_current = false;
    return FG_OK;
  }

  fg_status gradient_norm(double* out) override {  // src/lsmr.rs:496-498
    if (source == HOST) {
      double m = 0;
      for (double g : h_grad) {
        if (!std::isfinite(g)) {
          set_error("nonfinite gradient");
          return FG_INVALID_EVALUATION;
        }
        m = std::max(m, std::fabs(g));
      }
      *out = m;
      return FG_OK;
    }
    FG_TRY(sync_model());
    FG_TRY(device_gradient());
    return device_norm_inf(d_grad.get(), dim, out);
  }

  fg_status solve_undamped(bool copy_to_host) override {  // src/lsmr.rs:500-520
    diag = fg_lsmr_diagnostics{};
    FG_TRY(sync_model());
    EventTimer tl;
    if (opt.collect_timings) tl.start(st);
    unsigned its = 0;
    int term = FG_TERM_NONE;
    double normar = 0, normar0 = 0;
    bool ran = false;
    FG_TRY(run(GRAPH_UNDAMPED, 0.0, &ran, &its, &term, &normar, &normar0));
    if (opt.collect_timings) tim.linear_solve += tl.stop(st);
    if (!ran) {
      diag.termination = FG_TERM_CONVERGED;
      diag.finite_step = 1;
    } else {
      FG_TRY(finish_run(its, term, normar, normar0));
    }
    if (copy_to_host && dim) {
      FG_CUDA(cudaMemcpyAsync(h_step.get(), d_step.get(), dim * sizeof(double), cudaMemcpyDeviceToHost, st));
      FG_CUDA(cudaStreamSynchronize(st));
    }
    if (diag.termination != FG_TERM_CONVERGED) {
      set_error("LSMR solve did not converge");
      return FG_LINEAR_SOLVE_FAILED;
    }
    return FG_OK;
  }

  fg_status prepare_damping(double floor) override {  // src/lsmr.rs:521-546
    prepared_mode = MODE_NONE;
    EventTimer tm;
    if (opt.collect_timings) tm.start(st);
    if (!std::isfinite(floor) || floor <= 0) {
      set_error("min_column_norm must be finite and positive");
      return FG_INVALID_OPTIONS;
    }
    FG_TRY(sync_model());
    if (source == DEVICE && npieces > pp0) {  // the point halves, contiguous (BAL segment pass)
      FG_TRY(d_ptvals.resize((size_t)(npieces - pp0) * 6));
      FG_LAUNCH(k_lsmr_point_copy<TS>, grid_for(npieces - pp0, 256), 256, 0, st, npieces - pp0, pp0, d_pstart.get(),
                d_values.get(), d_ptvals.get());
      ptvals_current = true;
    }
    // Column norms with the floor (LinearizedModel::prepare_scales).
    {
      LsmrState s0{};
      s0.min_scale_bits = 0x7ff0000000000000ull;  // +inf
      s0.max_scale_bits = 0;
      FG_CUDA(cudaMemcpyAsync(d_state.get(), &s0, sizeof(LsmrState), cudaMemcpyHostToDevice, st));
      SegArgs a{};
      a.out = d_scales.get();
      a.floor = floor;
      FG_TRY(launch_segments<SEG_SQUARES>(a, view(nullptr, false)));
      FG_CUDA(cudaMemcpyAsync(h_state.get(), d_state.get(), sizeof(LsmrState), cudaMemcpyDeviceToHost, st));
      FG_CUDA(cudaStreamSynchronize(st));
      const LsmrState& h = *h_state.get();
      if (h.nonfinite_scales) {
        set_error("nonfinite Jacobian column norm");
        return FG_INVALID_EVALUATION;
      }
      if (dim) {
        double mn, mx;
        std::memcpy(&mn, &h.min_scale_bits, sizeof(double));
        std::memcpy(&mx, &h.max_scale_bits, sizeof(double));
        min_scale = mn;
        max_scale = mx;
      }
    }
    const int mode = requested_mode();
    if (mode == MODE_BLOCK) {
      // BlockFactors::prepare (src/linear_model/block_factors.rs:47-111)
      if (!variables_consistent) {
        set_error("emissions use inconsistent or overlapping variable ranges");
        return FG_DIMENSION_MISMATCH;
      }
      if (variables_too_wide) {
        set_error("block preconditioning supports variable blocks of at most 32 columns");
        return FG_UNSUPPORTED_STRUCTURE;
      }
      if (n_entries) {
        LsmrDev<TS> D = view(d_scales.get(), false);
        D.s_fac = d_gram_off.get();
        FG_LAUNCH(k_lsmr_gram<TS>, grid_for(n_entries, LSMR_NT), LSMR_NT, 0, st, D, n_entries, d_entry_seg.get(),
                  d_entry_rc.get(), d_gram.get());
      }
    }
    if (opt.collect_timings) tim.preparation += tm.stop(st);
    prepared_mode = mode;
    return FG_OK;
  }

  fg_status solve_damped(double lambda, double* predicted, bool copy_to_host) override {  // src/lsmr.rs:548-585
    diag = fg_lsmr_diagnostics{};
    const int mode = prepared_mode;
    if (mode == MODE_NONE || mode != requested_mode() || !std::isfinite(lambda) || lambda < 0) {
      set_error("solve_damped requires prepare_damping in the current mode and a finite nonnegative lambda");
      return FG_INVALID_OPTIONS;
    }
    const double root = std::sqrt(lambda);
    const bool scaled = mode != MODE_IDENTITY;
    diag.damping = lambda;
    diag.has_damping = 1;
    if (dim) {
      diag.min_scale = min_scale;
      diag.max_scale = max_scale;
      diag.has_scales = 1;
    }
    if (!std::isfinite(scaled ? root : root * max_scale)) {
      diag.termination = FG_TERM_NONFINITE;
      set_error("nonfinite damping diagonal");
      return FG_LINEAR_SOLVE_FAILED;
    }
    EventTimer tf, tl, tv;
    if (mode == MODE_BLOCK) {
      if (opt.collect_timings) tf.start(st);
      FG_TRY(factor(lambda));
      if (opt.collect_timings) tim.factorization += tf.stop(st);
    }
    if (opt.collect_timings) tl.start(st);
    unsigned its = 0;
    int term = FG_TERM_NONE;
    double normar = 0, normar0 = 0;
    bool ran = false;
    const int gmode = mode == MODE_BLOCK ? GRAPH_BLOCK : mode == MODE_DIAGONAL ? GRAPH_DIAGONAL : GRAPH_IDENTITY;
    FG_TRY(run(gmode, root, &ran, &its, &term, &normar, &normar0));
    if (opt.collect_timings) tim.linear_solve += tl.stop(st);
    if (!ran) {
      diag.termination = FG_TERM_CONVERGED;
      diag.finite_step = 1;
    } else {
      FG_TRY(finish_run(its, term, normar, normar0));
    }
    if (opt.collect_timings) tv.start(st);
    double pred = 0;
    fg_status verified = verify(lambda, scaled, mode == MODE_BLOCK, &pred);
    if (opt.collect_timings) tim.residual_checks += tv.stop(st);
    if (copy_to_host && dim) {
      FG_CUDA(cudaMemcpyAsync(h_step.get(), d_step.get(), dim * sizeof(double), cudaMemcpyDeviceToHost, st));
      FG_CUDA(cudaStreamSynchronize(st));
    }
    if (verified != FG_OK) return verified;
    if (diag.termination != FG_TERM_CONVERGED) {
      set_error("LSMR solve did not converge");
      return FG_LINEAR_SOLVE_FAILED;
    }
    *predicted = pred;
    return FG_OK;
  }

  fg_status step_norm_inf(double* out) override { return device_norm_inf(d_step.get(), dim, out); }
  const double* step_host() const override { return h_step.get(); }
  const double* step_device() const override { return d_step.get(); }
  size_t dimension() const override { return dim; }
  void work(size_t* s, size_t* i) const override {
    *s = solves;
    *i = iterations;
  }
  void lsmr_diagnostics(fg_lsmr_diagnostics* d) const override { *d = diag; }
  void lsmr_timings(fg_lsmr_timings* t) const override { *t = tim; }
  bool is_f32() const override { return !std::is_same<TS, double>::value; }
  int device() const override { return dev; }
  cudaStream_t stream() const override { return st; }
  void* values_device() override { return d_values.get(); }
  double* negres_device() override { return d_negres.get(); }

  // ---------------------------------------------------------- device BAL path
  void mark_device_model(size_t nrows) override {
    source = DEVICE;
    rows = nrows;
    model_current = true;
    ptvals_current = false;
    gradient_current = false;
    prepared_mode = MODE_NONE;
  }

  fg_status bind_bal(const BalObservations& ob) override {
    const uint64_t id = ob.problem_id;
    const size_t cams = ob.cameras, pts = ob.points, obs = ob.observations;
    if (dim != 9 * cams + 3 * pts) return FG_DIMENSION_MISMATCH;
    prepared_mode = MODE_NONE;
    if (!(bal_bound == id && structure_built)) {
      const uint32_t *ocam = nullptr, *opt_ = nullptr;
      FG_TRY(ob.host(&ocam, &opt_));
      // Emission k: rows 2k..2k+1, camera block (9 columns) then point block.
      h_erow.resize(obs + 1);
      h_eblk.resize(obs + 1);
      h_eval.resize(obs);
      h_bcol.resize(2 * obs);
      h_bcols.resize(2 * obs);
      for (size_t k = 0; k < obs; ++k) {
        h_erow[k] = 2 * (int64_t)k;
        h_eblk[k] = 2 * (int64_t)k;
        h_eval[k] = 24 * (int64_t)k;
        h_bcol[2 * k] = 9 * (int64_t)ocam[k];
        h_bcol[2 * k + 1] = 9 * (int64_t)cams + 3 * (int64_t)opt_[k];
        h_bcols[2 * k] = 9;
        h_bcols[2 * k + 1] = 3;
      }
      h_erow[obs] = 2 * (int64_t)obs;
      h_eblk[obs] = 2 * (int64_t)obs;
      rows = 2 * obs;
      point_col0 = 9 * (int64_t)cams;
      FG_TRY(build_structure());
      bal_bound = id;
    }
    nvalues = 24 * obs;
    FG_TRY(d_values.resize(std::max<size_t>(nvalues, 1)));
    FG_TRY(d_negres.resize(std::max<size_t>(2 * obs, 1)));
    FG_TRY(resize_rows(2 * obs));
    source = DEVICE;
    return FG_OK;
  }

  // The linearization in the reference layout: emission k has rows
  // [h_erow[k], h_erow[k+1]), blocks [h_eblk[k], h_eblk[k+1]) and its values
  // start at h_eval[k], each block column-major.
  fg_status model_host(HostModel* m) override {
    FG_TRY(sync_model());
    const size_t ne = h_eval.size();
    m->rows = rows;
    m->cols = dim;
    m->blocks.clear();
    for (size_t k = 0; k < ne; ++k) {
      const size_t r0 = (size_t)h_erow[k], nr = (size_t)(h_erow[k + 1] - h_erow[k]);
      size_t start = (size_t)h_eval[k];
      for (int64_t b = h_eblk[k]; b < h_eblk[k + 1]; ++b) {
        m->blocks.push_back(HostBlock{r0, (size_t)h_bcol[b], nr, (size_t)h_bcols[b], start});
        start += nr * (size_t)h_bcols[b];
      }
    }
    m->values.assign(std::max<size_t>(nvalues, 1), 0.0);
    m->negres.assign(std::max<size_t>(rows, 1), 0.0);
    FG_CUDA(cudaStreamSynchronize(st));
    if (nvalues) {
      std::vector<TS> tmp(nvalues);
      FG_CUDA(cudaMemcpy(tmp.data(), d_values.get(), nvalues * sizeof(TS), cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < nvalues; ++i) m->values[i] = (double)tmp[i];
    }
    if (rows) FG_CUDA(cudaMemcpy(m->negres.data(), d_negres.get(), rows * sizeof(double), cudaMemcpyDeviceToHost));
    return FG_OK;
  }

  // ------------------------------------------------------------ test hooks
  fg_status damped_products(double lambda, int scaled, const double* x, double* fwd, const double* y,
                            double* tr) override {
    if (prepared_mode == MODE_NONE) {
      set_error("damped_products requires prepare_damping");
      return FG_INVALID_OPTIONS;
    }
    const size_t m = rows, n = dim;
    std::vector<double> hs(n), w(n);
    if (n) {
      FG_CUDA(cudaMemcpyAsync(hs.data(), d_scales.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st));
      FG_CUDA(cudaStreamSynchronize(st));
    }
    for (size_t j = 0; j < n; ++j) w[j] = scaled ? x[j] / hs[j] : x[j];
    DBuf<double> dw, dytop, dybot, dout;
    FG_TRY(upload(dw, w.data(), n, st));
    FG_TRY(upload(dytop, y, m, st));
    FG_TRY(upload(dybot, y + m, n, st));
    FG_TRY(dout.resize(std::max<size_t>(n, 1)));
    LsmrState s0{};
    s0.root = std::sqrt(lambda);
    FG_CUDA(cudaMemcpyAsync(d_state.get(), &s0, sizeof(LsmrState), cudaMemcpyHostToDevice, st));
    LsmrDev<TS> D = view(d_scales.get(), false);
    const unsigned eb = grid_for(std::max<int64_t>(E, 1), LSMR_NT), bb = grid_for(std::max<size_t>(n, 1), LSMR_NT);
    FG_LAUNCH((k_lsmr_rows<TS, ROWS_PRODUCT>), eb + bb, LSMR_NT, 0, st, D, eb, dw.get(), d_u.get(), d_ub.get(),
              d_negres.get(), d_pr.get(), d_partials.get(), d_state.get(), d_ver.get());
    SegArgs a{};
    a.vec = dytop.get();
    a.ub = dybot.get();
    a.out = dout.get();
    a.scaled = scaled;
    FG_TRY(launch_segments<SEG_PRODUCT>(a, D));
    if (m) FG_CUDA(cudaMemcpyAsync(fwd, d_pr.get(), m * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (n) {
      FG_CUDA(cudaMemcpyAsync(fwd + m, d_ub.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st));
      FG_CUDA(cudaMemcpyAsync(tr, dout.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    FG_CUDA(cudaStreamSynchronize(st));
    return FG_OK;
  }

  fg_status time_iteration(double lambda, size_t reps, double* seconds, double* bytes) override {
    const int mode = prepared_mode;
    if (mode == MODE_NONE || !std::isfinite(lambda) || lambda < 0) {
      set_error("time_iteration requires prepare_damping and a finite nonnegative lambda");
      return FG_INVALID_OPTIONS;
    }
    if (mode == MODE_BLOCK) FG_TRY(factor(lambda));
    const int gmode = mode == MODE_BLOCK ? GRAPH_BLOCK : mode == MODE_DIAGONAL ? GRAPH_DIAGONAL : GRAPH_IDENTITY;
    const size_t graphs = std::max<size_t>((reps + LSMR_GRAPH_ITERS - 1) / LSMR_GRAPH_ITERS, 1);
    FG_TRY(start(gmode, std::sqrt(lambda), 0.0, 0xffffffffu));
    FG_TRY(launch_graph(gmode));  // warm
    EventTimer t;
    t.start(st);
    for (size_t k = 0; k < graphs; ++k) FG_TRY(launch_graph(gmode));
    double sec = t.stop(st);
    *seconds = sec / (double)(graphs * LSMR_GRAPH_ITERS);
    *bytes = iteration_bytes(gmode);
    return FG_OK;
  }

 private:
  enum Source { HOST, DEVICE };
  fg_lsmr_options opt;
  int dev;
  cudaStream_t st = nullptr;
  size_t dim = 0, rows = 0, nvalues = 0;
  Source source = HOST;
  bool model_current = false, gradient_current = false, structure_built = false;
  int prepared_mode = MODE_NONE;
  uint64_t bal_bound = 0;
  size_t solves = 0, iterations = 0;
  fg_lsmr_diagnostics diag{};
  fg_lsmr_timings tim{};
  double min_scale = 0, max_scale = 0;

  // host model (reference layout)
  std::vector<int64_t> h_erow, h_eblk, h_eval, h_bcol;
  std::vector<int32_t> h_bcols;
  std::vector<double> h_values, h_negres, h_grad;
  // structure that the device copy was built from
  std::vector<int64_t> b_erow, b_eblk, b_bcol;
  std::vector<int32_t> b_bcols;

  // structure sizes
  int64_t E = 0, S = 0, npieces = 0, n_entries = 0, n_fac = 0;
  int64_t point_col0 = -1, pp0 = 0;  // BAL: first point column / first point piece
  bool ptvals_current = false;
  DBuf<TS> d_ptvals;
  int fused_ncam = 0;            // > 0: the fused BAL iteration pass applies (camera segments)
  DBuf<double> d_csum, d_pcon;   // its camera column sums and per-emission point contributions
  int32_t n_wide = 0, n_narrow = 0;
  int maxw = 4;
  bool variables_consistent = true, variables_too_wide = false;

  // device buffers
  DBuf<int64_t> d_erow, d_eblk, d_eval, d_bcol, d_scol, d_spc, d_pstart, d_prow, d_gram_off, d_active, d_entry_seg;
  DBuf<int32_t> d_bcols, d_prows, d_swide, d_snarrow, d_entry_rc;
  DBuf<TS> d_values, d_u;
  DBuf<double> d_negres, d_grad, d_scales, d_gram, d_factors, d_ub, d_v, d_w, d_h, d_hbar, d_y, d_step, d_pr,
      d_partials, d_norm;
  DBuf<LsmrState> d_state;
  DBuf<LsmrVerify> d_ver;
  DBuf<unsigned> d_fallbacks, d_counter;
  HBuf<LsmrState> h_state;
  HBuf<LsmrVerify> h_ver;
  HBuf<double> h_step, h_norm;

  cudaGraphExec_t g_exec[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t g_nodes[4] = {0, 0, 0, 0};
  // A solve as one graph launch: a WHILE node over LSMR_COND_ITERS iterations
  // and k_lsmr_continue (no host poll between batches, no gated iterations
  // past the stop beyond the last trip); the polled graphs above are the
  // fallback if the driver refuses the conditional graph.
  cudaGraphExec_t c_exec[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t c_nodes[4] = {0, 0, 0, 0};
  bool cond_failed = false;

  int requested_mode() const {  // src/lsmr.rs:391-399
    return opt.block_preconditioning ? MODE_BLOCK : opt.diagonal_preconditioning ? MODE_DIAGONAL : MODE_IDENTITY;
  }

  void drop_graphs() {
    for (int k = 0; k < 4; ++k) {
      if (g_exec[k]) cudaGraphExecDestroy(g_exec[k]);
      g_exec[k] = nullptr;
      if (c_exec[k]) cudaGraphExecDestroy(c_exec[k]);
      c_exec[k] = nullptr;
    }
  }

  // Column-sized buffers; a reallocation invalidates the graphs.
  fg_status resize_columns() {
    const size_t n = std::max<size_t>(dim, 1);
    DBuf<double>* cols[] = {&d_grad, &d_scales, &d_ub, &d_v, &d_w, &d_h, &d_hbar, &d_y, &d_step};
    for (DBuf<double>* b : cols) {
      double* before = b->get();
      FG_TRY(b->resize(n));
      if (b->get() != before) drop_graphs();
    }
    return FG_OK;
  }
  fg_status resize_rows(size_t m) {
    TS* u0 = d_u.get();
    double* p0 = d_pr.get();
    FG_TRY(d_u.resize(std::max<size_t>(m, 1)));
    FG_TRY(d_pr.resize(std::max<size_t>(m, 1)));
    if (d_u.get() != u0 || d_pr.get() != p0) drop_graphs();
    return FG_OK;
  }

  LsmrDev<TS> view(const double* scales, bool block) const {
    LsmrDev<TS> D{};
    D.values = d_values.get();
    D.m = (int64_t)rows;
    D.n = (int64_t)dim;
    D.E = E;
    D.e_row = d_erow.get();
    D.e_blk = d_eblk.get();
    D.e_val = d_eval.get();
    D.b_col = d_bcol.get();
    D.b_cols = d_bcols.get();
    D.S = S;
    D.s_col = d_scol.get();
    D.s_pc = d_spc.get();
    D.p_start = d_pstart.get();
    D.p_row = d_prow.get();
    D.p_rows = d_prows.get();
    D.s_wide = d_swide.get();
    D.s_narrow = d_snarrow.get();
    D.n_wide = n_wide;
    D.n_narrow = n_narrow;
    D.factors = block ? d_factors.get() : nullptr;
    D.s_fac = block ? d_active.get() : nullptr;
    D.scales = scales;
    D.bal = source == DEVICE ? 1 : 0;
    D.ptvals = D.bal && ptvals_current ? d_ptvals.get() : nullptr;
    D.pp0 = pp0;
    return D;
  }

  unsigned segment_grid() const { return (unsigned)n_wide + grid_for(std::max<int32_t>(n_narrow, 1), LSMR_NT); }
  unsigned emission_grid() const { return grid_for(std::max<int64_t>(E, 1), LSMR_NT); }
  unsigned bottom_grid() const { return grid_for(std::max<size_t>(dim, 1), LSMR_NT); }

  template <int MODE>
  fg_status launch_segments(const SegArgs& a, const LsmrDev<TS>& D) {
    if (S == 0) return FG_OK;
    LSMR_DISPATCH(maxw, FG_LAUNCH((k_lsmr_segments<TS, MW_, MODE>), segment_grid(), LSMR_NT, 0, st, D, a,
                                  d_partials.get(), d_state.get(), d_ver.get()));
    return FG_OK;
  }

  // ---- structure: emissions, column segments and pieces
  fg_status build_structure() {
    drop_graphs();
    bal_bound = 0;
    const int64_t n = (int64_t)dim;
    E = (int64_t)h_erow.size() - 1;
    const int64_t nb = (int64_t)h_bcol.size();
    // Segment boundaries at every block edge, widths split at 32.
    std::vector<uint8_t> mark(n + 1, 0);
    mark[0] = 1;
    mark[n] = 1;
    for (int64_t b = 0; b < nb; ++b) {
      if (h_bcols[b] == 0) continue;
      mark[h_bcol[b]] = 1;
      mark[h_bcol[b] + h_bcols[b]] = 1;
    }
    std::vector<int64_t> scol;
    scol.reserve(n / 3 + 2);
    for (int64_t c = 0; c < n;) {
      int64_t e = c + 1;
      while (e < n && !mark[e]) ++e;
      for (int64_t a = c; a < e; a += LSMR_MAX_WIDTH) scol.push_back(a);
      c = e;
    }
    scol.push_back(n);
    S = (int64_t)scol.size() - 1;
    std::vector<int64_t> segof(std::max<int64_t>(n, 1));
    maxw = 4;
    for (int64_t s = 0; s < S; ++s) {
      for (int64_t c = scol[s]; c < scol[s + 1]; ++c) segof[c] = s;
      maxw = std::max(maxw, width_class(scol[s + 1] - scol[s]));
    }
    // Variable consistency (src/linear_model/block_factors.rs:52-87).
    variables_consistent = true;
    variables_too_wide = false;
    {
      std::vector<int64_t> owner(std::max<int64_t>(n, 1), -1);
      std::vector<int32_t> varw(std::max<int64_t>(n, 1), 0);
      for (int64_t b = 0; b < nb && variables_consistent; ++b) {
        const int64_t col = h_bcol[b], w = h_bcols[b];
        if (w == 0) continue;
        if (owner[col] < 0) {
          for (int64_t c = col; c < col + w; ++c)
            if (owner[c] >= 0) variables_consistent = false;
          if (!variables_consistent) break;
          for (int64_t c = col; c < col + w; ++c) owner[c] = col;
          varw[col] = (int32_t)w;
          if (w > LSMR_MAX_WIDTH) variables_too_wide = true;
        } else if (owner[col] != col || varw[col] != w) {
          variables_consistent = false;
        }
      }
    }
    // Pieces: count per segment, then fill in emission order.
    std::vector<int64_t> spc(S + 1, 0);
    for (int64_t e = 0; e < E; ++e)
      for (int64_t b = h_eblk[e]; b < h_eblk[e + 1]; ++b) {
        if (h_bcols[b] == 0) continue;
        for (int64_t s = segof[h_bcol[b]]; s <= segof[h_bcol[b] + h_bcols[b] - 1]; ++s) spc[s + 1]++;
      }
    for (int64_t s = 0; s < S; ++s) spc[s + 1] += spc[s];
    npieces = spc[S];
    std::vector<int64_t> pstart(std::max<int64_t>(npieces, 1)), prow(std::max<int64_t>(npieces, 1));
    std::vector<int32_t> prows(std::max<int64_t>(npieces, 1));
    {
      std::vector<int64_t> fill(spc.begin(), spc.end() - 1);
      for (int64_t e = 0; e < E; ++e) {
        const int64_t r0 = h_erow[e], nr = h_erow[e + 1] - r0;
        int64_t vs = h_eval.empty() ? 0 : h_eval[e];
        for (int64_t b = h_eblk[e]; b < h_eblk[e + 1]; ++b) {
          const int64_t col = h_bcol[b], w = h_bcols[b];
          if (w) {
            for (int64_t s = segof[col]; s <= segof[col + w - 1]; ++s) {
              const int64_t p = fill[s]++;
              pstart[p] = vs + (scol[s] - col) * nr;
              prow[p] = r0;
              prows[p] = (int32_t)nr;
            }
          }
          vs += w * nr;
        }
      }
    }
    // BAL: the first point piece (point columns start at point_col0)
    pp0 = npieces;
    if (point_col0 >= 0 && point_col0 < n) pp0 = spc[segof[point_col0]];
    ptvals_current = false;
    // Wide / narrow segment lists.
    std::vector<int32_t> wide, narrow;
    for (int64_t s = 0; s < S; ++s) (spc[s + 1] - spc[s] > LSMR_WIDE_DEGREE ? wide : narrow).push_back((int32_t)s);
    n_wide = (int32_t)wide.size();
    n_narrow = (int32_t)narrow.size();
    // Gram layout for block preconditioning: one w x w block per covered segment.
    std::vector<int64_t> goff(std::max<int64_t>(S, 1), -1), eseg;
    std::vector<int32_t> erc;
    n_fac = 0;
    if (variables_consistent && !variables_too_wide) {
      for (int64_t s = 0; s < S; ++s) {
        if (spc[s + 1] == spc[s]) continue;
        const int64_t w = scol[s + 1] - scol[s];
        goff[s] = n_fac;
        n_fac += w * w;
        for (int64_t c = 0; c < w; ++c)
          for (int64_t r = c; r < w; ++r) {
            eseg.push_back(s);
            erc.push_back((int32_t)((c << 8) | r));
          }
      }
    }
    n_entries = (int64_t)eseg.size();
    // Upload.
    FG_TRY(upload(d_erow, h_erow.data(), h_erow.size(), st));
    FG_TRY(upload(d_eblk, h_eblk.data(), h_eblk.size(), st));
    std::vector<int64_t> eval = h_eval;
    if (eval.empty()) eval.push_back(0);
    FG_TRY(upload(d_eval, eval.data(), eval.size(), st));
    std::vector<int64_t> bcol = h_bcol;
    std::vector<int32_t> bcols = h_bcols;
    if (bcol.empty()) {
      bcol.push_back(0);
      bcols.push_back(0);
    }
    FG_TRY(upload(d_bcol, bcol.data(), bcol.size(), st));
    FG_TRY(upload(d_bcols, bcols.data(), bcols.size(), st));
    FG_TRY(upload(d_scol, scol.data(), scol.size(), st));
    FG_TRY(upload(d_spc, spc.data(), spc.size(), st));
    FG_TRY(upload(d_pstart, pstart.data(), pstart.size(), st));
    FG_TRY(upload(d_prow, prow.data(), prow.size(), st));
    FG_TRY(upload(d_prows, prows.data(), prows.size(), st));
    if (wide.empty()) wide.push_back(0);
    if (narrow.empty()) narrow.push_back(0);
    FG_TRY(upload(d_swide, wide.data(), wide.size(), st));
    FG_TRY(upload(d_snarrow, narrow.data(), narrow.size(), st));
    FG_TRY(upload(d_gram_off, goff.data(), goff.size(), st));
    FG_TRY(d_active.resize(std::max<int64_t>(S, 1)));
    if (eseg.empty()) {
      eseg.push_back(0);
      erc.push_back(0);
    }
    FG_TRY(upload(d_entry_seg, eseg.data(), eseg.size(), st));
    FG_TRY(upload(d_entry_rc, erc.data(), erc.size(), st));
    FG_TRY(d_gram.resize(std::max<int64_t>(n_fac, 1)));
    FG_TRY(d_factors.resize(std::max<int64_t>(n_fac, 1)));
    // The fused iteration pass (device BAL layout): camera segments first, one
    // 9-column camera block each, their pieces the camera blocks of one
    // contiguous range of emissions in order; then 3-column point segments of
    // point blocks.
    fused_ncam = 0;
    if (point_col0 > 0 && point_col0 <= n) {
      const int64_t ncs = point_col0 == n ? S : segof[point_col0];
      bool ok = ncs * 9 == point_col0;
      for (int64_t sg = 0; sg < ncs && ok; ++sg) {
        ok = scol[sg + 1] - scol[sg] == 9;
        const int64_t q0 = spc[sg], q1 = spc[sg + 1];
        for (int64_t q = q0; q < q1 && ok; ++q) ok = pstart[q] % 24 == 0 && pstart[q] == pstart[q0] + 24 * (q - q0);
      }
      for (int64_t sg = ncs; sg < S && ok; ++sg) {
        ok = scol[sg + 1] - scol[sg] == 3;
        for (int64_t q = spc[sg]; q < spc[sg + 1] && ok; ++q) ok = pstart[q] % 24 == 18;
      }
      if (ok && ncs > 0 && ncs < (int64_t)1 << 30) fused_ncam = (int)ncs;
    }
    if (fused_ncam) {
      FG_TRY(d_csum.resize((size_t)9 * fused_ncam));
      FG_TRY(d_pcon.resize(std::max<size_t>((size_t)3 * E, 1)));
    }
    const size_t parts = std::max<size_t>(
        (size_t)std::max<unsigned>(std::max<unsigned>(segment_grid() * SEG_K, emission_grid() + bottom_grid()),
                                   (unsigned)fused_ncam + bottom_grid()),
        8192);
    FG_TRY(d_partials.resize(parts));
    FG_TRY(resize_rows(rows));
    FG_CUDA(cudaStreamSynchronize(st));  // host staging vectors die here
    b_erow = h_erow;
    b_eblk = h_eblk;
    b_bcol = h_bcol;
    b_bcols = h_bcols;
    structure_built = true;
    return FG_OK;
  }

  fg_status sync_model() {
    if (source == DEVICE) {
      if (!model_current) {
        set_error("device model not linearized");
        return FG_INVALID_OPTIONS;
      }
      return FG_OK;
    }
    if (model_current) return FG_OK;
    point_col0 = -1;  // host emissions: generic layout
    if (!structure_built || b_erow != h_erow || b_eblk != h_eblk || b_bcol != h_bcol || b_bcols != h_bcols)
      FG_TRY(build_structure());
    nvalues = h_values.size();
    {
      TS* before = d_values.get();
      if (nvalues == 0) {
        FG_TRY(d_values.resize(1));
      } else if (std::is_same<TS, double>::value) {
        FG_TRY(upload(d_values, (const TS*)(const void*)h_values.data(), nvalues, st));
      } else {
        std::vector<TS> conv(std::max<size_t>(nvalues, 1));
        for (size_t i = 0; i < nvalues; ++i) conv[i] = (TS)h_values[i];
        FG_TRY(upload(d_values, conv.data(), conv.size(), st));
        FG_CUDA(cudaStreamSynchronize(st));
      }
      if (d_values.get() != before) drop_graphs();
    }
    {
      double* before = d_negres.get();
      std::vector<double> neg = h_negres;
      if (neg.empty()) neg.push_back(0);
      FG_TRY(upload(d_negres, neg.data(), neg.size(), st));
      FG_CUDA(cudaStreamSynchronize(st));
      if (d_negres.get() != before) drop_graphs();
    }
    if (dim) FG_CUDA(cudaMemcpyAsync(d_grad.get(), h_grad.data(), dim * sizeof(double), cudaMemcpyHostToDevice, st));
    FG_TRY(resize_rows(rows));
    FG_CUDA(cudaStreamSynchronize(st));
    model_current = true;
    gradient_current = true;
    return FG_OK;
  }

  fg_status device_gradient() {
    if (gradient_current) return FG_OK;
    SegArgs a{};
    a.vec = d_negres.get();
    a.out = d_grad.get();
    FG_TRY(launch_segments<SEG_GRADIENT>(a, view(nullptr, false)));
    gradient_current = true;
    return FG_OK;
  }

  fg_status device_norm_inf(const double* x, size_t n, double* out) {
    if (n == 0) {
      *out = 0;
      return FG_OK;
    }
    unsigned g = std::min<unsigned>(grid_for(n, NT), 4 * sm_count(dev));
    FG_LAUNCH(k_norm_inf<double>, g, NT, 0, st, (int64_t)n, x, d_partials.get(), d_counter.get(), d_norm.get());
    FG_CUDA(cudaMemcpyAsync(h_norm.get(), d_norm.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    if (h_norm.get()[1] != 0) {
      set_error("nonfinite value");
      return FG_INVALID_EVALUATION;
    }
    *out = h_norm.get()[0];
    return FG_OK;
  }

  // BlockFactors::factor at lambda; fallbacks go to the diagnostics.
  fg_status factor(double lambda) {
    FG_CUDA(cudaMemsetAsync(d_fallbacks.get(), 0, sizeof(unsigned), st));
    if (S) {
      FG_LAUNCH(k_lsmr_factor, grid_for(S, LSMR_NT), LSMR_NT, 0, st, S, d_scol.get(), d_gram_off.get(),
                d_gram.get(), lambda, d_factors.get(), d_active.get(), d_fallbacks.get());
    }
    unsigned fb = 0;
    FG_CUDA(cudaMemcpyAsync(&fb, d_fallbacks.get(), sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    diag.block_fallbacks = fb;
    return FG_OK;
  }

  // ---- the LSMR loop
  const double* graph_scales(int gmode) const { return gmode == GRAPH_UNDAMPED ? nullptr : d_scales.get(); }

  fg_status start(int gmode, double root, double tolerance, unsigned max_its) {
    LsmrState s0{};
    s0.tolerance = tolerance;
    s0.max_iterations = max_its;
    s0.root = root;
    FG_CUDA(cudaMemcpyAsync(d_state.get(), &s0, sizeof(LsmrState), cudaMemcpyHostToDevice, st));
    for (DBuf<double>* b : {&d_ub, &d_v, &d_h, &d_hbar, &d_y})
      FG_CUDA(cudaMemsetAsync(b->get(), 0, dim * sizeof(double), st));
    const bool block = gmode == GRAPH_BLOCK;
    LsmrDev<TS> D = view(graph_scales(gmode), block);
    const unsigned eb = emission_grid();
    FG_LAUNCH((k_lsmr_rows<TS, ROWS_START>), eb, LSMR_NT, 0, st, D, eb, d_w.get(), d_u.get(), d_ub.get(),
              d_negres.get(), d_pr.get(), d_partials.get(), d_state.get(), d_ver.get());
    SegArgs a = iteration_args(gmode);
    FG_TRY(launch_segments<SEG_START>(a, D));
    FG_TRY(launch_update(gmode, D));
    return FG_OK;
  }

  SegArgs iteration_args(int gmode) {
    SegArgs a{};
    a.vec = d_u.get();
    a.ub = d_ub.get();
    a.v = d_v.get();
    a.scaled = gmode == GRAPH_DIAGONAL || gmode == GRAPH_BLOCK;
    return a;
  }

  fg_status launch_update(int gmode, const LsmrDev<TS>& D) {
    const int scaled = gmode == GRAPH_DIAGONAL || gmode == GRAPH_BLOCK;
    LSMR_DISPATCH(maxw, FG_LAUNCH((k_lsmr_update<TS, MW_, false>), grid_for(std::max<int64_t>(S, 1), LSMR_NT), LSMR_NT,
                                  0, st, D, d_v.get(), d_h.get(), d_hbar.get(), d_y.get(), d_w.get(), scaled,
                                  d_state.get()));
    return FG_OK;
  }

  fg_status iteration_body(int gmode, EventTimer* tf, EventTimer* tt, EventTimer* tp) {
    const bool block = gmode == GRAPH_BLOCK;
    LsmrDev<TS> D = view(graph_scales(gmode), block);
    const unsigned eb = emission_grid(), bb = gmode == GRAPH_UNDAMPED ? 0 : bottom_grid();
    if (fused_ncam && D.bal) {
      // one read of the emissions: u <- J w - alpha u with the camera sums and
      // point contributions of J^T u, then every segment's finish
      if (tf) tf->start(st);
      FG_LAUNCH((k_lsmr_fused_rows<TS>), (unsigned)fused_ncam + bb, LSMR_NT, 0, st, D, fused_ncam, d_w.get(),
                d_u.get(), d_ub.get(), d_csum.get(), d_pcon.get(), d_partials.get(), d_state.get());
      if (tf) tim.forward += tf->stop(st);
      if (tt) tt->start(st);
      LSMR_DISPATCH(maxw, FG_LAUNCH((k_lsmr_fused_segments<TS, MW_>), grid_for(std::max<int64_t>(S, 1), LSMR_NT),
                                    LSMR_NT, 0, st, D, iteration_args(gmode), fused_ncam, d_csum.get(),
                                    d_pcon.get(), d_partials.get(), d_state.get()));
      if (tt) tim.transpose += tt->stop(st);
    } else {
      if (tf) tf->start(st);
      FG_LAUNCH((k_lsmr_rows<TS, ROWS_ITER>), eb + bb, LSMR_NT, 0, st, D, eb, d_w.get(), d_u.get(), d_ub.get(),
                d_negres.get(), d_pr.get(), d_partials.get(), d_state.get(), d_ver.get());
      if (tf) tim.forward += tf->stop(st);
      if (tt) tt->start(st);
      FG_TRY(launch_segments<SEG_ITER>(iteration_args(gmode), D));
      if (tt) tim.transpose += tt->stop(st);
    }
    if (tp) tp->start(st);
    FG_TRY(launch_update(gmode, D));
    if (tp) tim.preconditioner += tp->stop(st);
    return FG_OK;
  }

  fg_status launch_graph(int gmode) {
    if (!g_exec[gmode]) {
      cudaGraph_t graph = nullptr;
      uint64_t before = g_launches.load();
      FG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      fg_status s = FG_OK;
      for (int k = 0; k < LSMR_GRAPH_ITERS && s == FG_OK; ++k) s = iteration_body(gmode, nullptr, nullptr, nullptr);
      cudaError_t e = cudaStreamEndCapture(st, &graph);
      g_nodes[gmode] = g_launches.load() - before;
      g_launches.fetch_sub(g_nodes[gmode]);  // captured, not launched
      if (s != FG_OK) {
        if (graph) cudaGraphDestroy(graph);
        return s;
      }
      FG_CUDA(e);
      e = cudaGraphInstantiate(&g_exec[gmode], graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        g_exec[gmode] = nullptr;
        return cuda_status(e, "cudaGraphInstantiate");
      }
    }
    FG_CUDA(cudaGraphLaunch(g_exec[gmode], st));
    g_launches.fetch_add(g_nodes[gmode]);
    return FG_OK;
  }

  fg_status launch_continue(cudaGraphConditionalHandle h) {
    FG_LAUNCH(k_lsmr_continue, 1, 1, 0, st, h, d_state.get());
    return FG_OK;
  }
  fg_status capture_cond_graph(int gmode, cudaGraph_t* out) {
    FG_CUDA(cudaGraphCreate(out, 0));
    cudaGraphConditionalHandle h;
    FG_CUDA(cudaGraphConditionalHandleCreate(&h, *out, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    FG_CUDA(cudaGraphAddNode(&node, *out, nullptr, 0, &np));
    const uint64_t before = g_launches.load();
    FG_CUDA(cudaStreamBeginCaptureToGraph(st, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
    fg_status s = FG_OK;
    for (int k = 0; k < LSMR_COND_ITERS && s == FG_OK; ++k) s = iteration_body(gmode, nullptr, nullptr, nullptr);
    if (s == FG_OK) s = launch_continue(h);
    cudaGraph_t body = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &body);
    c_nodes[gmode] = g_launches.load() - before;
    g_launches.fetch_sub(c_nodes[gmode]);  // captured, not launched
    FG_TRY(s);
    FG_CUDA(e);
    return FG_OK;
  }
  fg_status launch_cond_graph(int gmode) {
    if (!c_exec[gmode]) {
      cudaGraph_t graph = nullptr;
      fg_status s = capture_cond_graph(gmode, &graph);
      cudaError_t e = s == FG_OK ? cudaGraphInstantiate(&c_exec[gmode], graph, 0) : cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
      if (s != FG_OK || e != cudaSuccess) {
        c_exec[gmode] = nullptr;
        cudaGetLastError();
        return s != FG_OK ? s : cuda_status(e, "cudaGraphInstantiate (conditional)");
      }
    }
    FG_CUDA(cudaGraphLaunch(c_exec[gmode], st));
    return FG_OK;
  }

  fg_status read_state() {
    FG_CUDA(cudaMemcpyAsync(h_state.get(), d_state.get(), sizeof(LsmrState), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    return FG_OK;
  }

  // One LSMR solve (src/lsmr.rs:228-288 around faer's lsmr); the step lands in
  // d_step (M y, divided by D when scaled). *ran = false for an empty system.
  fg_status run(int gmode, double root, bool* ran, unsigned* its, int* term, double* normar, double* normar0) {
    *ran = false;
    if (dim) FG_CUDA(cudaMemsetAsync(d_step.get(), 0, dim * sizeof(double), st));
    if (rows + (gmode == GRAPH_UNDAMPED ? 0 : dim) == 0 || dim == 0) return FG_OK;
    *ran = true;
    solves += 1;
    const unsigned max_its = (unsigned)std::min<size_t>(opt.max_iterations, 0xffffffffu);
    FG_TRY(start(gmode, root, opt.relative_tolerance, max_its));
    FG_TRY(read_state());
    size_t launched = 0, batch = 1;
    EventTimer tf, tt, tp;
    bool whole = false;  // the single-launch graph ran the solve
    if (!h_state.get()->stop && !opt.collect_timings && !cond_failed) {
      if (launch_cond_graph(gmode) == FG_OK) {
        FG_TRY(read_state());
        g_launches.fetch_add((uint64_t)h_state.get()->trips * c_nodes[gmode]);
        whole = true;
      } else {
        cond_failed = true;
      }
    }
    while (!whole && !h_state.get()->stop) {
      if (launched > (size_t)max_its + 2 * LSMR_GRAPH_ITERS) break;  // the device enforces the limit
      if (opt.collect_timings) {
        FG_TRY(iteration_body(gmode, &tf, &tt, &tp));
        launched += 1;
      } else {
        for (size_t k = 0; k < batch; ++k) FG_TRY(launch_graph(gmode));
        launched += batch * LSMR_GRAPH_ITERS;
        batch = std::min<size_t>(batch * 2, 8);
      }
      FG_TRY(read_state());
    }
    const LsmrState& h = *h_state.get();
    *its = h.iterations;
    *term = h.stop ? h.termination : FG_TERM_ITERATION_LIMIT;
    *normar = h.normar;
    *normar0 = h.normar0;
    // x = M y, then the diagonal scaling (src/lsmr.rs:421-428).
    const bool block = gmode == GRAPH_BLOCK;
    LsmrDev<TS> D = view(graph_scales(gmode), block);
    const int scaled = gmode == GRAPH_DIAGONAL || gmode == GRAPH_BLOCK;
    LSMR_DISPATCH(maxw, FG_LAUNCH((k_lsmr_update<TS, MW_, true>), grid_for(std::max<int64_t>(S, 1), LSMR_NT), LSMR_NT,
                                  0, st, D, d_v.get(), d_h.get(), d_hbar.get(), d_y.get(), d_step.get(), scaled,
                                  d_state.get()));
    return FG_OK;
  }

  // Iteration statistics and estimate diagnostics of a finished run.
  fg_status finish_run(unsigned its, int term, double normar, double normar0) {
    iterations += its;
    diag.iterations = its;
    diag.estimated_absolute_residual = normar;
    diag.estimated_relative_residual = normar0 > 0 ? normar / normar0 : 0.0;
    diag.has_estimated = 1;
    double tmp = 0;
    fg_status f = device_norm_inf(d_step.get(), dim, &tmp);
    if (f != FG_OK && f != FG_INVALID_EVALUATION) return f;
    diag.finite_step = f == FG_OK;
    const bool finite = diag.finite_step && std::isfinite(normar) && std::isfinite(diag.estimated_relative_residual);
    diag.termination = finite ? term : FG_TERM_NONFINITE;
    return FG_OK;
  }

  // recover_and_verify (src/lsmr.rs:418-456) after the step is in d_step.
  fg_status verify(double lambda, bool scaled, bool block, double* predicted) {
    LsmrDev<TS> D = view(d_scales.get(), block);
    const unsigned eb = emission_grid();
    FG_CUDA(cudaMemsetAsync(d_ver.get(), 0, sizeof(LsmrVerify), st));
    if (E)
      FG_LAUNCH((k_lsmr_rows<TS, ROWS_VERIFY>), eb, LSMR_NT, 0, st, D, eb, d_step.get(), d_u.get(), d_ub.get(),
                d_negres.get(), d_pr.get(), d_partials.get(), d_state.get(), d_ver.get());
    if (!gradient_current) FG_TRY(device_gradient());
    SegArgs a{};
    a.vec = d_pr.get();
    a.step = d_step.get();
    a.grad = d_grad.get();
    a.lambda = lambda;
    a.scaled = scaled;
    FG_TRY(launch_segments<SEG_VERIFY>(a, D));
    FG_CUDA(cudaMemcpyAsync(h_ver.get(), d_ver.get(), sizeof(LsmrVerify), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    const LsmrVerify& v = *h_ver.get();
    const double nr = std::sqrt(v.nr2), g = std::sqrt(v.g2), snr = std::sqrt(v.snr2), sg = std::sqrt(v.sg2);
    diag.finite_step = !v.nonfinite_step;
    diag.original_absolute_residual = nr;
    diag.original_relative_residual = g == 0 ? nr : nr / g;
    diag.scaled_absolute_residual = snr;
    diag.scaled_relative_residual = sg == 0 ? snr : snr / sg;
    diag.has_original = diag.has_scaled = 1;
    if (!diag.finite_step || !std::isfinite(nr) || !std::isfinite(snr)) {
      diag.termination = FG_TERM_NONFINITE;
      set_error("nonfinite LSMR step or residual");
      return FG_LINEAR_SOLVE_FAILED;
    }
    *predicted = -v.gd - 0.5 * v.jd2;  // LinearizedModel::predicted_reduction
    return FG_OK;
  }

  double iteration_bytes(int gmode) const {
    const double s = sizeof(TS), m = (double)rows, n = (double)dim, nv = (double)nvalues;
    const double nb = (double)b_bcol.size();
    double fwd = nv * s + 2 * m * s + (double)E * 24 + nb * 12 + n * 8;
    double tr = nv * s + m * s + (double)npieces * 20 + (double)S * 20;
    if (fused_ncam && source == DEVICE) {
      // one read of the values: u in and out, the point block's column index
      // and w, the point contributions out and back in (3 doubles per
      // emission), the camera sums out and in, the point pieces' starts
      const double nc = (double)fused_ncam, E_ = (double)E;
      fwd = nv * s + 2 * m * s + E_ * (8 + 24) + E_ * 24 + nc * (72 + 72);
      tr = E_ * 24 + E_ * 8 + nc * 72 + (double)S * 16;
    }
    double upd = n * 8 * 9 + (double)S * 8;
    if (gmode != GRAPH_UNDAMPED) {
      fwd += n * 8 * 3;  // scales, bottom rows in and out
      tr += n * 8 * 4;   // scales, bottom rows, v in and out
      upd += n * 8;
    } else {
      tr += n * 8 * 2;
    }
    if (gmode == GRAPH_BLOCK) {
      tr += (double)n_fac * 8;
      upd += (double)n_fac * 8;
    }
    return fwd + tr + upd;
  }
};

fg_status make_lsmr(const fg_lsmr_options& o, Backend** out) {
  if (o.precision != FG_PRECISION_F64 && o.precision != FG_PRECISION_F32_REFINED) {
    set_error("unknown precision");
    return FG_INVALID_OPTIONS;
  }
  if (o.precision == FG_PRECISION_F64) {
    auto* b = new LsmrImpl<double>(o);
    fg_status s = b->init();
    if (s != FG_OK) {
      delete b;
      return s;
    }
    *out = b;
  } else {
    auto* b = new LsmrImpl<float>(o);
    fg_status s = b->init();
    if (s != FG_OK) {
      delete b;
      return s;
    }
    *out = b;
  }
  return FG_OK;
}

}  // namespace fg

using namespace fg;

FG_API void fg_lsmr_default_options(fg_lsmr_options* o) {
  if (!o) return;
  o->max_iterations = 1000;
  o->relative_tolerance = std::max(1e-10, std::numeric_limits<double>::epsilon() * 128.0);
  o->diagonal_preconditioning = 1;
  o->block_preconditioning = 0;
  o->collect_timings = 0;
  o->precision = FG_PRECISION_F64;
  o->device = 0;
}

FG_API fg_status fg_lsmr_create(const fg_lsmr_options* options, fg_backend** out) {
  if (!out) return FG_NULL_ARGUMENT;
  *out = nullptr;
  try {
    fg_lsmr_options o;
    fg_lsmr_default_options(&o);
    if (options) o = *options;
    Backend* b = nullptr;
    FG_TRY(make_lsmr(o, &b));
    *out = new fg_backend{b};
    return FG_OK;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return FG_OUT_OF_MEMORY;
  } catch (...) {
    set_error("unexpected host exception");
    return FG_CUDA_ERROR;
  }
}

FG_API fg_status fg_lsmr_set_options(fg_backend* b, const fg_lsmr_options* o) {
  if (!b || !b->impl || !o) return FG_NULL_ARGUMENT;
  return b->impl->set_lsmr_options(*o);
}

FG_API fg_status fg_lsmr_get_diagnostics(const fg_backend* b, fg_lsmr_diagnostics* d) {
  if (!b || !b->impl || !d) return FG_NULL_ARGUMENT;
  if (b->impl->kind() != 1) {
    set_error("not an LSMR backend");
    return FG_INVALID_OPTIONS;
  }
  b->impl->lsmr_diagnostics(d);
  return FG_OK;
}

FG_API fg_status fg_lsmr_get_timings(const fg_backend* b, fg_lsmr_timings* t) {
  if (!b || !b->impl || !t) return FG_NULL_ARGUMENT;
  if (b->impl->kind() != 1) {
    set_error("not an LSMR backend");
    return FG_INVALID_OPTIONS;
  }
  b->impl->lsmr_timings(t);
  return FG_OK;
}

FG_API fg_status fg_lsmr_damped_products(fg_backend* b, double lambda, int scaled, const double* x, double* fwd,
                                         const double* y, double* tr) {
  if (!b || !b->impl || !x || !fwd || !y || !tr) return FG_NULL_ARGUMENT;
  try {
    return b->impl->damped_products(lambda, scaled, x, fwd, y, tr);
  } catch (...) {
    set_error("unexpected host exception");
    return FG_CUDA_ERROR;
  }
}

FG_API fg_status fg_lsmr_time_iteration(fg_backend* b, double lambda, size_t reps, double* seconds, double* bytes) {
  if (!b || !b->impl || !seconds || !bytes) return FG_NULL_ARGUMENT;
  try {
    return b->impl->time_iteration(lambda, reps, seconds, bytes);
  } catch (...) {
    set_error("unexpected host exception");
    return FG_CUDA_ERROR;
  }
}
