// The extern "C" surface declared in include/fagra_b200.h.
#include "common.cuh"
#include "schur.cuh"
#include "bal.cuh"
#include "lm.cuh"
#include <mutex>
#include <new>

namespace fg {

std::atomic<uint64_t> g_launches{0};
static thread_local std::string t_error;

void set_error(const std::string& text) { t_error = text; }

fg_status cuda_status(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return FG_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return FG_NO_DEVICE;
  return FG_CUDA_ERROR;
}

namespace {
std::mutex g_mu;
cudaStream_t g_streams[64] = {};
int g_sms[64] = {};
}  // namespace

fg_status select_device(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    set_error("no CUDA device available");
    return FG_NO_DEVICE;
  }
  if (device < 0 || device >= n || device >= 64) {
    set_error("invalid device ordinal");
    return FG_INVALID_OPTIONS;
  }
  FG_CUDA(cudaSetDevice(device));
  return FG_OK;
}

fg_status device_stream(int device, cudaStream_t* out) {
  FG_TRY(select_device(device));
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_streams[device]) {
    FG_CUDA(cudaStreamCreateWithFlags(&g_streams[device], cudaStreamNonBlocking));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    g_sms[device] = sms > 0 ? sms : 148;
  }
  *out = g_streams[device];
  return FG_OK;
}

cudaMemPool_t library_pool(int device) {
  static cudaMemPool_t pools[64] = {};
  static bool tried[64] = {};
  if (device < 0 || device >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!tried[device]) {
    tried[device] = true;
    int supported = 0;
    cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, device);
    if (supported) {
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = device;
      cudaMemPool_t p = nullptr;
      if (cudaMemPoolCreate(&p, &props) == cudaSuccess) {
        uint64_t keep = (uint64_t)4 << 30;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[device] = p;
      } else {
        cudaGetLastError();
      }
    }
  }
  return pools[device];
}

int sm_count(int device) { return (device >= 0 && device < 64 && g_sms[device]) ? g_sms[device] : 148; }

}  // namespace fg

using namespace fg;

#define FG_GUARD_BEGIN try {
#define FG_GUARD_END                       \
  }                                        \
  catch (const std::bad_alloc&) {          \
    set_error("host allocation failed");   \
    return FG_OUT_OF_MEMORY;               \
  }                                        \
  catch (...) {                            \
    set_error("unexpected host exception"); \
    return FG_CUDA_ERROR;                  \
  }

FG_API const char* fg_version(void) { return "fagra_b200 0.1.0 (sm_100a)"; }
FG_API const char* fg_last_error(void) { return t_error.c_str(); }
FG_API uint64_t fg_kernel_launches(void) { return g_launches.load(); }

FG_API fg_status fg_device_count(int* count) {
  if (!count) return FG_NULL_ARGUMENT;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
    return FG_OK;
  }
  *count = n;
  return FG_OK;
}

FG_API fg_status fg_device_stream(int device, void** stream) {
  if (!stream) return FG_NULL_ARGUMENT;
  cudaStream_t s;
  FG_TRY(device_stream(device, &s));
  *stream = (void*)s;
  return FG_OK;
}

FG_API void fg_schur_default_options(fg_schur_options* o) {
  if (!o) return;
  o->max_iterations = 1000;
  o->relative_tolerance = std::max(1e-10, std::numeric_limits<double>::epsilon() * 128.0);
  o->collect_timings = 0;
  o->precision = FG_PRECISION_F64;
  o->preconditioner = FG_PRECOND_RETAINED_BLOCKS;
  o->device = 0;
  o->residual_replacement = 0;  // automatic spacing
  o->operator_variant = 0;
  o->coarse_correction = 0;
  o->learned_policy = 0;
}

FG_API fg_status fg_schur_create(size_t retained, size_t cw, size_t pw, const fg_schur_options* options,
                                 fg_backend** out) {
  if (!out) return FG_NULL_ARGUMENT;
  *out = nullptr;
  FG_GUARD_BEGIN
  fg_schur_options o;
  fg_schur_default_options(&o);
  if (options) o = *options;
  Backend* b = nullptr;
  FG_TRY(make_schur(retained, cw, pw, o, &b));
  *out = new fg_backend{b};
  return FG_OK;
  FG_GUARD_END
}

FG_API void fg_backend_destroy(fg_backend* b) {
  if (!b) return;
  delete b->impl;
  delete b;
}

#define FG_NEED(b) \
  if (!(b) || !(b)->impl) return FG_NULL_ARGUMENT;

FG_API fg_status fg_schur_set_options(fg_backend* b, const fg_schur_options* o) {
  FG_NEED(b);
  if (!o) return FG_NULL_ARGUMENT;
  return b->impl->set_options(*o);
}
FG_API fg_status fg_backend_prepare(fg_backend* b, size_t dim) {
  FG_NEED(b);
  FG_GUARD_BEGIN return b->impl->prepare(dim);
  FG_GUARD_END
}
FG_API fg_status fg_backend_clear(fg_backend* b) {
  FG_NEED(b);
  return b->impl->clear();
}
FG_API fg_status fg_backend_accumulate(fg_backend* b, size_t rows, const double* r, size_t nb, const size_t* cols,
                                       const size_t* widths, const double* const* jac, const ptrdiff_t* rs,
                                       const ptrdiff_t* cs) {
  FG_NEED(b);
  FG_GUARD_BEGIN return b->impl->accumulate(rows, r, nb, cols, widths, jac, rs, cs);
  FG_GUARD_END
}
FG_API fg_status fg_backend_gradient_norm(fg_backend* b, double* out) {
  FG_NEED(b);
  if (!out) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return b->impl->gradient_norm(out);
  FG_GUARD_END
}
FG_API fg_status fg_backend_prepare_damping(fg_backend* b, double floor) {
  FG_NEED(b);
  FG_GUARD_BEGIN return b->impl->prepare_damping(floor);
  FG_GUARD_END
}
FG_API fg_status fg_backend_solve_damped(fg_backend* b, double lambda, const double** delta, size_t* len,
                                         double* predicted) {
  FG_NEED(b);
  FG_GUARD_BEGIN
  double p = 0;
  fg_status s = b->impl->solve_damped(lambda, &p, true);
  if (s != FG_OK) return s;
  if (delta) *delta = b->impl->step_host();
  if (len) *len = b->impl->dimension();
  if (predicted) *predicted = p;
  return FG_OK;
  FG_GUARD_END
}
FG_API fg_status fg_backend_solve_damped_device(fg_backend* b, double lambda, const double** delta,
                                                double* predicted) {
  FG_NEED(b);
  FG_GUARD_BEGIN
  double p = 0;
  fg_status s = b->impl->solve_damped(lambda, &p, false);
  if (s != FG_OK) return s;
  if (delta) *delta = b->impl->step_device();
  if (predicted) *predicted = p;
  return FG_OK;
  FG_GUARD_END
}
FG_API fg_status fg_backend_solve(fg_backend* b, const double** delta, size_t* len) {
  FG_NEED(b);
  FG_GUARD_BEGIN
  FG_TRY(b->impl->solve_undamped(true));
  if (delta) *delta = b->impl->step_host();
  if (len) *len = b->impl->dimension();
  return FG_OK;
  FG_GUARD_END
}
FG_API fg_status fg_backend_linear_solve_work(const fg_backend* b, size_t* solves, size_t* iterations,
                                              int* available) {
  FG_NEED(b);
  size_t s = 0, i = 0;
  b->impl->work(&s, &i);
  if (solves) *solves = s;
  if (iterations) *iterations = i;
  if (available) *available = 1;
  return FG_OK;
}
FG_API fg_status fg_schur_get_diagnostics(const fg_backend* b, fg_schur_diagnostics* d) {
  FG_NEED(b);
  if (!d) return FG_NULL_ARGUMENT;
  b->impl->diagnostics(d);
  return FG_OK;
}
FG_API fg_status fg_schur_get_timings(const fg_backend* b, fg_schur_timings* t) {
  FG_NEED(b);
  if (!t) return FG_NULL_ARGUMENT;
  b->impl->timings(t);
  return FG_OK;
}
FG_API fg_status fg_schur_structure_sizes(fg_backend* b, size_t* nb, size_t* ne, size_t* nv, size_t* nvar,
                                          size_t* rows, size_t* cols) {
  FG_NEED(b);
  FG_GUARD_BEGIN return b->impl->structure_sizes(nb, ne, nv, nvar, rows, cols);
  FG_GUARD_END
}
FG_API fg_status fg_schur_export_structure(fg_backend* b, uint64_t* b5, uint64_t* e4, uint64_t* owners, uint64_t* v3) {
  FG_NEED(b);
  FG_GUARD_BEGIN return b->impl->export_structure(b5, e4, owners, v3);
  FG_GUARD_END
}
FG_API fg_status fg_schur_export_model(fg_backend* b, double* values, double* negres, double* g, double* scales,
                                       double* gram, double* cross) {
  FG_NEED(b);
  FG_GUARD_BEGIN return b->impl->export_model(values, negres, g, scales, gram, cross);
  FG_GUARD_END
}
FG_API fg_status fg_schur_reduced_apply(fg_backend* b, double lambda, const double* x, double* y) {
  FG_NEED(b);
  if (!x || !y) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return b->impl->reduced_apply(lambda, x, y);
  FG_GUARD_END
}

// ---- BAL
static fg_status bal_make(size_t c, size_t p, size_t o, const double* cp, const double* pp, const uint32_t* oc,
                          const uint32_t* op, const double* px, int device, bool on_device, fg_bal_problem** out) {
  if (!out) return FG_NULL_ARGUMENT;
  *out = nullptr;
  if ((c && !cp) || (p && !pp) || (o && (!oc || !op || !px))) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN
  fg_bal_problem* b = new fg_bal_problem();
  fg_status s = b->impl.init(c, p, o, cp, pp, oc, op, px, device, on_device);
  if (s != FG_OK) {
    delete b;
    return s;
  }
  *out = b;
  return FG_OK;
  FG_GUARD_END
}
FG_API fg_status fg_bal_create(size_t c, size_t p, size_t o, const double* cp, const double* pp, const uint32_t* oc,
                               const uint32_t* op, const double* px, int device, fg_bal_problem** out) {
  return bal_make(c, p, o, cp, pp, oc, op, px, device, false, out);
}
FG_API fg_status fg_bal_create_device(size_t c, size_t p, size_t o, const double* cp, const double* pp,
                                      const uint32_t* oc, const uint32_t* op, const double* px, int device,
                                      fg_bal_problem** out) {
  return bal_make(c, p, o, cp, pp, oc, op, px, device, true, out);
}
FG_API void fg_bal_destroy(fg_bal_problem* p) { delete p; }
FG_API fg_status fg_bal_set_parameters(fg_bal_problem* p, const double* cp, const double* pp) {
  if (!p) return FG_NULL_ARGUMENT;
  return p->impl.set_parameters(cp, pp);
}
FG_API fg_status fg_bal_get_parameters(fg_bal_problem* p, double* cp, double* pp) {
  if (!p) return FG_NULL_ARGUMENT;
  return p->impl.get_parameters(cp, pp);
}
FG_API fg_status fg_bal_cost(fg_bal_problem* p, double* out) {
  if (!p || !out) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return p->impl.cost(false, out);
  FG_GUARD_END
}
FG_API fg_status fg_bal_linearize(fg_bal_problem* p, fg_backend* b) {
  if (!p) return FG_NULL_ARGUMENT;
  FG_NEED(b);
  FG_GUARD_BEGIN return p->impl.linearize(b->impl);
  FG_GUARD_END
}

// ---- optimizers
FG_API void fg_optimize_default_options(fg_optimize_options* o) {
  if (!o) return;
  const double eps = std::numeric_limits<double>::epsilon();
  o->max_iterations = 50;
  o->gradient_tolerance = std::max(1e-8, eps * 8.0);
  o->step_tolerance = std::max(1e-10, eps);
  o->cost_tolerance = std::max(1e-12, eps);
}
FG_API void fg_lm_default_options(fg_lm_options* o) {
  if (!o) return;
  o->initial_damping = 1e-3;
  o->min_damping = 1e-12;
  o->max_damping = 1e12;
  o->min_column_norm = 1e-6;
  o->acceptance_threshold = 1e-4;
  o->max_trials = 16;
}
FG_API fg_status fg_lm_solve_bal(fg_backend* b, fg_bal_problem* p, const fg_optimize_options* o,
                                 const fg_lm_options* lo, fg_optimize_report* rep, fg_lm_statistics* st,
                                 fg_accept_callback cb, void* user) {
  FG_NEED(b);
  if (!p || !o || !lo || !rep || !st) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return lm_solve_bal(b->impl, &p->impl, *o, *lo, rep, st, cb, user);
  FG_GUARD_END
}
FG_API fg_status fg_lm_solve_bal_to_cost(fg_backend* b, fg_bal_problem* p, const fg_optimize_options* o,
                                         const fg_lm_options* lo, double target, fg_optimize_report* rep,
                                         fg_lm_statistics* st) {
  FG_NEED(b);
  if (!p || !o || !lo || !rep || !st) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return lm_solve_bal(b->impl, &p->impl, *o, *lo, rep, st, nullptr, nullptr, target);
  FG_GUARD_END
}
FG_API fg_status fg_bal_restore_initial(fg_bal_problem* p) {
  if (!p) return FG_NULL_ARGUMENT;
  return p->impl.restore_initial();
}
FG_API fg_status fg_schur_time_operator_kernel(fg_backend* b, double lambda, size_t reps, double* seconds,
                                               double* bytes) {
  FG_NEED(b);
  if (!seconds || !bytes) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return b->impl->time_operator_kernel(lambda, reps, seconds, bytes);
  FG_GUARD_END
}
FG_API fg_status fg_schur_time_operator(fg_backend* b, double lambda, size_t reps, double* seconds, double* bytes) {
  FG_NEED(b);
  if (!seconds || !bytes) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return b->impl->time_operator(lambda, reps, seconds, bytes);
  FG_GUARD_END
}
FG_API fg_status fg_schur_operator_info(fg_backend* b, int* variant, double* seconds4) {
  FG_NEED(b);
  if (!variant) return FG_NULL_ARGUMENT;
  b->impl->operator_info(variant, seconds4);
  return FG_OK;
}
FG_API fg_status fg_schur_accumulate_pairs_device(fg_backend* b, size_t count, size_t rows,
                                                  const uint32_t* retained_variable,
                                                  const uint32_t* eliminated_variable, const double* residual,
                                                  const double* retained_jacobian,
                                                  const double* eliminated_jacobian) {
  FG_NEED(b);
  FG_GUARD_BEGIN return b->impl->accumulate_pairs(count, rows, retained_variable, eliminated_variable, residual,
                                                  retained_jacobian, eliminated_jacobian);
  FG_GUARD_END
}
FG_API fg_status fg_schur_set_poll_limit(fg_backend* b, unsigned polls) {
  FG_NEED(b);
  FG_GUARD_BEGIN return b->impl->set_poll_limit(polls);
  FG_GUARD_END
}
FG_API fg_status fg_schur_attach_learned(fg_backend* b, fg_gnn* g) {
  FG_NEED(b);
  FG_GUARD_BEGIN return b->impl->attach_learned(g);
  FG_GUARD_END
}
FG_API fg_status fg_schur_capture_system(fg_backend* b, fg_gnn* g, double lambda, size_t probes, uint64_t seed,
                                         int kind, size_t* index) {
  FG_NEED(b);
  if (!g || !index) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return b->impl->capture_system(g, lambda, probes, seed, kind, index);
  FG_GUARD_END
}
FG_API fg_status fg_gn_solve_bal(fg_backend* b, fg_bal_problem* p, const fg_optimize_options* o,
                                 fg_optimize_report* rep) {
  FG_NEED(b);
  if (!p || !o || !rep) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return gn_solve_bal(b->impl, &p->impl, *o, rep);
  FG_GUARD_END
}
FG_API fg_status fg_lm_optimize(fg_backend* b, const fg_problem_callbacks* cb, void* user, double* x,
                                const fg_optimize_options* o, const fg_lm_options* lo, fg_optimize_report* rep,
                                fg_lm_statistics* st) {
  FG_NEED(b);
  if (!cb || !cb->cost || !cb->linearize || (!x && cb->dimension) || !o || !lo || !rep || !st)
    return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return lm_callbacks(b->impl, cb, user, x, *o, *lo, rep, st);
  FG_GUARD_END
}
FG_API fg_status fg_gn_optimize(fg_backend* b, const fg_problem_callbacks* cb, void* user, double* x,
                                const fg_optimize_options* o, fg_optimize_report* rep) {
  FG_NEED(b);
  if (!cb || !cb->cost || !cb->linearize || (!x && cb->dimension) || !o || !rep) return FG_NULL_ARGUMENT;
  FG_GUARD_BEGIN return gn_callbacks(b->impl, cb, user, x, *o, rep);
  FG_GUARD_END
}
