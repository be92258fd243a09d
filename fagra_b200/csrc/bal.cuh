// Device-resident BAL problem (examples/bal/model.rs) with transactional trials.
#pragma once
#include "common.cuh"
#include "schur.cuh"

namespace fg {

// Projection of one observation (examples/bal/model.rs:147-156) from the
// per-camera rotation R (row major) and camera parameters.
struct ObsEval {
  double p[3], q[2], r2, radial, pixel[2];
  bool ok;
};
__device__ __forceinline__ ObsEval bal_eval(const double* R, const double* cam, const double* X) {
  ObsEval o;
  for (int i = 0; i < 3; ++i) o.p[i] = R[3 * i] * X[0] + R[3 * i + 1] * X[1] + R[3 * i + 2] * X[2] + cam[3 + i];
  o.q[0] = -o.p[0] / o.p[2];
  o.q[1] = -o.p[1] / o.p[2];
  o.r2 = o.q[0] * o.q[0] + o.q[1] * o.q[1];
  o.radial = 1. + cam[7] * o.r2 + cam[8] * o.r2 * o.r2;
  double s = cam[6] * o.radial;
  o.pixel[0] = s * o.q[0];
  o.pixel[1] = s * o.q[1];
  o.ok = !(o.p[2] == 0.) && isfinite(o.pixel[0]) && isfinite(o.pixel[1]);
  return o;
}

// Error-free addition (Knuth TwoSum) for compensated cost reductions.
__device__ __forceinline__ void two_sum(double a, double b, double* s, double* e) {
  double x = a + b;
  double bv = x - a;
  double av = x - bv;
  *s = x;
  *e = (a - av) + (b - bv);
}
__device__ __forceinline__ void dd_add(double& hi, double& lo, double bhi, double blo) {
  double s, e;
  two_sum(hi, bhi, &s, &e);
  e += lo + blo;
  two_sum(s, e, &hi, &lo);
}

// Per-camera rotation and right factor (defined in bal.cu).
__global__ void k_bal_camera_prep(int64_t nc, const double* cams, double* prep);

struct BalProblem {
  uint64_t id = 0;
  int dev = 0, nsm = 148;
  cudaStream_t st = nullptr;
  size_t nc = 0, np = 0, no = 0;
  std::vector<uint32_t> h_oc, h_op;  // host copies of oc and op, downloaded on first use
  bool host_obs = false;
  DBuf<uint32_t> oc, op;
  DBuf<double> px, cams, pts, tcams, tpts, prep, tprep, partials, result, init_cams, init_pts, gauge;
  DBuf<unsigned> counters;
  DBuf<int> d_flag;
  // device LM trials: the trial state (lm.cuh LmTrialState) and the step norm
  DBuf<double> lm_state;
  HBuf<double> h_lm_state;
  HBuf<double> h_result;
  HBuf<int> h_flag;
  bool trial_active = false;

  fg_status init(size_t c, size_t p, size_t o, const double* cp, const double* pp, const uint32_t* ocam,
                 const uint32_t* opt, const double* pix, int device, bool on_device);
  fg_status set_parameters(const double* cp, const double* pp);
  fg_status get_parameters(double* cp, double* pp);
  fg_status cost(bool trial, double* out);
  fg_status linearize(Backend* b);
  fg_status host_observations(const uint32_t** cam, const uint32_t** pt);
  fg_status stage(const double* d_delta);
  // stage + trial cost enqueued without a sync; [cost, invalid] at result
  fg_status stage_and_cost_device(const double* d_delta);
  void accept();
  void reject();
  fg_status restore_initial();
  size_t dimension() const { return 9 * nc + 3 * np; }
};

}  // namespace fg

struct fg_bal_problem {
  fg::BalProblem impl;
};
