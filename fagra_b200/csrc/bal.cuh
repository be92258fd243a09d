// Device-resident BAL problem (examples/bal/model.rs) with transactional trials.
#pragma once
#include "common.cuh"
#include "schur.cuh"

namespace fg {

struct BalProblem {
  uint64_t id = 0;
  int dev = 0, nsm = 148;
  cudaStream_t st = nullptr;
  size_t nc = 0, np = 0, no = 0;
  std::vector<size_t> order;  // emission position -> insertion index
  std::vector<uint32_t> h_oc, h_op;
  DBuf<uint32_t> oc, op;
  DBuf<double> px, cams, pts, tcams, tpts, prep, tprep, partials, result, init_cams, init_pts;
  DBuf<unsigned> counters;
  DBuf<int> d_flag;
  HBuf<double> h_result;
  HBuf<int> h_flag;
  bool trial_active = false;

  fg_status init(size_t c, size_t p, size_t o, const double* cp, const double* pp, const uint32_t* ocam,
                 const uint32_t* opt, const double* pix, int device, bool on_device);
  fg_status set_parameters(const double* cp, const double* pp);
  fg_status get_parameters(double* cp, double* pp);
  fg_status cost(bool trial, double* out);
  fg_status linearize(Backend* b);
  fg_status stage(const double* d_delta);
  void accept();
  void reject();
  fg_status restore_initial();
  size_t dimension() const { return 9 * nc + 3 * np; }
};

}  // namespace fg

struct fg_bal_problem {
  fg::BalProblem impl;
};
