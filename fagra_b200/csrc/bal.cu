// Device BAL problem: fagra's examples/bal/model.rs (Projection, Frame batch per
// camera) with the Stage/Accept/Reject transaction of src/optimization.rs:432-487
// kept on the device. Observations are stored in emission order.
#include "bal.cuh"
#include "kernels.cuh"
#include "sort.cuh"
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>

namespace fg {

namespace {
std::atomic<uint64_t> g_next_id{1};
}

// Per camera: rotation R (row major) from the unit quaternion exp(w/2)
// (nalgebra UnitQuaternion::from_scaled_axis + to_rotation_matrix) and the
// additive angle-axis right factor I - aK + bK^2 (model.rs:126-146).
__global__ void k_bal_camera_prep(int64_t nc, const double* cams, double* prep) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double* w = cams + 9 * c;
  double v0 = w[0] / 2, v1 = w[1] / 2, v2 = w[2] / 2;
  double nn = v0 * v0 + v1 * v1 + v2 * v2;
  const double eps = 2.220446049250313e-16;
  double qw, qi, qj, qk;
  if (nn <= eps * eps) {
    qw = 1; qi = qj = qk = 0;
  } else {
    double n = sqrt(nn), s = sin(n) / n;
    qw = cos(n); qi = v0 * s; qj = v1 * s; qk = v2 * s;
  }
  double ww = qw * qw, ii = qi * qi, jj = qj * qj, kk = qk * qk;
  double ij = qi * qj * 2, wk = qw * qk * 2, wj = qw * qj * 2, ik = qi * qk * 2, jk = qj * qk * 2, wi = qw * qi * 2;
  double* R = prep + 18 * c;
  R[0] = ww + ii - jj - kk; R[1] = ij - wk; R[2] = wj + ik;
  R[3] = wk + ij; R[4] = ww - ii + jj - kk; R[5] = jk - wi;
  R[6] = ik - wj; R[7] = wi + jk; R[8] = ww - ii - jj + kk;
  double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double a, b;
  if (t2 < 1e-8) {
    a = 0.5 - t2 / 24. + t2 * t2 / 720.;
    b = 1. / 6. - t2 / 120. + t2 * t2 / 5040.;
  } else {
    double t = sqrt(t2);
    a = (1. - cos(t)) / t2;
    b = (t - sin(t)) / (t2 * t);
  }
  double K[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
  double* Rt = prep + 18 * c + 9;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double k2 = 0;
      for (int k = 0; k < 3; ++k) k2 += K[3 * i + k] * K[3 * k + j];
      Rt[3 * i + j] = (i == j ? 1.0 : 0.0) - a * K[3 * i + j] + b * k2;
    }
}

// Camera part of the 7 similarity-gauge directions of bundle adjustment, in
// the Jacobian's own coordinates (additive angle-axis w, translation t,
// intrinsics): the reprojection residuals are invariant under X -> s Q X + d
// with the cameras moved to R Q^T, s t - R Q^T d, so to first order
//   rotation about world axis k:   dw = -J_r(w)^-1 e_k,  dt = 0
//   translation along k:           dw = 0,              dt = -R e_k
//   scale:                         dw = 0,              dt = t
// with J_r(w) the right factor of the camera prep (the rotation Jacobian
// d(R X)/dw = -R [X]x J_r(w) of k_bal_linearize). basis[j * 9nc + 9c + i].
__global__ void k_bal_gauge(int64_t nc, const double* cams, const double* prep, double* basis) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double* R = prep + 18 * c;
  const double* J = R + 9;
  const double* t = cams + 9 * c + 3;
  const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                     J[2] * (J[3] * J[7] - J[4] * J[6]);
  double inv[9] = {J[4] * J[8] - J[5] * J[7], J[2] * J[7] - J[1] * J[8], J[1] * J[5] - J[2] * J[4],
                   J[5] * J[6] - J[3] * J[8], J[0] * J[8] - J[2] * J[6], J[2] * J[3] - J[0] * J[5],
                   J[3] * J[7] - J[4] * J[6], J[1] * J[6] - J[0] * J[7], J[0] * J[4] - J[1] * J[3]};
  const int64_t n = 9 * nc;
  for (int j = 0; j < 7; ++j) {
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (j < 3) {
      for (int i = 0; i < 3; ++i) v[i] = -inv[3 * i + j] / det;
    } else if (j < 6) {
      for (int i = 0; i < 3; ++i) v[3 + i] = -R[3 * i + (j - 3)];
    } else {
      for (int i = 0; i < 3; ++i) v[3 + i] = t[i];
    }
    for (int i = 0; i < 9; ++i) basis[j * n + 9 * c + i] = v[i];
  }
}

// Reprojection residual and Jacobians (model.rs:157-185, 214-236) for every
// observation k in emission order, written in the packed block layout:
// values[24k .. 24k+18) = camera block (2x9 column major), [24k+18, 24k+24) =
// point block (2x3 column major), negres[2k..2k+1] = -r.
// Block of LIN_T observations; the 24 values of each are staged in shared
// memory (stride 25 words to spread banks) and stored with coalesced writes.
constexpr int LIN_T = 128;
template <class TS>
__global__ void __launch_bounds__(LIN_T) k_bal_linearize(int64_t no, const uint32_t* oc, const uint32_t* op,
                                                         const double* px, const double* cams, const double* pts,
                                                         const double* prep, TS* values, double* negres, int* error) {
  __shared__ TS tile[LIN_T * 25];
  __shared__ double nr[LIN_T * 2];
  const int64_t k0 = (int64_t)blockIdx.x * LIN_T;
  const int64_t k = k0 + threadIdx.x;
  const int nk = (int)min((int64_t)LIN_T, no - k0);
  if (k < no) {
  uint32_t c = oc[k], pi = op[k];
  const double* cam = cams + 9 * (int64_t)c;
  const double* R = prep + 18 * (int64_t)c;
  const double* right = R + 9;
  double X[3] = {pts[3 * (int64_t)pi], pts[3 * (int64_t)pi + 1], pts[3 * (int64_t)pi + 2]};
  ObsEval o = bal_eval(R, cam, X);
  double r[2] = {o.pixel[0] - px[2 * k], o.pixel[1] - px[2 * k + 1]};
  double f = cam[6], k1 = cam[7], k2 = cam[8];
  double cc = 2. * k1 + 4. * k2 * o.r2;
  double dq0 = f * (o.radial + cc * o.q[0] * o.q[0]), dq1 = f * (cc * o.q[0] * o.q[1]);
  double dq2 = f * (cc * o.q[1] * o.q[0]), dq3 = f * (o.radial + cc * o.q[1] * o.q[1]);
  double iz = -1. / o.p[2], iz2x = o.p[0] / (o.p[2] * o.p[2]), iz2y = o.p[1] / (o.p[2] * o.p[2]);
  // dp = dq * [[-1/z, 0, x/z^2], [0, -1/z, y/z^2]]
  double dp[6] = {dq0 * iz, dq1 * iz, dq0 * iz2x + dq1 * iz2y, dq2 * iz, dq3 * iz, dq2 * iz2x + dq3 * iz2y};
  // t1 = dp * (-R); t2 = t1 * skew(X); t3 = t2 * right
  double K[9] = {0, -X[2], X[1], X[2], 0, -X[0], -X[1], X[0], 0};
  double t1[6], t2[6], t3[6];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) {
      double s1 = 0;
      for (int m = 0; m < 3; ++m) s1 += dp[3 * i + m] * -R[3 * m + j];
      t1[3 * i + j] = s1;
    }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) {
      double s2 = 0;
      for (int m = 0; m < 3; ++m) s2 += t1[3 * i + m] * K[3 * m + j];
      t2[3 * i + j] = s2;
    }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) {
      double s3 = 0;
      for (int m = 0; m < 3; ++m) s3 += t2[3 * i + m] * right[3 * m + j];
      t3[3 * i + j] = s3;
    }
  double jc[18], jp[6];
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 2; ++i) {
      jc[2 * j + i] = t3[3 * i + j];
      jc[2 * (3 + j) + i] = dp[3 * i + j];
    }
  for (int i = 0; i < 2; ++i) {
    jc[12 + i] = o.radial * o.q[i];
    jc[14 + i] = f * o.r2 * o.q[i];
    jc[16 + i] = f * o.r2 * o.r2 * o.q[i];
  }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int m = 0; m < 3; ++m) s += dp[3 * i + m] * R[3 * m + j];
      jp[2 * j + i] = s;
    }
  bool ok = o.ok && isfinite(r[0]) && isfinite(r[1]);
  TS* v = tile + threadIdx.x * 25;
  for (int i = 0; i < 18; ++i) {
    v[i] = (TS)jc[i];
    ok = ok && isfinite(jc[i]);
  }
  for (int i = 0; i < 6; ++i) {
    v[18 + i] = (TS)jp[i];
    ok = ok && isfinite(jp[i]);
  }
  nr[2 * threadIdx.x] = -r[0];
  nr[2 * threadIdx.x + 1] = -r[1];
  if (!ok) atomicOr(error, 1);
  }
  __syncthreads();
  TS* out = values + 24 * k0;
  for (int i = threadIdx.x; i < nk * 24; i += LIN_T) out[i] = tile[(i / 24) * 25 + (i % 24)];
  for (int i = threadIdx.x; i < nk * 2; i += LIN_T) negres[2 * k0 + i] = nr[i];
}

// Sum of 0.5 |r|^2 over observations (Frame::cost) in double-double, with
// an error flag for invalid projections. out[0] = cost, out[1] = error.
__global__ void k_bal_cost(int64_t no, const uint32_t* oc, const uint32_t* op, const double* px, const double* cams,
                           const double* pts, const double* prep, double* partials, unsigned* counter, double* out) {
  double hi = 0, lo = 0, bad = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < no; k += (int64_t)gridDim.x * blockDim.x) {
    uint32_t c = oc[k], pi = op[k];
    double X[3] = {pts[3 * (int64_t)pi], pts[3 * (int64_t)pi + 1], pts[3 * (int64_t)pi + 2]};
    ObsEval o = bal_eval(prep + 18 * (int64_t)c, cams + 9 * (int64_t)c, X);
    double r0 = o.pixel[0] - px[2 * k], r1 = o.pixel[1] - px[2 * k + 1];
    double v = 0.5 * (r0 * r0 + r1 * r1);
    if (!o.ok || !isfinite(v)) bad = 1;
    else dd_add(hi, lo, v, 0.0);
  }
  for (int o = 16; o > 0; o >>= 1) {
    double h2 = __shfl_down_sync(0xffffffffu, hi, o), l2 = __shfl_down_sync(0xffffffffu, lo, o);
    double b2 = __shfl_down_sync(0xffffffffu, bad, o);
    dd_add(hi, lo, h2, l2);
    bad = fmax(bad, b2);
  }
  __shared__ double sh[32][3];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { sh[warp][0] = hi; sh[warp][1] = lo; sh[warp][2] = bad; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int nw = (blockDim.x + 31) >> 5;
    for (int w = 1; w < nw; ++w) {
      dd_add(hi, lo, sh[w][0], sh[w][1]);
      bad = fmax(bad, sh[w][2]);
    }
    partials[3 * blockIdx.x] = hi;
    partials[3 * blockIdx.x + 1] = lo;
    partials[3 * blockIdx.x + 2] = bad;
  }
  if (arrive_last(counter)) {
    // the last block folds the per-block partials: thread-strided in
    // double-double, then the same fixed shuffle / shared-memory tree
    double H = 0, Lo = 0, B = 0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
      dd_add(H, Lo, ((volatile double*)partials)[3 * b], ((volatile double*)partials)[3 * b + 1]);
      B = fmax(B, ((volatile double*)partials)[3 * b + 2]);
    }
    for (int o = 16; o > 0; o >>= 1) {
      double h2 = __shfl_down_sync(0xffffffffu, H, o), l2 = __shfl_down_sync(0xffffffffu, Lo, o);
      double b2 = __shfl_down_sync(0xffffffffu, B, o);
      dd_add(H, Lo, h2, l2);
      B = fmax(B, b2);
    }
    __syncthreads();
    if (lane == 0) { sh[warp][0] = H; sh[warp][1] = Lo; sh[warp][2] = B; }
    __syncthreads();
    if (threadIdx.x == 0) {
      int nw = (blockDim.x + 31) >> 5;
      for (int w = 1; w < nw; ++w) {
        dd_add(H, Lo, sh[w][0], sh[w][1]);
        B = fmax(B, sh[w][2]);
      }
      out[0] = H + Lo;
      out[1] = B;
      *counter = 0;
    }
  }
}

// Trial retraction x + delta for additive Camera/Point variables.
__global__ void k_bal_stage(int64_t nc9, int64_t np3, const double* cams, const double* pts, const double* delta,
                            double* tcams, double* tpts) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < nc9) tcams[i] = cams[i] + delta[i];
  else if (i < nc9 + np3) tpts[i - nc9] = pts[i - nc9] + delta[i];
}

// Per-device staging of problem ingestion: the raw observations and the sort
// scratch, reused by every problem created on the device (allocated once, kept
// for the life of the process).
struct Ingest {
  std::mutex m;
  DBuf<uint32_t> cam, pt, order;
  DBuf<double> pix;
  DBuf<int> bad;
  HBuf<int> h_bad;
  SortScratch sort;
};
Ingest& ingest(int dev) {
  static std::mutex g;
  static std::map<int, Ingest*> pools;
  std::lock_guard<std::mutex> lock(g);
  Ingest*& p = pools[dev];
  if (!p) p = new Ingest();
  return *p;
}

// Observation checks of examples/bal/model.rs:78-79 (indices in range, finite
// pixels): any failure sets *bad.
__global__ void k_bal_validate(int64_t o, uint32_t nc, uint32_t np, const uint32_t* cam, const uint32_t* pt,
                               const double2* pix, int* bad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= o) return;
  const double2 x = pix[i];
  if (cam[i] >= nc || pt[i] >= np || !isfinite(x.x) || !isfinite(x.y)) *bad = 1;
}

// Emission k takes insertion index order[k]: camera, point and pixels.
__global__ void k_bal_gather(int64_t o, const uint32_t* order, const uint32_t* rc, const uint32_t* rp,
                             const double2* rx, uint32_t* oc, uint32_t* op, double2* px) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= o) return;
  const uint32_t i = order[k];
  oc[k] = rc[i];
  op[k] = rp[i];
  px[k] = rx[i];
}

fg_status BalProblem::init(size_t c, size_t p, size_t o, const double* cp, const double* pp, const uint32_t* ocam,
                           const uint32_t* opt, const double* pix, int device, bool on_device) {
  id = g_next_id.fetch_add(1);
  dev = device;
  nc = c; np = p; no = o;
  FG_TRY(select_device(dev));
  FG_TRY(device_stream(dev, &st));
  nsm = sm_count(dev);
  if (c >= ((size_t)1 << 32) || p >= ((size_t)1 << 32) || o >= ((size_t)1 << 32)) {
    set_error("BAL problem sizes must be below 2^32");
    return FG_INVALID_EMISSION;
  }
  const auto kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  // Problem storage comes from the library pool in the library stream's order:
  // creating and destroying problems maps and unmaps no device memory.
  oc.use_pool(dev, st);
  op.use_pool(dev, st);
  for (DBuf<double>* b : {&px, &cams, &pts, &tcams, &tpts, &prep, &tprep, &partials, &result, &init_cams, &init_pts,
                          &gauge})
    b->use_pool(dev, st);
  counters.use_pool(dev, st);
  d_flag.use_pool(dev, st);
  FG_TRY(oc.resize(std::max<size_t>(o, 1)));
  FG_TRY(op.resize(std::max<size_t>(o, 1)));
  FG_TRY(px.resize(std::max<size_t>(2 * o, 1)));
  if (o) {
    // Emission order: frames in camera order, factors in insertion order (a
    // stable order by camera); validated and gathered on the device.
    Ingest& in = ingest(dev);
    std::lock_guard<std::mutex> lock(in.m);
    FG_TRY(in.cam.resize(o));
    FG_TRY(in.pt.resize(o));
    FG_TRY(in.order.resize(o));
    FG_TRY(in.pix.resize(2 * o));
    FG_TRY(in.bad.resize(1));
    FG_TRY(in.h_bad.resize(1));
    FG_CUDA(cudaMemsetAsync(in.bad.get(), 0, sizeof(int), st));
    FG_CUDA(cudaMemcpyAsync(in.cam.get(), ocam, o * sizeof(uint32_t), kind, st));
    FG_CUDA(cudaMemcpyAsync(in.pt.get(), opt, o * sizeof(uint32_t), kind, st));
    FG_CUDA(cudaMemcpyAsync(in.pix.get(), pix, 2 * o * sizeof(double), kind, st));
    const double2* raw = reinterpret_cast<const double2*>(in.pix.get());
    FG_LAUNCH(k_bal_validate, grid_for(o, 256), 256, 0, st, (int64_t)o, (uint32_t)nc, (uint32_t)np, in.cam.get(),
              in.pt.get(), raw, in.bad.get());
    FG_TRY(stable_order(in.cam.get(), o, (uint32_t)nc, in.order.get(), nullptr, in.sort, st));
    FG_LAUNCH(k_bal_gather, grid_for(o, 256), 256, 0, st, (int64_t)o, in.order.get(), in.cam.get(), in.pt.get(), raw,
              oc.get(), op.get(), reinterpret_cast<double2*>(px.get()));
    FG_CUDA(cudaMemcpyAsync(in.h_bad.get(), in.bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));  // the staging is free for the next problem after this
    if (in.h_bad.get()[0]) {
      set_error("invalid observation index or value");
      return FG_INVALID_EMISSION;
    }
  }
  FG_TRY(cams.resize(std::max<size_t>(9 * nc, 1)));
  FG_TRY(pts.resize(std::max<size_t>(3 * np, 1)));
  FG_TRY(tcams.resize(std::max<size_t>(9 * nc, 1)));
  FG_TRY(tpts.resize(std::max<size_t>(3 * np, 1)));
  FG_TRY(prep.resize(std::max<size_t>(18 * nc, 1)));
  FG_TRY(tprep.resize(std::max<size_t>(18 * nc, 1)));
  FG_TRY(partials.resize(3 * 4096));
  FG_TRY(counters.resize(4));
  FG_TRY(result.resize(4));
  FG_TRY(h_result.resize(4));
  FG_TRY(h_flag.resize(2));
  FG_TRY(d_flag.resize(2));
  FG_CUDA(cudaMemsetAsync(counters.get(), 0, 4 * sizeof(unsigned), st));
  if (nc) FG_CUDA(cudaMemcpyAsync(cams.get(), cp, 9 * nc * sizeof(double), kind, st));
  if (np) FG_CUDA(cudaMemcpyAsync(pts.get(), pp, 3 * np * sizeof(double), kind, st));
  FG_TRY(init_cams.resize(std::max<size_t>(9 * nc, 1)));
  FG_TRY(init_pts.resize(std::max<size_t>(3 * np, 1)));
  if (nc) FG_CUDA(cudaMemcpyAsync(init_cams.get(), cams.get(), 9 * nc * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (np) FG_CUDA(cudaMemcpyAsync(init_pts.get(), pts.get(), 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st));
  FG_CUDA(cudaStreamSynchronize(st));
  return FG_OK;
}

fg_status BalProblem::host_observations(const uint32_t** cam, const uint32_t** pt) {
  if (!host_obs) {
    h_oc.resize(no);
    h_op.resize(no);
    if (no) {
      FG_CUDA(cudaMemcpyAsync(h_oc.data(), oc.get(), no * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      FG_CUDA(cudaMemcpyAsync(h_op.data(), op.get(), no * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      FG_CUDA(cudaStreamSynchronize(st));
    }
    host_obs = true;
  }
  *cam = h_oc.data();
  *pt = h_op.data();
  return FG_OK;
}

fg_status BalProblem::restore_initial() {
  if (nc) FG_CUDA(cudaMemcpyAsync(cams.get(), init_cams.get(), 9 * nc * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (np) FG_CUDA(cudaMemcpyAsync(pts.get(), init_pts.get(), 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st));
  FG_CUDA(cudaStreamSynchronize(st));
  trial_active = false;
  return FG_OK;
}

fg_status BalProblem::set_parameters(const double* cp, const double* pp) {
  if (nc) FG_CUDA(cudaMemcpyAsync(cams.get(), cp, 9 * nc * sizeof(double), cudaMemcpyHostToDevice, st));
  if (np) FG_CUDA(cudaMemcpyAsync(pts.get(), pp, 3 * np * sizeof(double), cudaMemcpyHostToDevice, st));
  FG_CUDA(cudaStreamSynchronize(st));
  trial_active = false;
  return FG_OK;
}

fg_status BalProblem::get_parameters(double* cp, double* pp) {
  if (cp && nc) FG_CUDA(cudaMemcpyAsync(cp, cams.get(), 9 * nc * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (pp && np) FG_CUDA(cudaMemcpyAsync(pp, pts.get(), 3 * np * sizeof(double), cudaMemcpyDeviceToHost, st));
  FG_CUDA(cudaStreamSynchronize(st));
  return FG_OK;
}

fg_status BalProblem::cost(bool trial, double* out) {
  const double* C = trial ? tcams.get() : cams.get();
  const double* P = trial ? tpts.get() : pts.get();
  double* R = trial ? tprep.get() : prep.get();
  if (nc) FG_LAUNCH(k_bal_camera_prep, grid_for(nc, 128), 128, 0, st, (int64_t)nc, C, R);
  unsigned g = std::min<unsigned>(grid_for(std::max<size_t>(no, 1), 256), 4 * nsm);
  FG_LAUNCH(k_bal_cost, g, 256, 0, st, (int64_t)no, oc.get(), op.get(), px.get(), C, P, R, partials.get(),
            counters.get(), result.get());
  FG_CUDA(cudaMemcpyAsync(h_result.get(), result.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  FG_CUDA(cudaStreamSynchronize(st));
  double c = h_result.get()[0];
  if (h_result.get()[1] != 0 || !std::isfinite(c) || c < 0) {  // checked_cost, storage.rs:612-618
    set_error("invalid BAL evaluation");
    return FG_INVALID_EVALUATION;
  }
  *out = c;
  return FG_OK;
}

fg_status BalProblem::linearize(Backend* b) {
  FG_TRY(b->clear());
  BalObservations ob;
  ob.problem_id = id;
  ob.cameras = nc;
  ob.points = np;
  ob.observations = no;
  ob.cam = oc.get();
  ob.pt = op.get();
  ob.host = [this](const uint32_t** c, const uint32_t** p) { return host_observations(c, p); };
  FG_TRY(b->bind_bal(ob));
  if (nc) FG_LAUNCH(k_bal_camera_prep, grid_for(nc, 128), 128, 0, st, (int64_t)nc, cams.get(), prep.get());
  FG_CUDA(cudaMemsetAsync(d_flag.get(), 0, sizeof(int), st));
  if (no) {
    if (b->is_f32()) {
      FG_LAUNCH(k_bal_linearize<float>, grid_for(no, LIN_T), LIN_T, 0, st, (int64_t)no, oc.get(), op.get(), px.get(),
                cams.get(), pts.get(), prep.get(), (float*)b->values_device(), b->negres_device(), d_flag.get());
    } else {
      FG_LAUNCH(k_bal_linearize<double>, grid_for(no, LIN_T), LIN_T, 0, st, (int64_t)no, oc.get(), op.get(), px.get(),
                cams.get(), pts.get(), prep.get(), (double*)b->values_device(), b->negres_device(), d_flag.get());
    }
  }
  FG_CUDA(cudaMemcpyAsync(h_flag.get(), d_flag.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  FG_CUDA(cudaStreamSynchronize(st));
  b->mark_device_model(2 * no);
  if (nc) {  // the gauge directions at these estimates, for two-level PCG
    FG_TRY(gauge.resize(7 * 9 * nc));
    FG_LAUNCH(k_bal_gauge, grid_for(nc, 128), 128, 0, st, (int64_t)nc, cams.get(), prep.get(), gauge.get());
    FG_TRY(b->set_coarse_basis(gauge.get(), 7));
  }
  if (h_flag.get()[0]) {
    set_error("invalid BAL linearization");
    return FG_INVALID_EVALUATION;
  }
  return FG_OK;
}

fg_status BalProblem::stage(const double* d_delta) {
  size_t n = 9 * nc + 3 * np;
  if (n) FG_LAUNCH(k_bal_stage, grid_for(n, 256), 256, 0, st, (int64_t)(9 * nc), (int64_t)(3 * np), cams.get(),
                   pts.get(), d_delta, tcams.get(), tpts.get());
  trial_active = true;
  return FG_OK;
}

fg_status BalProblem::stage_and_cost_device(const double* d_delta) {
  FG_TRY(stage(d_delta));
  if (nc) FG_LAUNCH(k_bal_camera_prep, grid_for(nc, 128), 128, 0, st, (int64_t)nc, tcams.get(), tprep.get());
  unsigned g = std::min<unsigned>(grid_for(std::max<size_t>(no, 1), 256), 4 * nsm);
  FG_LAUNCH(k_bal_cost, g, 256, 0, st, (int64_t)no, oc.get(), op.get(), px.get(), tcams.get(), tpts.get(),
            tprep.get(), partials.get(), counters.get(), result.get());
  return FG_OK;
}

void BalProblem::accept() {
  if (trial_active) {
    std::swap(cams.ptr, tcams.ptr);
    std::swap(cams.cap, tcams.cap);
    std::swap(pts.ptr, tpts.ptr);
    std::swap(pts.cap, tpts.cap);
    trial_active = false;
  }
}

void BalProblem::reject() { trial_active = false; }

}  // namespace fg
