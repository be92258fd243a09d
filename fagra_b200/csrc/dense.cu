// Dense direct backends on the device, behind the same LeastSquaresBackend
// entry points as the sparse ones:
//   DenseNormalCholesky (src/normal.rs:65-392): lower J^T J and -J^T r, LLT,
//     LM damping lambda * max(sqrt(H_jj), floor)^2, information factor with the
//     pivot rank screen;
//   DenseSchur (src/dense_schur.rs:92-401): scaled normal equations, damping
//     lambda I in scaled coordinates, landmark / retained partition checks.
//     The device factors the whole scaled system with the landmark
//     coordinates ordered first: its Cholesky factor is then exactly the
//     per-landmark factors followed by the factor of the reduced retained
//     system S = B - E C^-1 E^T that the reference forms, so success, the
//     rank screen and the retained covariance follow the reference's
//     elimination;
//   DenseQr (src/qr.rs:65-242): column-pivoted Householder QR of
//     [J D^-1 | -r; sqrt(lambda) I] (or [J | -r] undamped), rank cutoff,
//     back substitution;
//   selected covariance (src/covariance.rs:225-255): Sigma = Y^T Y with
//     L Y = D^-1 E_sel from the (scaled) information factor.
// Emissions are packed on the host exactly as LinearizedModel::accumulate
// (src/linear_model.rs:180-210), which also keeps the gradient in the
// reference's summation order. J^T J is assembled on the device from the
// packed blocks; factorizations and solves run in one CTA per system
// (dense.cuh), sized for the bounded systems these backends are meant for.
#include "common.cuh"
#include "schur.cuh"
#include "dense.cuh"
#include <algorithm>
#include <set>
#include <memory>

namespace fg {

namespace {
enum { DK_NORMAL = 0, DK_SCHUR = 1, DK_QR = 2 };
enum { DM_NORMAL_SOLVE = 0, DM_NORMAL_DAMPED = 1, DM_SCHUR_DAMPED = 2, DM_INFO = 3, DM_SCHUR_INFO = 4 };
constexpr int DCB = 32;
}  // namespace

// Lower J^T J: one CTA per block pair of an emission; duplicates add.
__global__ void k_dense_pairs(const int64_t* blocks5, const int64_t* pairs, const double* values, double* N,
                              int64_t n, const int64_t* perm) {
  const int64_t a = pairs[2 * blockIdx.x], b = pairs[2 * blockIdx.x + 1];
  const int64_t* A = blocks5 + 5 * a;
  const int64_t* B = blocks5 + 5 * b;
  const int64_t rows = A[2], ca = A[3], cb = B[3];
  for (int64_t e = threadIdx.x; e < ca * cb; e += blockDim.x) {
    const int64_t i = e % ca, j = e / ca;
    if (a == b && i < j) continue;
    double v = 0;
    for (int64_t k = 0; k < rows; ++k) v += values[A[4] + i * rows + k] * values[B[4] + j * rows + k];
    int64_t r = A[1] + i, c = B[1] + j;
    if (perm) {
      r = perm[r];
      c = perm[c];
    }
    const int64_t hi = r > c ? r : c, lo = r > c ? c : r;
    atomicAdd(&N[lo * n + hi], v);
  }
}

// Column scales max(sqrt(N_cc), floor); out[0] = 1 if a lower entry is
// nonfinite, out[1] = 1 if a diagonal entry is negative.
__global__ void k_dense_scales(const double* N, int64_t n, double floor, const int64_t* perm, double* scales,
                               double* out) {
  __shared__ double red[WNT / 32];
  double bad = 0, neg = 0;
  for (int64_t c = threadIdx.x; c < n; c += WNT) {
    const int64_t pc = perm ? perm[c] : c;
    const double d = N[pc * n + pc];
    if (!isfinite(d)) bad = 1;
    if (d < 0) neg = 1;
    scales[c] = fmax(sqrt(fmax(d, 0.0)), floor);
  }
  for (int64_t e = threadIdx.x; e < n * n; e += WNT) {
    const int64_t r = e % n, c = e / n;
    if (r >= c && !isfinite(N[e])) bad = 1;
  }
  bad = wmax(bad, red);
  neg = wmax(neg, red);
  if (threadIdx.x == 0) {
    out[0] = bad;
    out[1] = neg;
  }
}

struct DenseArgs {
  const double* N;  // lower J^T J (coordinates permuted by perm when given)
  double* F;        // factor workspace (n*n)
  int64_t n;
  const double* rhs;     // NORMAL: -J^T r; SCHUR: gradient g
  const double* scales;  // per original coordinate
  const int64_t* perm;   // original coordinate -> factor position (SCHUR), or null
  double lambda;
  double* step;          // original coordinates
  double* work;          // n doubles
  double* diag;          // n doubles: original diagonal (information factor)
  double tol;            // rank screen tolerance
  double* out;           // [status, predicted, nonfinite step]
};

// Single-CTA dense factor + solve.
__global__ void __launch_bounds__(WNT) k_dense_solve(DenseArgs A, int mode) {
  extern __shared__ __align__(16) double dsm[];
  __shared__ double red[WNT / 32];
  __shared__ int flag;
  const int tid = threadIdx.x;
  const int64_t n = A.n;
  double* F = A.F;
  if (tid == 0) flag = 0;
  // Factor input: lower triangle of the (scaled) matrix plus damping.
  double bad = 0;
  for (int64_t e = tid; e < n * n; e += WNT) {
    const int64_t r = e % n, c = e / n;
    if (r < c) continue;
    double v = A.N[e];
    if (mode == DM_SCHUR_DAMPED || mode == DM_SCHUR_INFO) {
      // position -> original coordinate for the scales
      v = v / (A.work[r] * A.work[c]);
      if (r == c) v += A.lambda;
    } else if (mode == DM_NORMAL_DAMPED && r == c) {
      const double d = sqrt(A.lambda) * A.scales[r];
      v += d * d;
    }
    if (!isfinite(v)) bad = 1;
    F[e] = v;
  }
  bad = wmax(bad, red);
  double status = 0;
  if (bad != 0) status = (mode == DM_NORMAL_DAMPED) ? FG_LINEAR_SOLVE_FAILED : FG_INVALID_EVALUATION;
  if (status == 0 && (mode == DM_INFO || mode == DM_SCHUR_INFO)) {
    for (int64_t c = tid; c < n; c += WNT) A.diag[c] = F[c * n + c];
  }
  __syncthreads();
  bool ok = status == 0 && cta_cholesky<double, DCB>(F, (int)n, (int)n, dsm, &flag, nullptr);
  __syncthreads();
  if (status == 0 && !ok) status = FG_LINEAR_SOLVE_FAILED;
  if (status == 0 && (mode == DM_INFO || mode == DM_SCHUR_INFO)) {
    // information_factor (normal.rs:367-392) / check_rank (dense_schur.rs:446-461)
    double sing = 0, inval = 0;
    for (int64_t i = tid; i < n; i += WNT) {
      const double pivot = F[i * n + i], d = A.diag[i];
      if (!isfinite(pivot) || !isfinite(d)) inval = 1;
      const double q = pivot / sqrt(d);
      if (d <= 0 || pivot <= 0 || q * q <= A.tol) sing = 1;
    }
    inval = wmax(inval, red);
    sing = wmax(sing, red);
    if (inval != 0) status = FG_INVALID_INFORMATION;
    else if (sing != 0) status = FG_SINGULAR_INFORMATION;
  }
  if (status == 0 && mode != DM_INFO && mode != DM_SCHUR_INFO) {
    double* v = A.work;
    if (mode == DM_SCHUR_DAMPED) {
      // rhs -g / D at factor positions; work held the position scales.
      __syncthreads();
      for (int64_t c = tid; c < n; c += WNT) {
        const int64_t pc = A.perm ? A.perm[c] : c;
        A.step[pc] = -A.rhs[c] / A.scales[c];
      }
      __syncthreads();
      for (int64_t c = tid; c < n; c += WNT) v[c] = A.step[c];
    } else {
      for (int64_t c = tid; c < n; c += WNT) v[c] = A.rhs[c];
    }
    __syncthreads();
    cta_llt_solve<double, DCB>(F, (int)n, (int)n, v, dsm, nullptr);
    double nf = 0;
    for (int64_t c = tid; c < n; c += WNT) {
      double d;
      if (mode == DM_SCHUR_DAMPED) {
        const int64_t pc = A.perm ? A.perm[c] : c;
        d = v[pc] / A.scales[c];
      } else {
        d = v[c];
      }
      if (!isfinite(d)) nf = 1;
      A.step[c] = d;
    }
    nf = wmax(nf, red);
    // predicted reduction
    double p = 0;
    if (mode == DM_NORMAL_DAMPED) {
      // normal.rs:218-226: sum rhs d - d H_cc d / 2 - sum_{r>c} d_c H_rc d_r
      for (int64_t c = tid; c < n; c += WNT) {
        const double d = A.step[c];
        p += A.rhs[c] * d - 0.5 * d * A.N[c * n + c] * d;
        for (int64_t r = c + 1; r < n; ++r) p -= d * A.N[c * n + r] * A.step[r];
      }
    } else if (mode == DM_SCHUR_DAMPED) {
      // -g.d - |J d|^2 / 2 with |J d|^2 = d^T H d (H in factor positions)
      for (int64_t c = tid; c < n; c += WNT) {
        const int64_t pc = A.perm ? A.perm[c] : c;
        const double d = A.step[c];
        p -= A.rhs[c] * d;
        double hd = 0;
        for (int64_t c2 = 0; c2 < n; ++c2) {
          const int64_t p2 = A.perm ? A.perm[c2] : c2;
          const int64_t hi = pc > p2 ? pc : p2, lo = pc > p2 ? p2 : pc;
          hd += A.N[lo * n + hi] * A.step[c2];
        }
        p -= 0.5 * d * hd;
      }
    }
    p = wsum(p, red);
    if (nf != 0) status = FG_LINEAR_SOLVE_FAILED;
    if (tid == 0) {
      A.out[1] = p;
      A.out[2] = nf;
    }
  }
  if (tid == 0) A.out[0] = status;
}

// Selected covariance: Y = L^-1 (D^-1 E_sel) column by column, Sigma = Y^T Y.
__global__ void __launch_bounds__(WNT) k_dense_cov(const double* L, int64_t n, const int64_t* cols, int64_t k,
                                                   const double* scales, const int64_t* perm, double* Y,
                                                   double* out, double* status) {
  extern __shared__ __align__(16) double dsm[];
  __shared__ double red[WNT / 32];
  for (int64_t j = 0; j < k; ++j) {
    double* y = Y + j * n;
    for (int64_t i = threadIdx.x; i < n; i += WNT) y[i] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
      const int64_t c = cols[j];
      y[perm ? perm[c] : c] = 1.0 / (scales ? scales[c] : 1.0);
    }
    __syncthreads();
    // forward substitution only: L y = e
    for (int k0 = 0; k0 < n; k0 += DCB) {
      const int kb = (int)(n - k0 < DCB ? n - k0 : DCB);
      for (int e = threadIdx.x; e < kb * kb; e += WNT) {
        const int r = e % kb, c = e / kb;
        if (r >= c) dsm[r * (DCB + 1) + c] = L[(size_t)(k0 + c) * n + k0 + r];
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        double x = lane < kb ? y[k0 + lane] : 0.0;
        for (int c = 0; c < kb; ++c) {
          const double xc = __shfl_sync(0xffffffffu, x, c) / dsm[c * (DCB + 1) + c];
          if (lane == c) x = xc;
          else if (lane > c && lane < kb) x -= dsm[lane * (DCB + 1) + c] * xc;
        }
        if (lane < kb) y[k0 + lane] = x;
      }
      __syncthreads();
      for (int64_t i = k0 + kb + threadIdx.x; i < n; i += WNT) {
        double s = y[i];
        for (int q = 0; q < kb; ++q) s -= L[(size_t)(k0 + q) * n + i] * y[k0 + q];
        y[i] = s;
      }
      __syncthreads();
    }
  }
  double bad = 0;
  for (int64_t e = threadIdx.x; e < k * k; e += WNT) {
    const int64_t a = e % k, b = e / k;
    double s = 0;
    for (int64_t i = 0; i < n; ++i) s += Y[a * n + i] * Y[b * n + i];
    out[e] = s;
    if (!isfinite(s)) bad = 1;
  }
  bad = wmax(bad, red);
  if (threadIdx.x == 0) *status = bad != 0 ? FG_INVALID_INFORMATION : 0;
}

// DenseQr::factor_solve (qr.rs:65-176) in one CTA. M is height x (n+1).
__global__ void __launch_bounds__(WNT) k_dense_qr(const int64_t* blocks5, int64_t nblocks, const double* values,
                                                  const double* negres, const double* scales, int64_t m, int64_t n,
                                                  int damped, double lambda, double tol, double* M, double* step,
                                                  double* out) {
  extern __shared__ __align__(16) double qsm[];
  __shared__ double red[WNT / 32];
  __shared__ int flag;
  double* norms = qsm;
  int* perm = reinterpret_cast<int*>(qsm + n + 8);
  const int tid = threadIdx.x;
  const int64_t height = m + (damped ? n : 0), width = n + 1;
  for (int64_t e = tid; e < height * width; e += WNT) M[e] = 0;
  __syncthreads();
  for (int64_t b = 0; b < nblocks; ++b) {
    const int64_t* B = blocks5 + 5 * b;
    for (int64_t e = tid; e < B[2] * B[3]; e += WNT) {
      const int64_t r = e % B[2], c = e / B[2];
      const double sc = damped ? scales[B[1] + c] : 1.0;
      M[(B[1] + c) * height + B[0] + r] = values[B[4] + c * B[2] + r] / sc;
    }
    __syncthreads();
  }
  for (int64_t r = tid; r < m; r += WNT) M[n * height + r] = negres[r];
  if (damped)
    for (int64_t c = tid; c < n; c += WNT) M[c * height + m + c] = sqrt(lambda);
  __syncthreads();
  double largest = 0, bad = 0;
  for (int64_t e = tid; e < height * width; e += WNT) {
    const double v = M[e];
    if (!isfinite(v)) bad = 1;
    if (e / height < n) largest = fmax(largest, fabs(v));
  }
  bad = wmax(bad, red);
  largest = wmax(largest, red);
  double status = 0;
  if (bad != 0 || largest == 0) status = FG_LINEAR_SOLVE_FAILED;
  if (status == 0) {
    cta_qr(M, (int)height, (int)width, 0, 0, (int)n, perm, norms, red, &flag);
    double big = 0, nfp = 0;
    for (int64_t c = tid; c < n; c += WNT) {
      const double p = fabs(M[c * height + c]);
      if (!isfinite(p)) nfp = 1;
      big = fmax(big, p);
    }
    big = wmax(big, red);
    nfp = wmax(nfp, red);
    if (nfp != 0) status = FG_LINEAR_SOLVE_FAILED;
    if (status == 0 && tid == 0) {
      for (int64_t c = n - 1; c >= 0; --c) {
        const double pivot = M[c * height + c];
        if (fabs(pivot) <= tol * big) {
          status = FG_LINEAR_SOLVE_FAILED;
          break;
        }
        double v = M[n * height + c];
        for (int64_t j = c + 1; j < n; ++j) v -= M[j * height + c] * step[perm[j]];
        step[perm[c]] = v / pivot;
      }
      red[0] = status;
    }
    __syncthreads();
    status = red[0];
    __syncthreads();
    if (status == 0) {
      double nf = 0;
      for (int64_t c = tid; c < n; c += WNT) {
        if (damped) step[c] /= scales[c];
        if (!isfinite(step[c])) nf = 1;
      }
      nf = wmax(nf, red);
      if (nf != 0) status = FG_LINEAR_SOLVE_FAILED;
    }
  }
  if (tid == 0) out[0] = status;
}

// -g.d - |J d|^2 / 2 from the lower J^T J (LinearizedModel::predicted_reduction).
__global__ void __launch_bounds__(WNT) k_dense_predict(const double* N, int64_t n, const double* g,
                                                       const double* d, double* out) {
  __shared__ double red[WNT / 32];
  double p = 0;
  for (int64_t c = threadIdx.x; c < n; c += WNT) {
    p -= g[c] * d[c];
    double hd = 0;
    for (int64_t c2 = 0; c2 < n; ++c2) {
      const int64_t hi = c > c2 ? c : c2, lo = c > c2 ? c2 : c;
      hd += N[lo * n + hi] * d[c2];
    }
    p -= 0.5 * d[c] * hd;
  }
  p = wsum(p, red);
  if (threadIdx.x == 0) out[1] = p;
}

class DenseImpl final : public Backend {
 public:
  DenseImpl(int kind, int device) : dk(kind), dev(device) {}
  fg_status init() {
    FG_TRY(select_device(dev));
    FG_TRY(device_stream(dev, &st));
    FG_TRY(d_out.resize(8));
    FG_TRY(h_out.resize(8));
    return FG_OK;
  }
  int kind() const override { return 2 + dk; }

  size_t retained = 0;
  std::vector<size_t> widths;
  double qr_tol = 64.0 * std::numeric_limits<double>::epsilon();

  fg_status prepare(size_t dimension) override {
    ready = factorized = false;
    solves = 0;
    if (dk == DK_QR && !(qr_tol >= 0 && qr_tol < 1)) {
      set_error("relative_rank_tolerance must lie in [0, 1)");
      return FG_INVALID_OPTIONS;
    }
    if (dk == DK_SCHUR) {  // dense_schur.rs:211-271
      if (dimension < retained) return invalid("retained dimension exceeds the graph dimension");
      landmarks.clear();
      size_t offset = retained;
      for (size_t w : widths) {
        const size_t end = offset + w;
        if (w == 0 || end < offset || end > dimension) return invalid("invalid landmark widths");
        landmarks.push_back({offset, end});
        offset = end;
      }
      if (offset != dimension) return invalid("landmark widths do not cover the graph dimension");
      owners.assign(dimension - retained, 0);
      for (size_t id = 0; id < landmarks.size(); ++id)
        for (size_t c = landmarks[id].first; c < landmarks[id].second; ++c) owners[c - retained] = id;
      // factor order: landmark coordinates first, then the retained prefix
      std::vector<int64_t> perm(dimension);
      for (size_t c = 0; c < dimension; ++c)
        perm[c] = (int64_t)(c < retained ? dimension - retained + c : c - retained);
      if (dimension) FG_TRY(upload(d_perm, perm.data(), dimension, st));
      else FG_TRY(d_perm.resize(1));
    }
    n = dimension;
    FG_TRY(select_device(dev));
    FG_TRY(h_step.resize(std::max<size_t>(n, 1)));
    FG_TRY(d_step.resize(std::max<size_t>(n, 1)));
    FG_TRY(d_scales.resize(std::max<size_t>(n, 1)));
    FG_TRY(d_work.resize(std::max<size_t>(n, 1)));
    FG_TRY(d_diag.resize(std::max<size_t>(n, 1)));
    FG_TRY(d_N.resize(std::max<size_t>(n * n, 1)));
    FG_TRY(d_F.resize(std::max<size_t>(n * n, 1)));
    return clear();
  }
  fg_status clear() override {
    ready = factorized = false;
    blocks.clear();
    values.clear();
    negres.clear();
    grad.assign(n, 0.0);
    rows = 0;
    model_on_device = false;
    return FG_OK;
  }
  fg_status accumulate(size_t nrows, const double* r, size_t nb, const size_t* cols, const size_t* w,
                       const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) override {
    ready = false;
    if (nrows && !r) return FG_NULL_ARGUMENT;
    if (nb && (!cols || !w || !jac || !rs || !cs)) return FG_NULL_ARGUMENT;
    bool has_landmark = false;
    for (size_t i = 0; i < nb; ++i) {
      const size_t end = cols[i] + w[i];
      if (end < cols[i] || end > n) {
        set_error("Jacobian block outside the prepared dimension");
        return FG_DIMENSION_MISMATCH;
      }
      if (w[i] && nrows && !jac[i]) return FG_NULL_ARGUMENT;
      if (dk != DK_SCHUR || w[i] == 0) continue;
      // dense_schur.rs:278-306
      if (cols[i] >= retained) {
        const size_t id = owners[cols[i] - retained];
        if (landmarks[id].first != cols[i] || landmarks[id].second != end || has_landmark)
          return unsupported("an emission may touch at most one complete landmark");
        has_landmark = true;
      } else if (end > retained) {
        return unsupported("a retained block crosses into the landmarks");
      }
      for (size_t o = 0; o < i; ++o)
        if (cols[i] < cols[o] + w[o] && cols[o] < end) {
          set_error("overlapping blocks in one emission");
          return FG_DIMENSION_MISMATCH;
        }
    }
    if (dk == DK_NORMAL && factorized) factorized = false;
    const size_t row = rows;
    for (size_t i = 0; i < nrows; ++i) negres.push_back(-r[i]);
    for (size_t b = 0; b < nb; ++b) {
      blocks.push_back({row, cols[b], nrows, w[b], values.size()});
      for (size_t j = 0; j < w[b]; ++j) {
        double g = 0;
        for (size_t i = 0; i < nrows; ++i) {
          const double v = jac[b][(ptrdiff_t)i * rs[b] + (ptrdiff_t)j * cs[b]];
          values.push_back(v);
          g += v * r[i];
        }
        grad[cols[b] + j] += g;
      }
    }
    rows = row + nrows;
    model_on_device = false;
    return FG_OK;
  }
  fg_status gradient_norm(double* out) override {
    double m = 0;
    for (double g : grad) {
      if (!std::isfinite(g)) {
        set_error("nonfinite gradient");
        return FG_INVALID_EVALUATION;
      }
      m = std::max(m, std::fabs(g));
    }
    *out = m;
    return FG_OK;
  }

  fg_status prepare_damping(double floor) override {
    ready = false;
    if (dk == DK_NORMAL && factorized) {
      set_error("prepare_damping after a destructive solve needs a fresh model");
      return FG_INVALID_OPTIONS;
    }
    if (!std::isfinite(floor) || floor <= 0) return invalid("min_column_norm must be finite and positive");
    double gn;
    FG_TRY(gradient_norm(&gn));
    FG_TRY(sync_model());
    if (n) {
      FG_LAUNCH(k_dense_scales, 1, WNT, 0, st, d_N.get(), (int64_t)n, floor,
                dk == DK_SCHUR ? d_perm.get() : nullptr, d_scales.get(), d_out.get());
      FG_TRY(readback(2));
      if (h_out.get()[0] != 0 || (dk == DK_NORMAL && h_out.get()[1] != 0)) {
        set_error("nonfinite or negative normal-matrix entry");
        return FG_INVALID_EVALUATION;
      }
    }
    ready = true;
    return FG_OK;
  }

  fg_status solve_damped(double lambda, double* predicted, bool copy_to_host) override {
    if (!ready || !std::isfinite(lambda) || lambda < 0) {
      set_error("solve_damped requires prepare_damping and a finite nonnegative lambda");
      return FG_INVALID_OPTIONS;
    }
    ++solves;
    if (n == 0) {
      *predicted = 0;
      return FG_OK;
    }
    if (dk == DK_QR) {
      FG_TRY(qr_solve(true, lambda));
      FG_LAUNCH(k_dense_predict, 1, WNT, 0, st, d_N.get(), (int64_t)n, d_grad.get(), d_step.get(), d_out.get());
      FG_TRY(readback(2));
      if (!std::isfinite(h_out.get()[1])) return failed("nonfinite prediction");
      *predicted = h_out.get()[1];
      return finish(copy_to_host);
    }
    FG_TRY(run_solve(dk == DK_NORMAL ? DM_NORMAL_DAMPED : DM_SCHUR_DAMPED, lambda, 0.0));
    const double status = h_out.get()[0];
    if (status != 0) {
      set_error("dense damped solve failed");
      return (fg_status)(int)status;
    }
    if (!std::isfinite(h_out.get()[1])) return failed("nonfinite prediction");
    *predicted = h_out.get()[1];
    return finish(copy_to_host);
  }

  fg_status solve_undamped(bool copy_to_host) override {
    if (dk == DK_SCHUR) return Backend::solve_undamped(copy_to_host);
    ready = false;
    if (n == 0) return FG_OK;
    if (dk == DK_QR) {
      FG_TRY(qr_solve(false, 0.0));
      return finish(copy_to_host);
    }
    FG_TRY(sync_model());
    FG_TRY(run_solve(DM_NORMAL_SOLVE, 0.0, 0.0));
    factorized = true;  // normal.rs:137-152 factors in place
    const double status = h_out.get()[0];
    if (status != 0) {
      set_error("dense normal solve failed");
      return (fg_status)(int)status;
    }
    return finish(copy_to_host);
  }

  // Selected covariance of the current model (covariance.rs:263-270).
  fg_status covariance(const size_t* cols, size_t k, double tol, double* out) {
    if (!(tol >= 0 && tol < 1)) {
      set_error("relative pivot tolerance must lie in [0, 1)");
      return FG_INVALID_RANK_TOLERANCE;
    }
    std::set<size_t> seen;
    for (size_t j = 0; j < k; ++j) {
      if (!seen.insert(cols[j]).second) {
        set_error("duplicate covariance column");
        return FG_DUPLICATE_COVARIANCE_BLOCK;
      }
      if (cols[j] >= n || (dk == DK_SCHUR && cols[j] >= retained)) {
        set_error("covariance column outside the supported coordinates");
        return FG_UNSUPPORTED_STRUCTURE;
      }
    }
    int mode = DM_INFO;
    if (dk == DK_SCHUR) {
      // prepare_damping(1e-6) + reduce(0, tol), errors mapped as dense_schur.rs:359-377
      fg_status s = prepare_damping(1e-6);
      if (s == FG_LINEAR_SOLVE_FAILED) return FG_SINGULAR_INFORMATION;
      if (s == FG_INVALID_EVALUATION) return FG_INVALID_INFORMATION;
      FG_TRY(s);
      mode = DM_SCHUR_INFO;
    } else {
      FG_TRY(sync_model());
    }
    if (n) {
      FG_TRY(run_solve(mode, 0.0, tol));
      double status = h_out.get()[0];
      if (status == FG_LINEAR_SOLVE_FAILED) status = FG_SINGULAR_INFORMATION;
      if (status == FG_INVALID_EVALUATION) status = FG_INVALID_INFORMATION;
      if (status != 0) {
        set_error("singular or invalid information");
        return (fg_status)(int)status;
      }
    }
    if (k == 0) return FG_OK;
    std::vector<int64_t> c64(cols, cols + k);
    DBuf<int64_t> dc;
    DBuf<double> dy, dout;
    FG_TRY(upload(dc, c64.data(), k, st));
    FG_TRY(dy.resize(n * k));
    FG_TRY(dout.resize(k * k));
    const size_t sm = (size_t)DCB * (DCB + 1) * sizeof(double);
    FG_LAUNCH(k_dense_cov, 1, WNT, sm, st, d_F.get(), (int64_t)n, dc.get(), (int64_t)k,
              dk == DK_SCHUR ? d_scales.get() : nullptr, dk == DK_SCHUR ? d_perm.get() : nullptr, dy.get(),
              dout.get(), d_out.get() + 3);
    FG_CUDA(cudaMemcpyAsync(out, dout.get(), k * k * sizeof(double), cudaMemcpyDeviceToHost, st));
    FG_TRY(readback(4));
    if (h_out.get()[3] != 0) {
      set_error("nonfinite covariance");
      return FG_INVALID_INFORMATION;
    }
    if (dk == DK_NORMAL) factorized = true;
    return FG_OK;
  }

  fg_status step_norm_inf(double* out) override {
    double m = 0;
    for (size_t i = 0; i < n; ++i) {
      if (!std::isfinite(h_step.get()[i])) return FG_INVALID_EVALUATION;
      m = std::max(m, std::fabs(h_step.get()[i]));
    }
    *out = m;
    return FG_OK;
  }
  const double* step_host() const override { return h_step.get(); }
  const double* step_device() const override { return d_step.get(); }
  size_t dimension() const override { return n; }
  void work(size_t* s, size_t* i) const override {
    *s = solves;
    *i = 0;
  }
  fg_status bind_bal(const BalObservations&) override {
    set_error("the dense backends take host emissions only");
    return FG_UNSUPPORTED_STRUCTURE;
  }
  void* values_device() override { return nullptr; }
  double* negres_device() override { return nullptr; }
  bool is_f32() const override { return false; }
  void mark_device_model(size_t) override {}
  int device() const override { return dev; }
  cudaStream_t stream() const override { return st; }

 private:
  int dk, dev;
  cudaStream_t st = nullptr;
  size_t n = 0, rows = 0, solves = 0;
  bool ready = false, factorized = false, model_on_device = false;
  std::vector<HostBlock> blocks;
  std::vector<double> values, negres, grad;
  std::vector<std::pair<size_t, size_t>> landmarks;
  std::vector<size_t> owners;
  DBuf<double> d_vals, d_neg, d_grad, d_N, d_F, d_scales, d_step, d_work, d_diag, d_out, d_M;
  DBuf<int64_t> d_blocks, d_pairs, d_perm;
  HBuf<double> h_step, h_out;

  fg_status invalid(const char* what) {
    set_error(what);
    return FG_INVALID_OPTIONS;
  }
  fg_status unsupported(const char* what) {
    set_error(what);
    return FG_UNSUPPORTED_STRUCTURE;
  }
  fg_status failed(const char* what) {
    set_error(what);
    return FG_LINEAR_SOLVE_FAILED;
  }
  fg_status readback(int count) {
    FG_CUDA(cudaMemcpyAsync(h_out.get(), d_out.get(), count * sizeof(double), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    return FG_OK;
  }
  // The host mirror is always refreshed: step_norm_inf reads it.
  fg_status finish(bool) {
    FG_CUDA(cudaMemcpyAsync(h_step.get(), d_step.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    return FG_OK;
  }

  // Upload the packed model and assemble the lower J^T J.
  fg_status sync_model() {
    if (model_on_device) return FG_OK;
    std::vector<int64_t> b5(std::max<size_t>(5 * blocks.size(), 5));
    for (size_t i = 0; i < blocks.size(); ++i) {
      b5[5 * i] = (int64_t)blocks[i].row;
      b5[5 * i + 1] = (int64_t)blocks[i].col;
      b5[5 * i + 2] = (int64_t)blocks[i].rows;
      b5[5 * i + 3] = (int64_t)blocks[i].cols;
      b5[5 * i + 4] = (int64_t)blocks[i].start;
    }
    // block pairs of each emission (same row, same row count)
    std::vector<int64_t> pairs;
    for (size_t a = 0; a < blocks.size(); ++a) {
      if (blocks[a].rows == 0 || blocks[a].cols == 0) continue;
      for (size_t b = a + 1; b-- > 0;) {
        if (blocks[b].row != blocks[a].row || blocks[b].rows != blocks[a].rows) break;
        if (blocks[b].cols == 0) continue;
        pairs.push_back((int64_t)a);
        pairs.push_back((int64_t)b);
      }
    }
    FG_TRY(upload(d_blocks, b5.data(), b5.size(), st));
    std::vector<int64_t> pv = pairs;
    if (pv.empty()) pv.assign(2, 0);
    FG_TRY(upload(d_pairs, pv.data(), pv.size(), st));
    std::vector<double> vals = values;
    if (vals.empty()) vals.push_back(0);
    FG_TRY(upload(d_vals, vals.data(), vals.size(), st));
    std::vector<double> neg = negres;
    if (neg.empty()) neg.push_back(0);
    FG_TRY(upload(d_neg, neg.data(), neg.size(), st));
    std::vector<double> gg = grad;
    if (gg.empty()) gg.push_back(0);
    FG_TRY(upload(d_grad, gg.data(), gg.size(), st));
    if (n) {
      FG_CUDA(cudaMemsetAsync(d_N.get(), 0, n * n * sizeof(double), st));
      if (!pairs.empty())
        FG_LAUNCH(k_dense_pairs, (unsigned)(pairs.size() / 2), 256, 0, st, d_blocks.get(), d_pairs.get(),
                  d_vals.get(), d_N.get(), (int64_t)n, dk == DK_SCHUR ? d_perm.get() : nullptr);
      // NORMAL keeps -J^T r as its rhs
      if (dk == DK_NORMAL) {
        std::vector<double> rhs(n);
        for (size_t i = 0; i < n; ++i) rhs[i] = -grad[i];
        FG_CUDA(cudaMemcpyAsync(d_work.get(), rhs.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
        FG_TRY(d_M.resize(n));
        FG_CUDA(cudaMemcpyAsync(d_M.get(), d_work.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, st));
      }
    }
    FG_CUDA(cudaStreamSynchronize(st));
    model_on_device = true;
    return FG_OK;
  }

  fg_status run_solve(int mode, double lambda, double tol) {
    DenseArgs A{};
    A.N = d_N.get();
    A.F = d_F.get();
    A.n = (int64_t)n;
    A.rhs = dk == DK_NORMAL ? d_M.get() : d_grad.get();
    A.scales = d_scales.get();
    A.perm = dk == DK_SCHUR ? d_perm.get() : nullptr;
    A.lambda = lambda;
    A.step = d_step.get();
    A.work = d_work.get();
    A.diag = d_diag.get();
    A.tol = tol;
    A.out = d_out.get();
    if (dk == DK_SCHUR) {
      // position scales: work[perm[c]] = scales[c]
      std::vector<double> sc(n), pos(n);
      FG_CUDA(cudaMemcpyAsync(sc.data(), d_scales.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st));
      FG_CUDA(cudaStreamSynchronize(st));
      for (size_t c = 0; c < n; ++c) pos[c < retained ? n - retained + c : c - retained] = sc[c];
      FG_CUDA(cudaMemcpyAsync(d_work.get(), pos.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
      if (mode == DM_INFO) mode = DM_SCHUR_INFO;
    }
    const size_t sm = ((size_t)DCB * (DCB + 1) + 2 * (size_t)WCT * (DCB + 1)) * sizeof(double);
    FG_CUDA(cudaFuncSetAttribute(k_dense_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    FG_LAUNCH(k_dense_solve, 1, WNT, sm, st, A, mode);
    return readback(3);
  }

  fg_status qr_solve(bool damped, double lambda) {
    FG_TRY(sync_model());
    const size_t height = rows + (damped ? n : 0);
    if (height < n) return failed("fewer rows than unknowns");
    FG_TRY(d_M.resize(std::max<size_t>(height * (n + 1), 1)));
    const size_t sm = (n + 8) * sizeof(double) + n * sizeof(int) + 64;
    FG_CUDA(cudaFuncSetAttribute(k_dense_qr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(sm, 1024)));
    FG_LAUNCH(k_dense_qr, 1, WNT, sm, st, d_blocks.get(), (int64_t)blocks.size(), d_vals.get(), d_neg.get(),
              d_scales.get(), (int64_t)rows, (int64_t)n, damped ? 1 : 0, lambda, qr_tol, d_M.get(), d_step.get(),
              d_out.get());
    FG_TRY(readback(1));
    if (h_out.get()[0] != 0) return failed("rank-deficient or nonfinite QR solve");
    return FG_OK;
  }

 public:
  void set_qr_tolerance(double t) { qr_tol = t; }
};

}  // namespace fg

using namespace fg;

namespace {
fg_status make_dense(int kind, int device, DenseImpl** out) {
  auto* b = new DenseImpl(kind, device);
  fg_status s = b->init();
  if (s != FG_OK) {
    delete b;
    return s;
  }
  *out = b;
  return FG_OK;
}
}  // namespace

FG_API fg_status fg_dense_normal_create(int device, fg_backend** out) {
  if (!out) return FG_NULL_ARGUMENT;
  DenseImpl* b = nullptr;
  FG_TRY(make_dense(DK_NORMAL, device, &b));
  *out = new fg_backend{b};
  return FG_OK;
}
FG_API fg_status fg_dense_schur_create(size_t retained_dimension, const size_t* eliminated_widths, size_t count,
                                       int device, fg_backend** out) {
  if (!out || (count && !eliminated_widths)) return FG_NULL_ARGUMENT;
  DenseImpl* b = nullptr;
  FG_TRY(make_dense(DK_SCHUR, device, &b));
  b->retained = retained_dimension;
  b->widths.assign(eliminated_widths, eliminated_widths + count);
  *out = new fg_backend{b};
  return FG_OK;
}
FG_API fg_status fg_dense_qr_create(double relative_rank_tolerance, int device, fg_backend** out) {
  if (!out) return FG_NULL_ARGUMENT;
  DenseImpl* b = nullptr;
  FG_TRY(make_dense(DK_QR, device, &b));
  b->set_qr_tolerance(relative_rank_tolerance);
  *out = new fg_backend{b};
  return FG_OK;
}
FG_API fg_status fg_dense_qr_set_tolerance(fg_backend* b, double tol) {
  if (!b || !b->impl) return FG_NULL_ARGUMENT;
  if (b->impl->kind() != 2 + DK_QR) {
    set_error("not a DenseQr backend");
    return FG_INVALID_OPTIONS;
  }
  static_cast<DenseImpl*>(b->impl)->set_qr_tolerance(tol);
  return FG_OK;
}
// LinearizedModel::covariance (src/linear_model.rs:122-167), which Schur and
// Lsmr delegate to: a DenseNormalCholesky over the cached Jacobian, replayed
// one row group at a time (blocks sharing row and rows; empty groups skipped)
// with -r as the residual, then the selected covariance of that normal matrix.
static fg_status model_covariance(Backend* src, const size_t* columns, size_t k, double tol, double* out) {
  HostModel m;
  FG_TRY(src->model_host(&m));
  DenseImpl* normal = nullptr;
  FG_TRY(make_dense(DK_NORMAL, src->device(), &normal));
  std::unique_ptr<DenseImpl> hold(normal);
  FG_TRY(normal->prepare(m.cols));
  FG_TRY(normal->clear());
  std::vector<size_t> cols, widths;
  std::vector<const double*> jac;
  std::vector<ptrdiff_t> rs, cs;
  size_t start = 0;
  while (start < m.blocks.size()) {
    const HostBlock& first = m.blocks[start];
    if (first.rows == 0) {
      ++start;
      continue;
    }
    size_t end = start + 1;
    while (end < m.blocks.size() && m.blocks[end].row == first.row && m.blocks[end].rows == first.rows) ++end;
    cols.clear(); widths.clear(); jac.clear(); rs.clear(); cs.clear();
    for (size_t i = start; i < end; ++i) {
      const HostBlock& b = m.blocks[i];
      cols.push_back(b.col);
      widths.push_back(b.cols);
      jac.push_back(m.values.data() + b.start);
      rs.push_back(1);
      cs.push_back((ptrdiff_t)b.rows);
    }
    FG_TRY(normal->accumulate(first.rows, m.negres.data() + first.row, end - start, cols.data(), widths.data(),
                              jac.data(), rs.data(), cs.data()));
    start = end;
  }
  return normal->covariance(columns, k, tol, out);
}

FG_API fg_status fg_backend_covariance(fg_backend* b, const size_t* columns, size_t k, double tol, double* out) {
  if (!b || !b->impl || (k && (!columns || !out))) return FG_NULL_ARGUMENT;
  try {
    if (b->impl->kind() < 2) return model_covariance(b->impl, columns, k, tol, out);
    return static_cast<DenseImpl*>(b->impl)->covariance(columns, k, tol, out);
  } catch (...) {
    set_error("unexpected host exception");
    return FG_CUDA_ERROR;
  }
}
