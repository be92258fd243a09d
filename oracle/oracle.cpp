// ORACLE — test infrastructure only.
//
// A plain, sequential, f64 CPU restatement of fagra's hot path, used as the
// checker for the CUDA backend. Only tests/, __graft_entry__.smoke() and the
// CPU-baseline legs of bench.py load this library; the product never does.
//
// It restates, function by function (citations are paths inside the fagra
// repository):
//   examples/bal/model.rs:116-237          Projection, Frame cost/linearize
//   src/optimization.rs:296-389,541-612     Layout and emission order
//   src/linear_model.rs:99-282              LinearizedModel
//   src/linear_model/block_factors.rs:47-205 BlockFactors
//   src/schur.rs:116-682                    Schur backend (+ cross_apply, Reduced)
//   faer 0.24.4 matrix_free::conjugate_gradient (the third-party CG called at
//     src/schur.rs:264-297), restated for one right-hand side: standard PCG
//     with the explicit zero start, relative threshold on ||r||_2 and the
//     per-iteration callback placed before the convergence test.
//   src/optimization/levenberg_marquardt.rs:330-472  LM loop
//   src/optimization/gauss_newton.rs:101-176         GN loop
//   src/lsmr.rs:126-595 + faer's LSMR               LSMR backend (see its section)
//   dense.hpp: DenseNormalCholesky, DenseSchur, DenseQr, square-root
//     elimination and selected covariance; posegraph.hpp: SE(3) geometry and
//     the pose-graph window workload.
//
// Parity pins: the reference's own known-answer tests (ported in tests/).
// Iteration counts of faer's CG are not pinned by any reference test except
// the one-iteration limit; they are reported, not matched.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstddef>
#include <limits>
#include <vector>
#include <algorithm>

#define OR_API extern "C" __attribute__((visibility("default")))

namespace {

// Status codes shared with include/fagra_b200.h (same numbering).
enum Status {
  OK = 0,
  DUPLICATE_COVARIANCE_BLOCK = 1,
  SINGULAR_INFORMATION = 2,
  INVALID_INFORMATION = 3,
  INVALID_RANK_TOLERANCE = 4,
  INVALID_OPTIONS = 6,
  LINEAR_SOLVE_FAILED = 8,
  NO_CONVERGENCE = 9,
  NO_PROGRESS = 10,
  INVALID_EVALUATION = 20,
  DIMENSION_MISMATCH = 21,
  INVALID_EMISSION = 22,
  UNSUPPORTED_STRUCTURE = 23,
};
enum Termination { T_NONE = 0, T_CONVERGED = 1, T_ITERATION_LIMIT = 2, T_NOT_PD = 3, T_NONFINITE = 4 };
const size_t NONE = std::numeric_limits<size_t>::max();

bool is_fin(double x) { return std::isfinite(x); }

// optimization.rs:653-662
int norm_inf(const double* v, size_t n, double* out) {
  double m = 0;
  for (size_t i = 0; i < n; ++i) {
    if (!is_fin(v[i])) return INVALID_EVALUATION;
    m = std::max(m, std::fabs(v[i]));
  }
  *out = m;
  return OK;
}
// linear_model.rs:325-337
double norm_l2(const double* v, size_t n) {
  double s = 0;
  for (size_t i = 0; i < n; ++i) s = std::hypot(s, v[i]);
  return s;
}
double relative(double norm, double ref) { return ref == 0 ? norm : norm / ref; }

// ---------------------------------------------------------------- BAL model
// examples/bal/model.rs:116-185
struct Projection {
  double cam[9], R[9], right[9];  // row-major 3x3
};
void skew(const double* v, double* K) {
  K[0] = 0; K[1] = -v[2]; K[2] = v[1];
  K[3] = v[2]; K[4] = 0; K[5] = -v[0];
  K[6] = -v[1]; K[7] = v[0]; K[8] = 0;
}
void mat3mul(const double* A, const double* B, double* C) {
  double T[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += A[3 * i + k] * B[3 * k + j];
      T[3 * i + j] = s;
    }
  std::memcpy(C, T, sizeof T);
}
// nalgebra UnitQuaternion::from_scaled_axis(w) = exp(w/2 as pure quaternion),
// identity when |w/2|^2 <= eps^2; to_rotation_matrix uses the ww+ii-jj-kk form.
void rotation_from_scaled_axis(const double* w, double* R) {
  double v[3] = {w[0] / 2, w[1] / 2, w[2] / 2};
  double nn = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  double eps = std::numeric_limits<double>::epsilon();
  double qw, qi, qj, qk;
  if (nn <= eps * eps) {
    qw = 1; qi = qj = qk = 0;
  } else {
    double n = std::sqrt(nn), s = std::sin(n) / n;
    qw = std::cos(n); qi = v[0] * s; qj = v[1] * s; qk = v[2] * s;
  }
  double ww = qw * qw, ii = qi * qi, jj = qj * qj, kk = qk * qk;
  double ij = qi * qj * 2, wk = qw * qk * 2, wj = qw * qj * 2, ik = qi * qk * 2, jk = qj * qk * 2,
         wi = qw * qi * 2;
  R[0] = ww + ii - jj - kk; R[1] = ij - wk; R[2] = wj + ik;
  R[3] = wk + ij; R[4] = ww - ii + jj - kk; R[5] = jk - wi;
  R[6] = ik - wj; R[7] = wi + jk; R[8] = ww - ii - jj + kk;
}
void projection_new(const double* cam, Projection* p) {
  std::memcpy(p->cam, cam, 9 * sizeof(double));
  const double* w = cam;
  double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double a, b;
  if (t2 < 1e-8) {
    a = 0.5 - t2 / 24. + t2 * t2 / 720.;
    b = 1. / 6. - t2 / 120. + t2 * t2 / 5040.;
  } else {
    double t = std::sqrt(t2);
    a = (1. - std::cos(t)) / t2;
    b = (t - std::sin(t)) / (t2 * t);
  }
  double K[9], K2[9];
  skew(w, K);
  mat3mul(K, K, K2);
  for (int i = 0; i < 9; ++i) p->right[i] = (i % 4 == 0 ? 1. : 0.) - a * K[i] + b * K2[i];
  rotation_from_scaled_axis(w, p->R);
}
// model.rs:147-156
int projection_value(const Projection& pr, const double* X, double* pix) {
  double p[3];
  for (int i = 0; i < 3; ++i)
    p[i] = pr.R[3 * i] * X[0] + pr.R[3 * i + 1] * X[1] + pr.R[3 * i + 2] * X[2] + pr.cam[3 + i];
  double q0 = -p[0] / p[2], q1 = -p[1] / p[2];
  double r2 = q0 * q0 + q1 * q1;
  double s = pr.cam[6] * (1. + pr.cam[7] * r2 + pr.cam[8] * r2 * r2);
  pix[0] = s * q0;
  pix[1] = s * q1;
  if (p[2] == 0. || !is_fin(pix[0]) || !is_fin(pix[1])) return INVALID_EVALUATION;
  return OK;
}
// model.rs:157-185. jc: 2x9 column-major, jp: 2x3 column-major.
void projection_jacobians(const Projection& pr, const double* X, double* jc, double* jp) {
  double p[3];
  for (int i = 0; i < 3; ++i)
    p[i] = pr.R[3 * i] * X[0] + pr.R[3 * i + 1] * X[1] + pr.R[3 * i + 2] * X[2] + pr.cam[3 + i];
  double q[2] = {-p[0] / p[2], -p[1] / p[2]};
  double r2 = q[0] * q[0] + q[1] * q[1];
  double f = pr.cam[6], k1 = pr.cam[7], k2 = pr.cam[8];
  double radial = 1. + k1 * r2 + k2 * r2 * r2;
  double c = 2. * k1 + 4. * k2 * r2;
  double dq[4];  // row-major 2x2
  dq[0] = f * (radial + c * q[0] * q[0]);
  dq[1] = f * (c * q[0] * q[1]);
  dq[2] = f * (c * q[1] * q[0]);
  dq[3] = f * (radial + c * q[1] * q[1]);
  double M[6] = {-1. / p[2], 0., p[0] / (p[2] * p[2]), 0., -1. / p[2], p[1] / (p[2] * p[2])};
  double dp[6];  // row-major 2x3
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) dp[3 * i + j] = dq[2 * i] * M[j] + dq[2 * i + 1] * M[3 + j];
  double negR[9], K[9], A[9];
  for (int i = 0; i < 9; ++i) negR[i] = -pr.R[i];
  skew(X, K);
  // ((dp * -R) * skew(X)) * right, evaluated left to right as in the source.
  double t1[6], t2[6], t3[6];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += dp[3 * i + k] * negR[3 * k + j];
      t1[3 * i + j] = s;
    }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += t1[3 * i + k] * K[3 * k + j];
      t2[3 * i + j] = s;
    }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += t2[3 * i + k] * pr.right[3 * k + j];
      t3[3 * i + j] = s;
    }
  (void)A;
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 2; ++i) {
      jc[2 * j + i] = t3[3 * i + j];
      jc[2 * (3 + j) + i] = dp[3 * i + j];
    }
  for (int i = 0; i < 2; ++i) {
    jc[2 * 6 + i] = radial * q[i];
    jc[2 * 7 + i] = f * r2 * q[i];
    jc[2 * 8 + i] = f * r2 * r2 * q[i];
  }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += dp[3 * i + k] * pr.R[3 * k + j];
      jp[2 * j + i] = s;
    }
}

// ------------------------------------------------------ LinearizedModel
struct Block {
  size_t row, col, rows, cols, start;
};
struct Model {
  size_t rows = 0, cols = 0;
  std::vector<Block> blocks;
  std::vector<double> values, negative_residual, gradient, scales;

  void prepare(size_t dim) {  // linear_model.rs:169-172
    cols = dim;
    gradient.resize(dim, 0.);
  }
  void clear() {  // :173-179
    rows = 0;
    blocks.clear();
    values.clear();
    negative_residual.clear();
    std::fill(gradient.begin(), gradient.end(), 0.);
  }
  // :180-210; jac[k] is column-major rows x widths[k] with the given strides.
  int accumulate(size_t nrows, const double* r, size_t nb, const size_t* bcols, const size_t* widths,
                 const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) {
    size_t row = rows;
    rows = row + nrows;
    for (size_t i = 0; i < nrows; ++i) negative_residual.push_back(-r[i]);
    for (size_t b = 0; b < nb; ++b) {
      blocks.push_back({row, bcols[b], nrows, widths[b], values.size()});
      for (size_t j = 0; j < widths[b]; ++j) {
        double g = 0;
        for (size_t i = 0; i < nrows; ++i) {
          double v = jac[b][(ptrdiff_t)i * rs[b] + (ptrdiff_t)j * cs[b]];
          values.push_back(v);
          g += v * r[i];
        }
        gradient[bcols[b] + j] += g;
      }
    }
    return OK;
  }
  int prepare_scales(double floor) {  // :211-230
    if (!is_fin(floor) || floor <= 0) return INVALID_OPTIONS;
    scales.assign(cols, 0.);
    for (auto& b : blocks)
      for (size_t c = 0; c < b.cols; ++c) {
        double& n = scales[b.col + c];
        for (size_t r = 0; r < b.rows; ++r) n = std::hypot(n, values[b.start + c * b.rows + r]);
      }
    double m;
    if (norm_inf(scales.data(), cols, &m)) return INVALID_EVALUATION;
    for (auto& s : scales) s = std::max(s, floor);
    return OK;
  }
  void apply(const double* x, double* out) const {  // :39-55
    std::fill(out, out + rows, 0.);
    for (auto& b : blocks)
      for (size_t j = 0; j < b.cols; ++j) {
        double xv = x[b.col + j];
        for (size_t i = 0; i < b.rows; ++i) out[b.row + i] += values[b.start + j * b.rows + i] * xv;
      }
  }
  void transpose_apply(const double* y, double* out) const {  // :64-87
    std::fill(out, out + cols, 0.);
    for (auto& b : blocks)
      for (size_t j = 0; j < b.cols; ++j) {
        double s = 0;
        for (size_t i = 0; i < b.rows; ++i) s += values[b.start + j * b.rows + i] * y[b.row + i];
        out[b.col + j] += s;
      }
  }
  double predicted_reduction(const double* step, double* product) const {  // :233-250
    apply(step, product);
    double p = 0;
    for (size_t j = 0; j < cols; ++j) p -= gradient[j] * step[j];
    for (size_t i = 0; i < rows; ++i) p -= (0.5 * product[i]) * product[i];
    return p;
  }
};
struct StepWork {  // linear_model.rs:284-318
  std::vector<double> step, product, normal_residual, reference;
  void prepare_verification(size_t rows, size_t cols) {
    product.resize(rows, 0.);
    normal_residual.resize(cols, 0.);
    reference.resize(cols, 0.);
  }
};
struct Verification {
  double predicted;
  bool finite_step;
  double residual_norm, reference_norm;
};
Verification verify_step(const Model& m, StepWork& w, double lambda) {  // :254-282
  Verification v;
  double tmp;
  v.finite_step = norm_inf(w.step.data(), m.cols, &tmp) == OK;
  v.predicted = m.predicted_reduction(w.step.data(), w.product.data());
  for (size_t i = 0; i < m.rows; ++i) w.product[i] -= m.negative_residual[i];
  m.transpose_apply(w.product.data(), w.normal_residual.data());
  v.residual_norm = 0;
  v.reference_norm = 0;
  for (size_t j = 0; j < m.cols; ++j) {
    double s = m.scales[j];
    w.normal_residual[j] += (lambda * (s * w.step[j])) * s;
    v.residual_norm = std::hypot(v.residual_norm, w.normal_residual[j]);
    v.reference_norm = std::hypot(v.reference_norm, m.gradient[j]);
  }
  w.reference = m.gradient;
  return v;
}

// ------------------------------------------------------- BlockFactors
// block_factors.rs:9-205; Cholesky restated as the textbook column LL^T.
struct VarBlock {
  size_t col, width, start;
  bool fallback;
};
struct BlockFactors {
  std::vector<VarBlock> blocks;
  std::vector<size_t> owners;
  std::vector<double> gram, factors;

  int prepare(const Model& m) {  // :47-111
    blocks.clear();
    gram.clear();
    owners.assign(m.cols, NONE);
    for (auto& b : m.blocks) {
      if (b.cols == 0) continue;
      size_t end = b.col + b.cols;
      if (end > m.cols) return DIMENSION_MISMATCH;
      size_t owner = owners[b.col], id;
      if (owner == NONE) {
        for (size_t c = b.col; c < end; ++c)
          if (owners[c] != NONE) return DIMENSION_MISMATCH;
        id = blocks.size();
        size_t start = gram.size();
        gram.resize(start + b.cols * b.cols, 0.);
        blocks.push_back({b.col, b.cols, start, false});
        for (size_t c = b.col; c < end; ++c) owners[c] = id;
      } else {
        if (blocks[owner].col != b.col || blocks[owner].width != b.cols) return DIMENSION_MISMATCH;
        id = owner;
      }
      size_t start = blocks[id].start;
      for (size_t c = 0; c < b.cols; ++c)
        for (size_t r = c; r < b.cols; ++r) {
          double s = 0;
          for (size_t k = 0; k < b.rows; ++k)
            s += (m.values[b.start + c * b.rows + k] / m.scales[b.col + c]) *
                 (m.values[b.start + r * b.rows + k] / m.scales[b.col + r]);
          gram[start + c * b.cols + r] += s;
        }
    }
    factors.resize(gram.size());
    return OK;
  }
  // In-place lower Cholesky of a column-major n x n matrix (lower triangle read).
  static bool cholesky(double* a, size_t n) {
    for (size_t j = 0; j < n; ++j) {
      double d = a[j * n + j];
      for (size_t k = 0; k < j; ++k) d -= a[k * n + j] * a[k * n + j];
      if (!(d > 0)) return false;
      d = std::sqrt(d);
      a[j * n + j] = d;
      for (size_t i = j + 1; i < n; ++i) {
        double s = a[j * n + i];
        for (size_t k = 0; k < j; ++k) s -= a[k * n + i] * a[k * n + j];
        a[j * n + i] = s / d;
      }
    }
    return true;
  }
  size_t factor(double lambda) {  // :113-138
    factors = gram;
    size_t fallbacks = 0;
    for (auto& b : blocks) {
      double* v = &factors[b.start];
      size_t w = b.width;
      for (size_t j = 0; j < w; ++j) v[j * w + j] += lambda;
      double tmp;
      b.fallback = norm_inf(v, w * w, &tmp) != OK || !cholesky(v, w);
      if (!b.fallback)
        for (size_t j = 0; j < w; ++j)
          if (!is_fin(v[j * w + j]) || v[j * w + j] <= 0) b.fallback = true;
      fallbacks += b.fallback;
    }
    return fallbacks;
  }
  static void solve_lower(const double* l, size_t n, double* x) {
    for (size_t i = 0; i < n; ++i) {
      double s = x[i];
      for (size_t k = 0; k < i; ++k) s -= l[k * n + i] * x[k];
      x[i] = s / l[i * n + i];
    }
  }
  static void solve_upper_t(const double* l, size_t n, double* x) {  // L^T x = b
    for (size_t ii = n; ii-- > 0;) {
      double s = x[ii];
      for (size_t k = ii + 1; k < n; ++k) s -= l[ii * n + k] * x[k];
      x[ii] = s / l[ii * n + ii];
    }
  }
  // :142-160 (transpose=false applies L^-T, true applies L^-1)
  void apply_factor_inverse(double* rhs, bool transpose) const {
    for (auto& b : blocks) {
      if (b.fallback) continue;
      if (transpose)
        solve_lower(&factors[b.start], b.width, rhs + b.col);
      else
        solve_upper_t(&factors[b.start], b.width, rhs + b.col);
    }
  }
  // :178-204, rhs covers coordinates [offset, offset+n).
  void solve_normal(double* rhs, size_t n, size_t offset, double lambda) const {
    for (auto& b : blocks) {
      if (b.col < offset || b.col >= offset + n) continue;
      double* part = rhs + (b.col - offset);
      solve_lower(&factors[b.start], b.width, part);
      solve_upper_t(&factors[b.start], b.width, part);
    }
    for (size_t i = 0; i < n; ++i)
      if (owners[offset + i] == NONE && lambda != 0) rhs[i] /= lambda;
  }
};

// ---------------------------------------------------------------- Schur
struct Edge {
  size_t retained, eliminated, retained_jacobian, eliminated_jacobian;
};
struct Diagnostics {
  int termination;
  size_t iterations;
  double damping;
  double estimated, reduced, scaled, original;
  int has_estimated, has_reduced, has_scaled, has_original;
};
// LeastSquaresBackend (optimization.rs:131-169) as the optimizers see it; the
// step of the last solve is left in work.step.
struct Linear {
  StepWork work;
  size_t solves = 0, iterations = 0;
  virtual ~Linear() {}
  virtual int prepare(size_t dim) = 0;
  virtual void clear() = 0;
  virtual int accumulate(size_t nrows, const double* r, size_t nb, const size_t* bcols, const size_t* widths,
                         const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) = 0;
  virtual int gradient_norm(double* out) const = 0;
  virtual int prepare_damping(double floor) = 0;
  virtual int solve_damped(double lambda, double* predicted) = 0;
  virtual int solve() = 0;
};

struct Schur : Linear {
  size_t max_iterations = 1000;
  double relative_tolerance = std::max(1e-10, std::numeric_limits<double>::epsilon() * 128.);
  size_t retained, cw, pw;
  Model model;
  BlockFactors blocks;
  std::vector<Edge> edges;
  std::vector<double> cross, reduced_rhs, reduced_step, scaled_work, reduced_residual, tmp;
  bool ready = false;
  Diagnostics diag{};

  void cross_apply(double* out, const double* rhs, bool transpose, double alpha) const {  // :558-582
    for (size_t e = 0; e < edges.size(); ++e)
      for (size_t p = 0; p < pw; ++p)
        for (size_t c = 0; c < cw; ++c) {
          double v = alpha * cross[(e * pw + p) * cw + c];
          if (transpose)
            out[edges[e].eliminated + p] += v * rhs[edges[e].retained + c];
          else
            out[edges[e].retained + c] += v * rhs[edges[e].eliminated + p];
        }
  }
  void reduced_apply(const double* x, double* out, double lambda) {  // :606-652
    for (size_t i = 0; i < retained; ++i) out[i] = lambda * x[i];
    for (auto& b : blocks.blocks) {
      if (b.col >= retained) continue;
      const double* g = &blocks.gram[b.start];
      size_t w = b.width;
      for (size_t j = 0; j < w; ++j)
        for (size_t i = 0; i < w; ++i) out[b.col + i] += g[std::min(i, j) * w + std::max(i, j)] * x[b.col + j];
    }
    size_t elim = model.cols - retained;
    tmp.assign(elim, 0.);
    cross_apply(tmp.data(), x, true, 1.);
    blocks.solve_normal(tmp.data(), elim, retained, lambda);
    cross_apply(out, tmp.data(), false, -1.);
  }
  void precondition(const double* r, double* z, double lambda) {  // :670-677
    std::memcpy(z, r, retained * sizeof(double));
    blocks.solve_normal(z, retained, 0, lambda);
  }

  int prepare(size_t dim) override {  // :409-431
    ready = false;
    solves = iterations = 0;
    diag = Diagnostics{};
    if (cw == 0 || pw == 0 || retained > dim || retained % cw || (dim - retained) % pw || max_iterations == 0 ||
        !(relative_tolerance >= 0 && relative_tolerance < 1))
      return INVALID_OPTIONS;
    model.prepare(dim);
    work.step.assign(dim, 0.);
    reduced_rhs.assign(retained, 0.);
    reduced_step.assign(retained, 0.);
    reduced_residual.assign(retained, 0.);
    scaled_work.assign(dim, 0.);
    return OK;
  }
  void clear() override {  // :432-437
    ready = false;
    edges.clear();
    cross.clear();
    model.clear();
  }
  int accumulate(size_t nrows, const double* r, size_t nb, const size_t* bcols, const size_t* widths,
                 const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) override {  // :438-482
    ready = false;
    bool has_left = false, has_right = false;
    size_t lcol = 0, lidx = 0, rcol = 0, ridx = 0;
    size_t start = model.blocks.size();
    for (size_t i = 0; i < nb; ++i) {
      size_t col = bcols[i], end = col + widths[i];
      if (end < col || end > model.cols) return DIMENSION_MISMATCH;
      if (col < retained) {
        if (col % cw || widths[i] != cw || end > retained || has_left) return UNSUPPORTED_STRUCTURE;
        has_left = true; lcol = col; lidx = start + i;
      } else {
        if ((col - retained) % pw || widths[i] != pw || has_right) return UNSUPPORTED_STRUCTURE;
        has_right = true; rcol = col - retained; ridx = start + i;
      }
    }
    model.accumulate(nrows, r, nb, bcols, widths, jac, rs, cs);
    if (has_left && has_right) edges.push_back({lcol, rcol, lidx, ridx});
    return OK;
  }
  int gradient_norm(double* out) const override { return norm_inf(model.gradient.data(), model.cols, out); }
  int prepare_damping(double floor) override {  // :490-526
    ready = false;
    int s = model.prepare_scales(floor);
    if (s) return s;
    work.prepare_verification(model.rows, model.cols);
    s = blocks.prepare(model);
    if (s) return s;
    cross.assign(cw * pw * edges.size(), 0.);
    for (size_t e = 0; e < edges.size(); ++e) {
      const Block& l = model.blocks[edges[e].retained_jacobian];
      const Block& r = model.blocks[edges[e].eliminated_jacobian];
      for (size_t p = 0; p < pw; ++p)
        for (size_t c = 0; c < cw; ++c) {
          double sum = 0;
          for (size_t row = 0; row < l.rows; ++row)
            sum += (model.values[l.start + c * l.rows + row] / model.scales[l.col + c]) *
                   (model.values[r.start + p * r.rows + row] / model.scales[r.col + p]);
          cross[(e * pw + p) * cw + c] = sum;
        }
    }
    double m;
    if (norm_inf(cross.data(), cross.size(), &m)) return INVALID_EVALUATION;
    ready = true;
    return OK;
  }
  // faer CG restated for one column (see file header).
  void solve_reduced(double lambda) {  // :249-310
    size_t n = retained;
    std::fill(reduced_step.begin(), reduced_step.end(), 0.);
    std::vector<double> r(n), p(n), z(n), Ap(n);
    const double* b = reduced_rhs.data();
    double* x = reduced_step.data();
    double bnorm = norm_l2(b, n);
    diag.has_estimated = 0;
    if (bnorm == 0) {
      diag.termination = T_CONVERGED;
      diag.estimated = 0; diag.has_estimated = 1;
      return;
    }
    double threshold = relative_tolerance * bnorm;
    reduced_apply(x, r.data(), lambda);  // MaybeNonZero: r = b - A*0
    for (size_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
    double abs_res = norm_l2(r.data(), n);
    if (abs_res < threshold) {
      diag.termination = T_CONVERGED;
      diag.estimated = abs_res / bnorm; diag.has_estimated = 1;
      return;
    }
    precondition(r.data(), z.data(), lambda);
    p = z;
    double rz = 0;
    for (size_t i = 0; i < n; ++i) rz += r[i] * z[i];
    for (size_t it = 0; it < max_iterations; ++it) {
      reduced_apply(p.data(), Ap.data(), lambda);
      double pAp = 0;
      for (size_t i = 0; i < n; ++i) pAp += p[i] * Ap[i];
      if (!(pAp > 0)) { diag.termination = T_NOT_PD; return; }
      double alpha = rz / pAp;
      for (size_t i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
      ++iterations; ++diag.iterations;  // callback
      abs_res = norm_l2(r.data(), n);
      if (abs_res < threshold) {
        diag.termination = T_CONVERGED;
        diag.estimated = abs_res / bnorm; diag.has_estimated = 1;
        return;
      }
      precondition(r.data(), z.data(), lambda);
      double rz_new = 0;
      for (size_t i = 0; i < n; ++i) rz_new += r[i] * z[i];
      if (!(rz > 0)) { diag.termination = T_NOT_PD; return; }
      double beta = rz_new / rz;
      rz = rz_new;
      for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    diag.termination = T_ITERATION_LIMIT;
  }
  void recover_step(double lambda) {  // :312-344
    size_t n = model.cols;
    std::copy(reduced_step.begin(), reduced_step.end(), scaled_work.begin());
    for (size_t j = retained; j < n; ++j) scaled_work[j] = -model.gradient[j] / model.scales[j];
    cross_apply(scaled_work.data() + retained, reduced_step.data(), true, -1.);
    blocks.solve_normal(scaled_work.data() + retained, n - retained, retained, lambda);
    for (size_t j = 0; j < n; ++j) work.step[j] = scaled_work[j] / model.scales[j];
  }
  int verify(double lambda, double* predicted) {  // :346-397
    reduced_apply(reduced_step.data(), reduced_residual.data(), lambda);
    for (size_t i = 0; i < retained; ++i) reduced_residual[i] -= reduced_rhs[i];
    diag.reduced = relative(norm_l2(reduced_residual.data(), retained), norm_l2(reduced_rhs.data(), retained));
    diag.has_reduced = 1;
    Verification v = verify_step(model, work, lambda);
    diag.original = relative(v.residual_norm, v.reference_norm);
    diag.has_original = 1;
    for (size_t j = 0; j < model.cols; ++j) {
      work.normal_residual[j] /= model.scales[j];
      work.reference[j] /= model.scales[j];
    }
    diag.scaled = relative(norm_l2(work.normal_residual.data(), model.cols), norm_l2(work.reference.data(), model.cols));
    diag.has_scaled = 1;
    if (!v.finite_step || !is_fin(v.predicted) || !is_fin(diag.reduced) || !is_fin(diag.scaled) ||
        !is_fin(diag.original) || (diag.has_estimated && !is_fin(diag.estimated))) {
      diag.termination = T_NONFINITE;
      return LINEAR_SOLVE_FAILED;
    }
    if (diag.termination != T_CONVERGED) return LINEAR_SOLVE_FAILED;
    *predicted = v.predicted;
    return OK;
  }
  int solve_damped(double lambda, double* predicted) override {  // :527-545, :192-247
    diag = Diagnostics{};
    diag.damping = lambda;
    if (!ready || !is_fin(lambda) || lambda < 0) return INVALID_OPTIONS;
    ++solves;
    if (blocks.factor(lambda) != 0) {
      diag.termination = T_NOT_PD;
      return LINEAR_SOLVE_FAILED;
    }
    size_t n = model.cols;
    for (size_t j = 0; j < n; ++j) scaled_work[j] = -model.gradient[j] / model.scales[j];
    blocks.solve_normal(scaled_work.data() + retained, n - retained, retained, lambda);
    std::copy(scaled_work.begin(), scaled_work.begin() + retained, reduced_rhs.begin());
    cross_apply(reduced_rhs.data(), scaled_work.data() + retained, false, -1.);
    solve_reduced(lambda);
    recover_step(lambda);
    return verify(lambda, predicted);
  }
  int solve() override {  // :486-489
    int s = prepare_damping(1e-6);
    if (s) return s;
    double predicted;
    return solve_damped(0., &predicted);
  }
};

// ------------------------------------------------------------------ LSMR
// src/lsmr.rs:126-595 and src/lsmr/preconditioner.rs. The iterative core is
// faer 0.24.4's matrix_free::lsmr (called at src/lsmr.rs:240-261; faer's
// source is not part of the fagra tree), restated here from Fong & Saunders,
// "LSMR: an iterative algorithm for sparse least-squares problems", SIAM J.
// Sci. Comput. 33(5), 2011, Algorithm 1, for one right-hand side with:
//  - a zero initial guess (InitialGuessStatus::Zero);
//  - a right preconditioner M: the iteration runs on A M and returns x = M y;
//  - the stopping test ||(A M)^T r|| <= rel_tol * ||(A M)^T b|| on the
//    recurrence estimate |zetabar|, made before each iteration, so an
//    iteration budget of k always performs k iterations when the start is
//    not already converged (src/lsmr.rs:733-777 pins this: a system that one
//    iteration solves exactly still reports IterationLimit at max 1);
//  - the per-iteration callback counting iterations.
// Zero norms leave the Golub-Kahan vector at zero instead of dividing.
enum { MODE_IDENTITY = 0, MODE_DIAGONAL = 1, MODE_BLOCK = 2, MODE_NONE = -1 };
struct LsmrDiagnostics {  // src/lsmr.rs:68-104 (has_* = Some)
  int termination;
  size_t iterations;
  int finite_step;
  double estimated_absolute, estimated_relative, original_absolute, original_relative, scaled_absolute,
      scaled_relative, min_scale, max_scale, damping;
  size_t block_fallbacks;
  int has_estimated, has_original, has_scaled, has_scales, has_damping;
};

// y = op(x) for an operator of shape m x n and its transpose.
struct LsmrOperator {
  size_t m, n;
  virtual ~LsmrOperator() {}
  virtual void apply(const double* x, double* out) const = 0;            // out[m]
  virtual void transpose_apply(const double* y, double* out) const = 0;  // out[n]
};
// FactorPreconditioner (preconditioner.rs): M = L^-T per block, M^T = L^-1;
// absent factors make it the identity.
struct LsmrPrecond {
  const BlockFactors* factors = nullptr;
  void apply(double* v) const {
    if (factors) factors->apply_factor_inverse(v, false);
  }
  void transpose_apply(double* v) const {
    if (factors) factors->apply_factor_inverse(v, true);
  }
};
struct LsmrResult {
  bool converged;
  double abs_residual, rel_residual;
};

LsmrResult lsmr_core(const LsmrOperator& A, const LsmrPrecond& M, const double* b, double* x, double rel_tol,
                     size_t max_iters, size_t* iterations) {
  size_t m = A.m, n = A.n;
  std::vector<double> u(b, b + m), v(n), t(n), h(n), hbar(n, 0.), y(n, 0.), w(m);
  auto scale = [](std::vector<double>& z, double s) {
    if (s > 0)
      for (double& e : z) e /= s;
  };
  double beta = norm_l2(u.data(), m);
  scale(u, beta);
  A.transpose_apply(u.data(), v.data());
  M.transpose_apply(v.data());
  double alpha = norm_l2(v.data(), n);
  scale(v, alpha);
  double zetabar = alpha * beta, alphabar = alpha, rho = 1, rhobar = 1, cbar = 1, sbar = 0;
  h = v;
  double normar0 = alpha * beta, normar = normar0;
  std::fill(x, x + n, 0.);
  if (normar0 == 0) return {true, 0., 0.};
  double threshold = rel_tol * normar0;
  auto solution = [&]() {  // x = M y
    t = y;
    M.apply(t.data());
    std::copy(t.begin(), t.end(), x);
  };
  for (size_t it = 0; it < max_iters; ++it) {
    if (normar <= threshold) {
      solution();
      return {true, normar, normar / normar0};
    }
    // Golub-Kahan step on A M.
    t = v;
    M.apply(t.data());
    A.apply(t.data(), w.data());
    for (size_t i = 0; i < m; ++i) u[i] = w[i] - alpha * u[i];
    beta = norm_l2(u.data(), m);
    scale(u, beta);
    A.transpose_apply(u.data(), t.data());
    M.transpose_apply(t.data());
    for (size_t j = 0; j < n; ++j) v[j] = t[j] - beta * v[j];
    alpha = norm_l2(v.data(), n);
    scale(v, alpha);
    // Rotations (Algorithm 1, steps 4-5).
    double rhoold = rho;
    rho = std::hypot(alphabar, beta);
    double c = alphabar / rho, s = beta / rho;
    double thetanew = s * alpha;
    alphabar = c * alpha;
    double rhobarold = rhobar;
    double thetabar = sbar * rho;
    double crho = cbar * rho;
    rhobar = std::hypot(crho, thetanew);
    cbar = crho / rhobar;
    sbar = thetanew / rhobar;
    double zeta = cbar * zetabar;
    zetabar = -sbar * zetabar;
    // Updates (step 6).
    double fhbar = thetabar * rho / (rhoold * rhobarold), fy = zeta / (rho * rhobar), fh = thetanew / rho;
    for (size_t j = 0; j < n; ++j) {
      hbar[j] = h[j] - fhbar * hbar[j];
      y[j] += fy * hbar[j];
      h[j] = v[j] - fh * h[j];
    }
    normar = std::fabs(zetabar);
    ++*iterations;  // callback
  }
  solution();
  return {false, normar, normar / normar0};
}

// Jacobian alone (the undamped solve) and the Damped augmented operator
// [J D^-1; diag] / [J; diag] (src/lsmr.rs:128-224).
struct JacobianOp : LsmrOperator {
  const Model* model;
  void apply(const double* x, double* out) const override { model->apply(x, out); }
  void transpose_apply(const double* y, double* out) const override { model->transpose_apply(y, out); }
};
struct DampedOp : LsmrOperator {
  const Model* model;
  const double* diagonal;
  const double* scales;  // null: no scaling
  mutable std::vector<double> tmp;
  void apply(const double* x, double* out) const override {
    size_t r = model->rows, c = model->cols;
    if (scales) {
      tmp.resize(c);
      for (size_t j = 0; j < c; ++j) tmp[j] = x[j] / scales[j];
      model->apply(tmp.data(), out);
    } else {
      model->apply(x, out);
    }
    for (size_t j = 0; j < c; ++j) out[r + j] = diagonal[j] * x[j];
  }
  void transpose_apply(const double* y, double* out) const override {
    size_t r = model->rows, c = model->cols;
    model->transpose_apply(y, out);
    for (size_t j = 0; j < c; ++j) {
      if (scales) out[j] /= scales[j];
      out[j] += diagonal[j] * y[r + j];
    }
  }
};

struct Lsmr : Linear {
  size_t max_iterations = 1000;
  double relative_tolerance = std::max(1e-10, std::numeric_limits<double>::epsilon() * 128.);
  bool diagonal_preconditioning = true, block_preconditioning = false;
  Model model;
  BlockFactors blocks;
  std::vector<double> diagonal, augmented_rhs;
  int prepared_mode = MODE_NONE;
  LsmrDiagnostics diag{};

  int requested_mode() const {  // :391-399
    return block_preconditioning ? MODE_BLOCK : diagonal_preconditioning ? MODE_DIAGONAL : MODE_IDENTITY;
  }
  // The shared solve() helper, src/lsmr.rs:228-288.
  int run(const LsmrOperator& op, const LsmrPrecond& pre, const double* rhs) {
    size_t n = op.n;
    work.step.assign(n, 0.);
    if (op.m == 0 || n == 0) {
      diag.termination = T_CONVERGED;
      diag.finite_step = 1;
      return OK;
    }
    ++solves;
    size_t its = 0;
    LsmrResult res = lsmr_core(op, pre, rhs, work.step.data(), relative_tolerance, max_iterations, &its);
    iterations += its;
    diag.iterations += its;
    diag.estimated_absolute = res.abs_residual;
    diag.estimated_relative = res.rel_residual;
    diag.has_estimated = 1;
    double tmp;
    diag.finite_step = norm_inf(work.step.data(), n, &tmp) == OK;
    if (diag.finite_step && is_fin(res.abs_residual) && is_fin(res.rel_residual))
      diag.termination = res.converged ? T_CONVERGED : T_ITERATION_LIMIT;
    else
      diag.termination = T_NONFINITE;
    return diag.termination == T_CONVERGED ? OK : LINEAR_SOLVE_FAILED;
  }
  int prepare(size_t dim) override {  // :469-480
    solves = iterations = 0;
    diag = LsmrDiagnostics{};
    prepared_mode = MODE_NONE;
    if (max_iterations == 0 || !(relative_tolerance >= 0 && relative_tolerance < 1)) return INVALID_OPTIONS;
    model.prepare(dim);
    work.step.assign(dim, 0.);
    return OK;
  }
  void clear() override {  // :482-485
    prepared_mode = MODE_NONE;
    model.clear();
  }
  int accumulate(size_t nrows, const double* r, size_t nb, const size_t* bcols, const size_t* widths,
                 const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) override {  // :487-494
    prepared_mode = MODE_NONE;
    for (size_t i = 0; i < nb; ++i)
      if (bcols[i] + widths[i] < bcols[i] || bcols[i] + widths[i] > model.cols) return DIMENSION_MISMATCH;
    return model.accumulate(nrows, r, nb, bcols, widths, jac, rs, cs);
  }
  int gradient_norm(double* out) const override { return norm_inf(model.gradient.data(), model.cols, out); }
  int solve() override {  // :500-520
    diag = LsmrDiagnostics{};
    JacobianOp op;
    op.m = model.rows;
    op.n = model.cols;
    op.model = &model;
    return run(op, LsmrPrecond{}, model.negative_residual.data());
  }
  int prepare_damping(double floor) override {  // :521-546
    prepared_mode = MODE_NONE;
    int s = model.prepare_scales(floor);
    if (s) return s;
    int mode = requested_mode();
    diagonal.assign(model.cols, 0.);
    work.prepare_verification(model.rows, model.cols);
    if (mode == MODE_BLOCK && (s = blocks.prepare(model))) return s;
    augmented_rhs.assign(model.rows + model.cols, 0.);
    std::copy(model.negative_residual.begin(), model.negative_residual.end(), augmented_rhs.begin());
    prepared_mode = mode;
    return OK;
  }
  // recover_and_verify, :418-456; returns the status, predicted in *predicted.
  int recover_and_verify(double lambda, int mode, double* predicted) {
    size_t n = model.cols;
    if (mode != MODE_IDENTITY)
      for (size_t j = 0; j < n; ++j) work.step[j] /= model.scales[j];
    Verification v = verify_step(model, work, lambda);
    diag.finite_step = v.finite_step;
    if (mode != MODE_IDENTITY)
      for (size_t j = 0; j < n; ++j) {
        work.normal_residual[j] /= model.scales[j];
        work.reference[j] /= model.scales[j];
      }
    if (mode == MODE_BLOCK) {
      blocks.apply_factor_inverse(work.normal_residual.data(), true);
      blocks.apply_factor_inverse(work.reference.data(), true);
    }
    double scaled_norm = norm_l2(work.normal_residual.data(), n);
    double scaled_reference = norm_l2(work.reference.data(), n);
    diag.original_absolute = v.residual_norm;
    diag.original_relative = relative(v.residual_norm, v.reference_norm);
    diag.scaled_absolute = scaled_norm;
    diag.scaled_relative = relative(scaled_norm, scaled_reference);
    diag.has_original = diag.has_scaled = 1;
    if (!v.finite_step || !is_fin(v.residual_norm) || !is_fin(scaled_norm)) {
      diag.termination = T_NONFINITE;
      return LINEAR_SOLVE_FAILED;
    }
    *predicted = v.predicted;
    return OK;
  }
  int solve_damped(double lambda, double* predicted) override {  // :548-585
    diag = LsmrDiagnostics{};
    int mode = prepared_mode;
    if (mode == MODE_NONE || mode != requested_mode() || !is_fin(lambda) || lambda < 0) return INVALID_OPTIONS;
    double root = std::sqrt(lambda);
    bool scaled = mode != MODE_IDENTITY;
    diag.damping = lambda;
    diag.has_damping = 1;
    if (model.cols) {
      diag.min_scale = *std::min_element(model.scales.begin(), model.scales.end());
      diag.max_scale = *std::max_element(model.scales.begin(), model.scales.end());
      diag.has_scales = 1;
    }
    for (size_t j = 0; j < model.cols; ++j) diagonal[j] = scaled ? root : root * model.scales[j];
    double tmp;
    if (norm_inf(diagonal.data(), model.cols, &tmp)) {
      diag.termination = T_NONFINITE;
      return LINEAR_SOLVE_FAILED;
    }
    if (mode == MODE_BLOCK) diag.block_fallbacks = blocks.factor(lambda);
    DampedOp op;
    op.m = model.rows + model.cols;
    op.n = model.cols;
    op.model = &model;
    op.diagonal = diagonal.data();
    op.scales = scaled ? model.scales.data() : nullptr;
    LsmrPrecond pre;
    if (mode == MODE_BLOCK) pre.factors = &blocks;
    int result = run(op, pre, augmented_rhs.data());
    double p = 0;
    int verified = recover_and_verify(lambda, mode, &p);
    if (verified) return verified;
    if (result) return result;
    *predicted = p;
    return OK;
  }
};

// cross_apply indexes rhs/out with edge offsets relative to each partition;
// the calls above pass partition base pointers, matching schur.rs:230-242,319-331.

#include "dense.hpp"

// ------------------------------------------------------ Problems for LM/GN
// A problem exposes the callbacks the optimizers need; the BAL problem below
// and the host-callback problem used by the scalar tests both implement it.
struct Problem {
  virtual ~Problem() {}
  virtual size_t dimension() = 0;
  virtual int cost(bool trial, double* out) = 0;  // optimization.rs:419-430
  virtual int linearize(Linear& s) = 0;             // :229-265
  virtual int stage(const double* delta) = 0;      // :432-459
  virtual void accept() = 0;
  virtual void reject() = 0;
};

// checked_cost, storage.rs:612-618
int checked(int st, double c) {
  if (st) return st;
  if (!is_fin(c) || c < 0) return INVALID_EVALUATION;
  return OK;
}

struct BalProblem : Problem {
  size_t nc, np, no;
  std::vector<double> cams, pts, tcams, tpts;
  std::vector<uint32_t> oc, op;
  std::vector<double> px;
  std::vector<size_t> order;     // emission order: stable by camera (frames in camera order)
  std::vector<size_t> frame_off; // nc+1
  bool trial_active = false;

  BalProblem(size_t c, size_t p, size_t o, const double* cp, const double* pp, const uint32_t* ocam,
             const uint32_t* opt, const double* pix)
      : nc(c), np(p), no(o), cams(cp, cp + 9 * c), pts(pp, pp + 3 * p), oc(ocam, ocam + o), op(opt, opt + o),
        px(pix, pix + 2 * o) {
    frame_off.assign(nc + 1, 0);
    for (size_t i = 0; i < no; ++i) frame_off[oc[i] + 1]++;
    for (size_t i = 0; i < nc; ++i) frame_off[i + 1] += frame_off[i];
    order.resize(no);
    std::vector<size_t> fill(frame_off.begin(), frame_off.end() - 1);
    for (size_t i = 0; i < no; ++i) order[fill[oc[i]]++] = i;
  }
  size_t dimension() override { return 9 * nc + 3 * np; }
  // Frame::cost, model.rs:201-213, summed per frame in frame order.
  int cost(bool trial, double* out) override {
    const double* C = trial ? tcams.data() : cams.data();
    const double* P = trial ? tpts.data() : pts.data();
    double total = 0;
    for (size_t c = 0; c < nc; ++c) {
      if (frame_off[c] == frame_off[c + 1]) continue;
      Projection pr;
      projection_new(C + 9 * c, &pr);
      double fc = 0;
      for (size_t k = frame_off[c]; k < frame_off[c + 1]; ++k) {
        size_t i = order[k];
        double pix[2];
        if (projection_value(pr, P + 3 * op[i], pix)) return INVALID_EVALUATION;
        double r0 = pix[0] - px[2 * i], r1 = pix[1] - px[2 * i + 1];
        fc += 0.5 * (r0 * r0 + r1 * r1);
      }
      int st = checked(OK, fc);
      if (st) return st;
      total += fc;
    }
    *out = total;
    return checked(OK, total);
  }
  // Frame::linearize, model.rs:214-236 through CheckedSink (optimization.rs:541-612).
  int linearize(Linear& s) override {
    s.clear();
    for (size_t c = 0; c < nc; ++c) {
      if (frame_off[c] == frame_off[c + 1]) continue;
      Projection pr;
      projection_new(&cams[9 * c], &pr);
      for (size_t k = frame_off[c]; k < frame_off[c + 1]; ++k) {
        size_t i = order[k];
        const double* X = &pts[3 * op[i]];
        double pix[2];
        if (projection_value(pr, X, pix)) return INVALID_EVALUATION;
        double r[2] = {pix[0] - px[2 * i], pix[1] - px[2 * i + 1]};
        double jc[18], jp[6];
        projection_jacobians(pr, X, jc, jp);
        for (double v : r) if (!is_fin(v)) return INVALID_EVALUATION;
        for (double v : jc) if (!is_fin(v)) return INVALID_EVALUATION;
        for (double v : jp) if (!is_fin(v)) return INVALID_EVALUATION;
        size_t cols[2] = {9 * c, 9 * nc + 3 * op[i]};
        size_t widths[2] = {9, 3};
        const double* jac[2] = {jc, jp};
        ptrdiff_t rs[2] = {1, 1}, cs[2] = {2, 2};
        int st = s.accumulate(2, r, 2, cols, widths, jac, rs, cs);
        if (st) return st;
      }
    }
    return OK;
  }
  int stage(const double* d) override {  // additive retraction of Camera/Point
    tcams.resize(cams.size());
    tpts.resize(pts.size());
    for (size_t i = 0; i < cams.size(); ++i) tcams[i] = cams[i] + d[i];
    for (size_t i = 0; i < pts.size(); ++i) tpts[i] = pts[i] + d[cams.size() + i];
    trial_active = true;
    return OK;
  }
  void accept() override {
    if (trial_active) {
      cams.swap(tcams);
      pts.swap(tpts);
      trial_active = false;
    }
  }
  void reject() override { trial_active = false; }
};

// Callback problem: variables are additive real vectors with the given widths,
// factors are evaluated by the caller.
typedef int (*cb_cost_t)(void* user, const double* x, double* out);
typedef int (*cb_linearize_t)(void* user, const double* x, void* sink);
struct CallbackProblem : Problem {
  size_t dim;
  std::vector<double> x, tx;
  bool trial = false;
  cb_cost_t cb_cost;
  cb_linearize_t cb_lin;
  void* user;
  Linear* sink = nullptr;
  size_t dimension() override { return dim; }
  int cost(bool t, double* out) override {
    double c = 0;
    int st = cb_cost(user, t ? tx.data() : x.data(), &c);
    *out = c;
    return checked(st, c);
  }
  int linearize(Linear& s) override {
    s.clear();
    sink = &s;
    return cb_lin(user, x.data(), this);
  }
  int stage(const double* d) override {
    tx.resize(dim);
    for (size_t i = 0; i < dim; ++i) tx[i] = x[i] + d[i];
    trial = true;
    return OK;
  }
  void accept() override {
    if (trial) { x.swap(tx); trial = false; }
  }
  void reject() override { trial = false; }
};

// ------------------------------------------------------------- optimizers
struct OptimizeOptions {
  size_t max_iterations;
  double gradient_tolerance, step_tolerance, cost_tolerance;
};
struct LmOptions {
  double initial_damping, min_damping, max_damping, min_column_norm, acceptance_threshold;
  size_t max_trials;
};
struct Report {
  size_t iterations;
  double initial_cost, final_cost;
  int termination;  // 0 none, 1 NoVariables, 2 GradientTolerance, 3 StepTolerance, 4 CostTolerance
};
struct LmStats {
  size_t linearizations, attempts, rejected_steps, accepted_steps, cost_evaluations;
  double damping, cost, gradient_norm, step_norm;
  int has_cost, has_gradient_norm, has_step_norm, last_rejection;  // 0 none,1 LinearSolve,2 Prediction,3 InvalidEvaluation,4 PoorAgreement
  size_t linear_solves, linear_iterations;
};
typedef void (*accept_cb_t)(void* user, const LmStats* stats);

int validate(const OptimizeOptions& o) {  // optimization.rs:69-84
  double v[3] = {o.gradient_tolerance, o.step_tolerance, o.cost_tolerance};
  if (o.max_iterations == 0) return INVALID_OPTIONS;
  for (double x : v) if (!is_fin(x) || x < 0) return INVALID_OPTIONS;
  return OK;
}
int validate(const LmOptions& o) {  // levenberg_marquardt.rs:47-67
  double v[5] = {o.initial_damping, o.min_damping, o.max_damping, o.min_column_norm, o.acceptance_threshold};
  if (o.max_trials == 0) return INVALID_OPTIONS;
  for (double x : v) if (!is_fin(x) || x <= 0) return INVALID_OPTIONS;
  if (o.min_damping > o.initial_damping || o.initial_damping > o.max_damping || o.acceptance_threshold >= 1)
    return INVALID_OPTIONS;
  return OK;
}

// levenberg_marquardt.rs:330-472
// target_cost > 0: also stop (termination 5) once an accepted cost is at or
// below it, the stopping rule of the time-to-cost measurement.
int lm_optimize(Linear& s, Problem& pb, const OptimizeOptions& opt, const LmOptions& lo, Report* rep, LmStats* st,
                accept_cb_t on_accept, void* user, double target_cost = 0.0) {
  *st = LmStats{};
  int e;
  if ((e = validate(opt)) || (e = validate(lo))) return e;
  double lambda = lo.initial_damping;
  st->damping = lambda;
  if ((e = s.prepare(pb.dimension()))) return e;
  st->cost_evaluations += 1;
  double initial;
  if ((e = pb.cost(false, &initial))) return e;
  st->cost = initial; st->has_cost = 1;
  double current = initial;
  bool stalled = false, tried_undamped = false;
  rep->initial_cost = initial;
  auto finish = [&](int term) {
    rep->final_cost = current;
    rep->iterations = st->accepted_steps;
    rep->termination = term;
    st->linear_solves = s.solves;
    st->linear_iterations = s.iterations;
    return OK;
  };
  for (;;) {
    if (pb.dimension() == 0) return finish(1);
    st->linearizations += 1;
    if ((e = pb.linearize(s))) return e;
    double g;
    if ((e = s.gradient_norm(&g))) return e;
    st->gradient_norm = g; st->has_gradient_norm = 1;
    if (g <= opt.gradient_tolerance) return finish(2);
    if (stalled && (tried_undamped || st->accepted_steps == opt.max_iterations)) return NO_PROGRESS;
    if (st->accepted_steps == opt.max_iterations) return NO_CONVERGENCE;
    if ((e = s.prepare_damping(lo.min_column_norm))) return e;
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
      int r = s.solve_damped(damping, &predicted);
      if (r == LINEAR_SOLVE_FAILED) {
        rejection = 1;
      } else if (r) {
        return r;
      } else {
        double norm;
        if (norm_inf(s.work.step.data(), s.work.step.size(), &norm)) return LINEAR_SOLVE_FAILED;
        st->step_norm = norm; st->has_step_norm = 1;
        if (!is_fin(predicted) || predicted <= 0) {
          rejection = 2;
        } else {
          pb.stage(s.work.step.data());
          st->cost_evaluations += 1;
          double value;
          int ce = pb.cost(true, &value);
          if (ce == INVALID_EVALUATION) {
            pb.reject();
            rejection = 3;
          } else if (ce) {
            pb.reject();
            return ce;
          } else {
            double actual = current - value;
            double ratio = std::min(actual / predicted, 2.0);
            if (actual > 0 && ratio >= lo.acceptance_threshold) {
              pb.accept();
              st->accepted_steps += 1;
              st->cost = value; st->has_cost = 1;
              stalled = opt.step_tolerance > 0 && norm <= opt.step_tolerance &&
                        (opt.cost_tolerance == 0 || actual / std::max(current, 1.0) <= opt.cost_tolerance);
              current = value;
              double c = 2.0 * std::min(ratio, 1.0) - 1.0;
              double update = std::max(1.0 - c * c * c, 1.0 / 3.0);
              lambda = std::min(std::max(lambda * update, lo.min_damping), lo.max_damping);
              accepted = true;
              st->linear_solves = s.solves;
              st->linear_iterations = s.iterations;
              if (on_accept) on_accept(user, st);
              if (target_cost > 0 && current <= target_cost) return finish(5);
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
    st->linear_solves = s.solves;
    st->linear_iterations = s.iterations;
    if (!accepted) return NO_PROGRESS;
  }
}

// gauss_newton.rs:101-176; the backend's solve() is Schur's prepare_damping +
// solve_damped(0) (schur.rs:486-489) or LSMR's undamped solve (lsmr.rs:500-520).
int gn_optimize(Linear& s, Problem& pb, const OptimizeOptions& opt, Report* rep) {
  int e;
  if ((e = validate(opt))) return e;
  if ((e = s.prepare(pb.dimension()))) return e;
  double initial;
  if ((e = pb.cost(false, &initial))) return e;
  double current = initial;
  size_t its = 0;
  rep->initial_cost = initial;
  auto report = [&](int term) {
    rep->final_cost = current;
    rep->iterations = its;
    rep->termination = term;
    return OK;
  };
  if (pb.dimension() == 0) return report(1);
  for (;;) {
    if ((e = pb.linearize(s))) return e;
    double g;
    if ((e = s.gradient_norm(&g))) return e;
    if (g <= opt.gradient_tolerance) return report(2);
    if (its == opt.max_iterations) return NO_CONVERGENCE;
    if ((e = s.solve())) return e;
    double norm;
    if (norm_inf(s.work.step.data(), s.work.step.size(), &norm)) return LINEAR_SOLVE_FAILED;
    if (norm <= opt.step_tolerance) return report(3);
    pb.stage(s.work.step.data());
    double tc;
    if ((e = pb.cost(true, &tc))) { pb.reject(); return e; }
    pb.accept();
    ++its;
    double dec = current - tc;
    bool conv = tc == 0 || (dec >= 0 && dec / std::max(current, 1.0) <= opt.cost_tolerance);
    current = tc;
    if (conv) return report(4);
  }
}

#include "posegraph.hpp"

}  // namespace

// ================================================================ C ABI
OR_API int or_bal_project(const double* cam, const double* X, double* pix) {
  Projection p;
  projection_new(cam, &p);
  return projection_value(p, X, pix);
}
OR_API void or_bal_jacobians(const double* cam, const double* X, double* jc, double* jp) {
  Projection p;
  projection_new(cam, &p);
  projection_jacobians(p, X, jc, jp);
}
OR_API void or_rotation(const double* w, double* R) { rotation_from_scaled_axis(w, R); }

// Backend handles are Linear* (Schur or Lsmr); the prepare / clear /
// accumulate / gradient / damping / solve / work entry points below dispatch
// on the dynamic type.
static Linear* LIN(void* h) { return (Linear*)h; }
static Schur* SCH(void* h) { return static_cast<Schur*>(LIN(h)); }
static Lsmr* LSM(void* h) { return static_cast<Lsmr*>(LIN(h)); }

OR_API void* or_schur_create(size_t retained, size_t cw, size_t pw) {
  Schur* s = new Schur();
  s->retained = retained; s->cw = cw; s->pw = pw;
  return (void*)(Linear*)s;
}
OR_API void or_schur_destroy(void* h) { delete LIN(h); }
OR_API void or_schur_set_limits(void* h, size_t max_iterations, double rel_tol) {
  SCH(h)->max_iterations = max_iterations;
  SCH(h)->relative_tolerance = rel_tol;
}
OR_API int or_schur_prepare(void* h, size_t dim) { return LIN(h)->prepare(dim); }
OR_API void or_schur_clear(void* h) { LIN(h)->clear(); }
OR_API int or_schur_accumulate(void* h, size_t rows, const double* r, size_t nb, const size_t* cols,
                               const size_t* widths, const double* const* jac, const ptrdiff_t* rs,
                               const ptrdiff_t* cs) {
  return LIN(h)->accumulate(rows, r, nb, cols, widths, jac, rs, cs);
}
OR_API int or_schur_gradient_norm(void* h, double* out) { return LIN(h)->gradient_norm(out); }
OR_API int or_schur_prepare_damping(void* h, double floor) { return LIN(h)->prepare_damping(floor); }
OR_API int or_schur_solve_damped(void* h, double lambda, double* delta, double* predicted) {
  Linear* s = LIN(h);
  double pred = 0;
  int st = s->solve_damped(lambda, &pred);
  if (st == OK || st == LINEAR_SOLVE_FAILED)
    if (delta) std::copy(s->work.step.begin(), s->work.step.end(), delta);
  if (predicted) *predicted = pred;
  return st;
}
OR_API int or_schur_solve(void* h, double* delta) {
  Linear* s = LIN(h);
  int st = s->solve();
  if ((st == OK || st == LINEAR_SOLVE_FAILED) && delta) std::copy(s->work.step.begin(), s->work.step.end(), delta);
  return st;
}
OR_API void or_schur_work(void* h, size_t* solves, size_t* iterations) {
  *solves = LIN(h)->solves;
  *iterations = LIN(h)->iterations;
}

// LSMR backend (src/lsmr.rs).
OR_API void* or_lsmr_create(void) { return (void*)(Linear*)new Lsmr(); }
OR_API void or_lsmr_set(void* h, size_t max_iterations, double rel_tol, int diagonal, int block) {
  Lsmr* s = LSM(h);
  s->max_iterations = max_iterations;
  s->relative_tolerance = rel_tol;
  s->diagonal_preconditioning = diagonal != 0;
  s->block_preconditioning = block != 0;
}
OR_API void or_lsmr_diagnostics(void* h, LsmrDiagnostics* d) { *d = LSM(h)->diag; }
// The Damped operator at damping lambda (scaled: [J D^-1; sqrt(lambda) I],
// else [J; sqrt(lambda) D]) applied to x[n] -> fwd[m+n] and to y[m+n] -> tr[n].
OR_API void or_lsmr_damped_products(void* h, double lambda, int scaled, const double* x, double* fwd,
                                    const double* y, double* tr) {
  Lsmr* s = LSM(h);
  std::vector<double> diagonal(s->model.cols);
  for (size_t j = 0; j < diagonal.size(); ++j)
    diagonal[j] = scaled ? std::sqrt(lambda) : std::sqrt(lambda) * s->model.scales[j];
  DampedOp op;
  op.m = s->model.rows + s->model.cols;
  op.n = s->model.cols;
  op.model = &s->model;
  op.diagonal = diagonal.data();
  op.scales = scaled ? s->model.scales.data() : nullptr;
  op.apply(x, fwd);
  op.transpose_apply(y, tr);
}
// Block factors of the last damped solve: L^-T x and L^-1 y per variable block.
OR_API void or_lsmr_precond(void* h, const double* x, double* px, const double* y, double* pty) {
  Lsmr* s = LSM(h);
  size_t n = s->model.cols;
  std::copy(x, x + n, px);
  std::copy(y, y + n, pty);
  s->blocks.apply_factor_inverse(px, false);
  s->blocks.apply_factor_inverse(pty, true);
}
OR_API void or_lsmr_scales(void* h, double* scales) {
  Lsmr* s = LSM(h);
  std::copy(s->model.scales.begin(), s->model.scales.end(), scales);
}
OR_API void or_schur_diagnostics(void* h, Diagnostics* d) { *d = SCH(h)->diag; }
OR_API void or_schur_sizes(void* h, size_t* nblocks, size_t* nedges, size_t* nvalues, size_t* nvar, size_t* ngram,
                           size_t* rows, size_t* cols) {
  Schur* s = SCH(h);
  *nblocks = s->model.blocks.size();
  *nedges = s->edges.size();
  *nvalues = s->model.values.size();
  *nvar = s->blocks.blocks.size();
  *ngram = s->blocks.gram.size();
  *rows = s->model.rows;
  *cols = s->model.cols;
}
// Structure and model export for bit-exact index-map and value checks.
OR_API void or_schur_export(void* h, size_t* blocks5, size_t* edges4, size_t* owners, size_t* var3, double* values,
                            double* negres, double* gradient, double* scales, double* gram, double* cross) {
  Schur* s = SCH(h);
  for (size_t i = 0; i < s->model.blocks.size(); ++i) {
    const Block& b = s->model.blocks[i];
    size_t v[5] = {b.row, b.col, b.rows, b.cols, b.start};
    std::copy(v, v + 5, blocks5 + 5 * i);
  }
  for (size_t i = 0; i < s->edges.size(); ++i) {
    const Edge& e = s->edges[i];
    size_t v[4] = {e.retained, e.eliminated, e.retained_jacobian, e.eliminated_jacobian};
    std::copy(v, v + 4, edges4 + 4 * i);
  }
  if (owners) std::copy(s->blocks.owners.begin(), s->blocks.owners.end(), owners);
  for (size_t i = 0; i < s->blocks.blocks.size(); ++i) {
    var3[3 * i] = s->blocks.blocks[i].col;
    var3[3 * i + 1] = s->blocks.blocks[i].width;
    var3[3 * i + 2] = s->blocks.blocks[i].start;
  }
  if (values) std::copy(s->model.values.begin(), s->model.values.end(), values);
  if (negres) std::copy(s->model.negative_residual.begin(), s->model.negative_residual.end(), negres);
  if (gradient) std::copy(s->model.gradient.begin(), s->model.gradient.end(), gradient);
  if (scales) std::copy(s->model.scales.begin(), s->model.scales.end(), scales);
  if (gram) std::copy(s->blocks.gram.begin(), s->blocks.gram.end(), gram);
  if (cross) std::copy(s->cross.begin(), s->cross.end(), cross);
}
// Reduced operator and preconditioner, for operator-level checks.
OR_API void or_schur_reduced_apply(void* h, double lambda, const double* x, double* y) {
  Schur* s = SCH(h);
  s->blocks.factor(lambda);
  s->reduced_apply(x, y, lambda);
}
OR_API void or_schur_reduced_rhs(void* h, double* rhs) {
  Schur* s = SCH(h);
  std::copy(s->reduced_rhs.begin(), s->reduced_rhs.end(), rhs);
}

// Model-level entry points for linear_model.rs:344-367.
OR_API void* or_model_create(size_t dim) {
  Model* m = new Model();
  m->prepare(dim);
  return m;
}
OR_API void or_model_destroy(void* h) { delete (Model*)h; }
OR_API int or_model_accumulate(void* h, size_t rows, const double* r, size_t nb, const size_t* cols,
                               const size_t* widths, const double* const* jac, const ptrdiff_t* rs,
                               const ptrdiff_t* cs) {
  return ((Model*)h)->accumulate(rows, r, nb, cols, widths, jac, rs, cs);
}
OR_API int or_model_prepare_scales(void* h, double floor) { return ((Model*)h)->prepare_scales(floor); }
OR_API void or_model_verify(void* h, const double* step, double lambda, double* out4, double* normal_residual,
                            double* reference) {
  Model* m = (Model*)h;
  StepWork w;
  w.step.assign(step, step + m->cols);
  w.prepare_verification(m->rows, m->cols);
  Verification v = verify_step(*m, w, lambda);
  out4[0] = v.predicted;
  out4[1] = v.finite_step;
  out4[2] = v.residual_norm;
  out4[3] = v.reference_norm;
  std::copy(w.normal_residual.begin(), w.normal_residual.end(), normal_residual);
  std::copy(w.reference.begin(), w.reference.end(), reference);
}
OR_API void or_model_state(void* h, double* gradient, double* negres) {
  Model* m = (Model*)h;
  std::copy(m->gradient.begin(), m->gradient.end(), gradient);
  std::copy(m->negative_residual.begin(), m->negative_residual.end(), negres);
}

// BlockFactors-level entry points for block_factors.rs:211-245.
OR_API int or_blockfactors_run(size_t rows, size_t cols, size_t nblocks, const size_t* blocks5, const double* values,
                               size_t nvalues, const double* scales, const double* lambdas, size_t nl,
                               size_t* fallbacks) {
  Model m;
  m.rows = rows;
  m.cols = cols;
  for (size_t i = 0; i < nblocks; ++i)
    m.blocks.push_back({blocks5[5 * i], blocks5[5 * i + 1], blocks5[5 * i + 2], blocks5[5 * i + 3], blocks5[5 * i + 4]});
  m.values.assign(values, values + nvalues);
  m.scales.assign(scales, scales + cols);
  BlockFactors bf;
  int st = bf.prepare(m);
  if (st) return st;
  for (size_t i = 0; i < nl; ++i) fallbacks[i] = bf.factor(lambdas[i]);
  return OK;
}

// BAL problem + LM/GN with the Schur backend.
OR_API void* or_bal_create(size_t nc, size_t np, size_t no, const double* cams, const double* pts,
                           const uint32_t* oc, const uint32_t* op, const double* px) {
  return new BalProblem(nc, np, no, cams, pts, oc, op, px);
}
OR_API void or_bal_destroy(void* h) { delete (BalProblem*)h; }
OR_API int or_bal_cost(void* h, double* out) { return ((BalProblem*)h)->cost(false, out); }
OR_API void or_bal_get(void* h, double* cams, double* pts) {
  BalProblem* b = (BalProblem*)h;
  std::copy(b->cams.begin(), b->cams.end(), cams);
  std::copy(b->pts.begin(), b->pts.end(), pts);
}
OR_API void or_bal_order(void* h, size_t* order) {
  BalProblem* b = (BalProblem*)h;
  std::copy(b->order.begin(), b->order.end(), order);
}
OR_API int or_bal_linearize(void* bal, void* schur) { return ((BalProblem*)bal)->linearize(*(Linear*)schur); }

OR_API int or_lm_bal(void* schur, void* bal, const OptimizeOptions* opt, const LmOptions* lo, Report* rep,
                     LmStats* st, accept_cb_t cb, void* user) {
  return lm_optimize(*(Linear*)schur, *(BalProblem*)bal, *opt, *lo, rep, st, cb, user);
}
OR_API int or_lm_bal_to_cost(void* schur, void* bal, const OptimizeOptions* opt, const LmOptions* lo,
                             double target_cost, Report* rep, LmStats* st) {
  return lm_optimize(*(Linear*)schur, *(BalProblem*)bal, *opt, *lo, rep, st, nullptr, nullptr, target_cost);
}
OR_API int or_gn_bal(void* schur, void* bal, const OptimizeOptions* opt, Report* rep) {
  return gn_optimize(*(Linear*)schur, *(BalProblem*)bal, *opt, rep);
}

// Callback problems (scalar/vector test graphs).
OR_API void* or_cbproblem_create(size_t dim, const double* x0, cb_cost_t c, cb_linearize_t l, void* user) {
  CallbackProblem* p = new CallbackProblem();
  p->dim = dim;
  p->x.assign(x0, x0 + dim);
  p->cb_cost = c;
  p->cb_lin = l;
  p->user = user;
  return p;
}
OR_API void or_cbproblem_destroy(void* h) { delete (CallbackProblem*)h; }
OR_API void or_cbproblem_get(void* h, double* x) {
  CallbackProblem* p = (CallbackProblem*)h;
  std::copy(p->x.begin(), p->x.end(), x);
}
// Emission entry used by callback linearizers: forwards to the active Schur sink.
OR_API int or_cbproblem_emit(void* sink, size_t rows, const double* r, size_t nb, const size_t* cols,
                             const size_t* widths, const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) {
  CallbackProblem* p = (CallbackProblem*)sink;
  for (size_t i = 0; i < rows; ++i)
    if (!is_fin(r[i])) return INVALID_EVALUATION;
  return p->sink->accumulate(rows, r, nb, cols, widths, jac, rs, cs);
}
OR_API int or_lm_cb(void* schur, void* prob, const OptimizeOptions* opt, const LmOptions* lo, Report* rep,
                    LmStats* st) {
  return lm_optimize(*(Linear*)schur, *(CallbackProblem*)prob, *opt, *lo, rep, st, nullptr, nullptr);
}
OR_API int or_gn_cb(void* schur, void* prob, const OptimizeOptions* opt, Report* rep) {
  return gn_optimize(*(Linear*)schur, *(CallbackProblem*)prob, *opt, rep);
}

// ---- Dense backends (src/normal.rs, src/dense_schur.rs, src/qr.rs); the
// generic or_schur_* entry points above drive them.
OR_API void* or_dense_normal_create(void) { return (void*)(Linear*)new DenseNormal(); }
OR_API void* or_dense_schur_create(size_t retained, const size_t* widths, size_t nwidths) {
  DenseSchur* s = new DenseSchur();
  s->retained = retained;
  s->widths.assign(widths, widths + nwidths);
  return (void*)(Linear*)s;
}
OR_API void* or_dense_qr_create(double relative_rank_tolerance) {
  DenseQr* q = new DenseQr();
  q->relative_rank_tolerance = relative_rank_tolerance;
  return (void*)(Linear*)q;
}
OR_API void or_dense_qr_set_tolerance(void* h, double tol) {
  static_cast<DenseQr*>(LIN(h))->relative_rank_tolerance = tol;
}
// Dense normal state: lower triangle of J^T J (n*n column-major) and -J^T r.
OR_API void or_dense_normal_state(void* h, double* normal, double* rhs) {
  DenseNormal* d = static_cast<DenseNormal*>(LIN(h));
  if (normal) std::copy(d->normal.begin(), d->normal.end(), normal);
  if (rhs) std::copy(d->rhs.begin(), d->rhs.end(), rhs);
}
OR_API int or_dense_normal_information(void* h, double tol) {
  return static_cast<DenseNormal*>(LIN(h))->information_factor(tol);
}
// Selected covariance of the backend's current model (covariance.rs:263-270):
// kind 0 = Schur/LSMR/DenseQr (LinearizedModel::covariance), 1 = DenseNormal,
// 2 = DenseSchur (retained selections). columns are model coordinates.
OR_API int or_backend_covariance(void* h, int kind, const size_t* columns, size_t k, double tol, double* out) {
  if (!(tol >= 0 && tol < 1)) return INVALID_RANK_TOLERANCE;
  std::vector<size_t> cols(columns, columns + k);
  std::vector<double> res;
  int st;
  Linear* b = LIN(h);
  if (kind == 1) {
    DenseNormal* d = static_cast<DenseNormal*>(b);
    st = d->information_factor(tol);
    if (!st) st = covariance_from_factor(d->normal.data(), d->n, nullptr, cols, res);
  } else if (kind == 2) {
    st = static_cast<DenseSchur*>(b)->covariance(cols, tol, res);
  } else {
    const Model* m = nullptr;
    if (auto* s = dynamic_cast<Schur*>(b)) m = &s->model;
    if (auto* l = dynamic_cast<Lsmr*>(b)) m = &l->model;
    if (auto* q = dynamic_cast<DenseQr*>(b)) m = &q->model;
    if (!m) return INVALID_OPTIONS;
    DenseNormal normal;
    st = model_covariance(*m, normal, cols, tol, res);
  }
  if (!st) std::copy(res.begin(), res.end(), out);
  return st;
}

// ---- Square-root elimination (src/marginalization.rs:458-513).
OR_API int or_eliminate(size_t m, size_t n, const double* rowmajor, size_t removed, double tol, double* a,
                        double* b, double* constant, size_t* rank, size_t* rows) {
  EliminationResult r;
  int st = eliminate(m, n, rowmajor, removed, tol, r);
  if (st) return st;
  std::copy(r.a.begin(), r.a.end(), a);
  std::copy(r.b.begin(), r.b.end(), b);
  *constant = r.constant;
  *rank = r.rank;
  *rows = r.rows;
  return OK;
}

// ---- SE(3) (examples/slam/geometry.rs); poses are [qw qx qy qz tx ty tz].
static Pose3 P7(const double* p) {
  Pose3 o;
  std::copy(p, p + 4, o.q);
  std::copy(p + 4, p + 7, o.t);
  return o;
}
static void W7(const Pose3& p, double* o) {
  std::copy(p.q, p.q + 4, o);
  std::copy(p.t, p.t + 3, o + 4);
}
OR_API void or_pose_exp(const double* d, double* out) { W7(pose_exp(d), out); }
OR_API void or_pose_log(const double* p, double* out) { pose_log(P7(p), out); }
OR_API void or_pose_compose(const double* a, const double* b, double* out) { W7(compose(P7(a), P7(b)), out); }
OR_API void or_pose_inverse(const double* a, double* out) { W7(inverse(P7(a)), out); }
OR_API void or_pose_adjoint(const double* p, double* out) { pose_adjoint(P7(p), out); }
OR_API void or_pose_right_jacobian(const double* d, double* out) { pose_right_jacobian(d, out); }
OR_API int or_pose_log_jacobian(const double* d, double* out) { return log_jacobian(d, out); }

// ---- Pose-graph windows: LM over DenseSchur(6n, []) then marginalization of
// the oldest `removed` poses. poses[7n] in/out; rel_ij[2*nrel]; rel_z[7*nrel].
static int window_solve(PoseWindow& w, size_t n, double* poses, const OptimizeOptions* opt, const LmOptions* lo,
                        size_t removed, Report* rep, LmStats* st, double* prior_a, double* prior_b,
                        double* prior_constant, size_t* prior_rows, uint32_t* separator, size_t* nseparator,
                        size_t* rank);
static void window_factors(PoseWindow& w, size_t n, const double* poses, size_t nrel, const uint32_t* rel_ij,
                           const double* rel_z) {
  w.x.resize(n);
  for (size_t k = 0; k < n; ++k) w.x[k] = P7(poses + 7 * k);
  w.rel.resize(nrel);
  for (size_t k = 0; k < nrel; ++k) {
    w.rel[k].i = rel_ij[2 * k];
    w.rel[k].j = rel_ij[2 * k + 1];
    w.rel[k].z = P7(rel_z + 7 * k);
  }
}
static void window_prior(PoseWindow& w, size_t s, size_t m, const double* A, const double* b, const double* refs) {
  w.prior.s = s;
  w.prior.m = m;
  w.prior.A.assign(A, A + m * 6 * s);
  w.prior.b.assign(b, b + m);
  w.prior.ref.resize(s);
  for (size_t k = 0; k < s; ++k) w.prior.ref[k] = P7(refs + 7 * k);
}
// A window with a prior on its first s poses (m rows, A m x 6s column-major,
// b, s reference poses) in place of the anchor.
OR_API int or_window_solve_prior(size_t n, double* poses, size_t s, size_t m, const double* A, const double* b,
                                 const double* refs, size_t nrel, const uint32_t* rel_ij, const double* rel_z,
                                 const OptimizeOptions* opt, const LmOptions* lo, size_t removed, Report* rep,
                                 LmStats* st, double* prior_a, double* prior_b, double* prior_constant,
                                 size_t* prior_rows, uint32_t* separator, size_t* nseparator, size_t* rank) {
  if (s == 0 || s > n || m == 0) return INVALID_OPTIONS;
  PoseWindow w;
  window_factors(w, n, poses, nrel, rel_ij, rel_z);
  window_prior(w, s, m, A, b, refs);
  return window_solve(w, n, poses, opt, lo, removed, rep, st, prior_a, prior_b, prior_constant, prior_rows, separator,
                      nseparator, rank);
}
OR_API int or_window_cost_prior(size_t n, const double* poses, size_t s, size_t m, const double* A, const double* b,
                                const double* refs, size_t nrel, const uint32_t* rel_ij, const double* rel_z,
                                double* out) {
  if (s == 0 || s > n || m == 0) return INVALID_OPTIONS;
  PoseWindow w;
  window_factors(w, n, poses, nrel, rel_ij, rel_z);
  window_prior(w, s, m, A, b, refs);
  return w.cost(false, out);
}
OR_API int or_window_solve(size_t n, double* poses, const double* prior, size_t nrel, const uint32_t* rel_ij,
                           const double* rel_z, const OptimizeOptions* opt, const LmOptions* lo, size_t removed,
                           Report* rep, LmStats* st, double* prior_a, double* prior_b, double* prior_constant,
                           size_t* prior_rows, uint32_t* separator, size_t* nseparator, size_t* rank) {
  PoseWindow w;
  window_factors(w, n, poses, nrel, rel_ij, rel_z);
  w.prior.anchor(P7(prior));
  return window_solve(w, n, poses, opt, lo, removed, rep, st, prior_a, prior_b, prior_constant, prior_rows, separator,
                      nseparator, rank);
}
static int window_solve(PoseWindow& w, size_t n, double* poses, const OptimizeOptions* opt, const LmOptions* lo,
                        size_t removed, Report* rep, LmStats* st, double* prior_a, double* prior_b,
                        double* prior_constant, size_t* prior_rows, uint32_t* separator, size_t* nseparator,
                        size_t* rank) {
  DenseSchur solver;
  solver.retained = 6 * n;
  int code = lm_optimize(solver, w, *opt, *lo, rep, st, nullptr, nullptr);
  for (size_t k = 0; k < n; ++k) W7(w.x[k], poses + 7 * k);
  if (code != OK && code != NO_PROGRESS && code != NO_CONVERGENCE) return code;
  if (removed) {
    WindowPrior wp;
    int s = marginalize_window(w, std::min(removed, n), wp);
    if (s) return s;
    std::copy(wp.elim.a.begin(), wp.elim.a.end(), prior_a);
    std::copy(wp.elim.b.begin(), wp.elim.b.end(), prior_b);
    *prior_constant = wp.elim.constant;
    *prior_rows = wp.elim.rows;
    *rank = wp.elim.rank;
    std::copy(wp.separator.begin(), wp.separator.end(), separator);
    *nseparator = wp.separator.size();
  }
  return code;
}
// Window cost at the given poses (PosePrior + relative factors).
OR_API int or_window_cost(size_t n, const double* poses, const double* prior, size_t nrel, const uint32_t* rel_ij,
                          const double* rel_z, double* out) {
  PoseWindow w;
  window_factors(w, n, poses, nrel, rel_ij, rel_z);
  w.prior.anchor(P7(prior));
  return w.cost(false, out);
}
