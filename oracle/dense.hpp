// ORACLE — test infrastructure only (included by oracle.cpp).
//
// Dense backends and dense kernels of fagra, restated:
//   src/normal.rs:65-392          DenseNormalCholesky (+ information_factor)
//   src/dense_schur.rs:92-462     DenseSchur
//   src/qr.rs:65-242              DenseQr
//   src/marginalization.rs:404-514 Elimination::qr / reduce (square-root elimination)
//   src/covariance.rs:225-255     SelectedCovariance::compute_factor
// faer's blocked Cholesky, triangular solves and column-pivoted Householder QR
// (faer 0.24.4, not part of the fagra tree) are restated as the textbook
// column algorithms: same factorizations, different summation order. The
// pivoted QR picks the remaining column of largest norm (norms recomputed, first
// maximum on ties) and uses LAPACK-style reflectors H = I - tau v v^T with
// R_kk = -sign(a_kk) ||a_k||; reflector signs may differ from faer's, which
// flips rows of R but leaves every least-squares objective unchanged.

// In-place lower Cholesky of the lower triangle of a column-major n x n matrix
// with leading dimension lda. False on a non-positive or nonfinite pivot.
bool chol_lower(double* a, size_t n, size_t lda) {
  for (size_t j = 0; j < n; ++j) {
    double d = a[j * lda + j];
    for (size_t k = 0; k < j; ++k) d -= a[k * lda + j] * a[k * lda + j];
    if (!(d > 0) || !is_fin(d)) return false;
    d = std::sqrt(d);
    a[j * lda + j] = d;
    for (size_t i = j + 1; i < n; ++i) {
      double s = a[j * lda + i];
      for (size_t k = 0; k < j; ++k) s -= a[k * lda + i] * a[k * lda + j];
      a[j * lda + i] = s / d;
    }
  }
  return true;
}
// x <- L^-1 x and x <- L^-T x for the lower factor L (column-major, lda).
void lsolve(const double* l, size_t n, size_t lda, double* x) {
  for (size_t i = 0; i < n; ++i) {
    double s = x[i];
    for (size_t k = 0; k < i; ++k) s -= l[k * lda + i] * x[k];
    x[i] = s / l[i * lda + i];
  }
}
void ltsolve(const double* l, size_t n, size_t lda, double* x) {
  for (size_t ii = n; ii-- > 0;) {
    double s = x[ii];
    for (size_t k = ii + 1; k < n; ++k) s -= l[ii * lda + k] * x[k];
    x[ii] = s / l[ii * lda + ii];
  }
}

// Column-pivoted Householder QR of rows [r0, m) x columns [c0, c0+w) of the
// column-major m x ncols matrix a; columns right of the block are transformed
// with it. perm[k] = original block column now at position k.
void qr_pivoted(double* a, size_t m, size_t lda, size_t ncols, size_t r0, size_t c0, size_t w,
                std::vector<size_t>& perm) {
  perm.resize(w);
  for (size_t k = 0; k < w; ++k) perm[k] = k;
  const size_t h = m - r0;
  const size_t steps = std::min(h, w);
  auto col = [&](size_t j) { return a + (c0 + j) * lda + r0; };
  for (size_t k = 0; k < steps; ++k) {
    size_t best = k;
    double bn = -1;
    for (size_t j = k; j < w; ++j) {
      double s = 0;
      const double* cj = col(j);
      for (size_t i = k; i < h; ++i) s += cj[i] * cj[i];
      if (s > bn) {
        bn = s;
        best = j;
      }
    }
    if (best != k) {
      double* x = col(k);
      double* y = col(best);
      for (size_t i = 0; i < h; ++i) std::swap(x[i], y[i]);
      std::swap(perm[k], perm[best]);
    }
    double* v = col(k);
    const double alpha = v[k];
    double xn = 0;
    for (size_t i = k + 1; i < h; ++i) xn = std::hypot(xn, v[i]);
    if (xn == 0) continue;  // already triangular in this column: H = I
    const double beta = -std::copysign(std::hypot(alpha, xn), alpha);
    const double tau = (beta - alpha) / beta;
    const double scale = 1.0 / (alpha - beta);
    for (size_t i = k + 1; i < h; ++i) v[i] *= scale;
    v[k] = beta;
    // Apply H = I - tau [1; v] [1; v]^T to the block's remaining columns and
    // every column to its right.
    for (size_t j = c0 + k + 1; j < ncols; ++j) {
      double* cj = a + j * lda + r0;
      double s = cj[k];
      for (size_t i = k + 1; i < h; ++i) s += v[i] * cj[i];
      s *= tau;
      cj[k] -= s;
      for (size_t i = k + 1; i < h; ++i) cj[i] -= s * v[i];
    }
  }
}

// --------------------------------------------------- DenseNormalCholesky
struct DenseNormal : Linear {
  size_t n = 0;
  std::vector<double> normal, rhs, diagonal, damped, scales;
  bool factorized = false, damping_ready = false;

  double& N(size_t r, size_t c) { return normal[c * n + r]; }
  int prepare(size_t dim) override {  // normal.rs:65-89
    damping_ready = false;
    n = dim;
    normal.assign(n * n, 0.);
    rhs.assign(n, 0.);
    diagonal.assign(n, 0.);
    work.step.assign(n, 0.);
    factorized = false;
    solves = iterations = 0;
    return OK;
  }
  void clear() override {  // :91-103
    damping_ready = false;
    factorized = false;
    for (size_t c = 0; c < n; ++c)
      for (size_t r = c; r < n; ++r) N(r, c) = 0.;
    std::fill(rhs.begin(), rhs.end(), 0.);
  }
  // accumulate_small / accumulate_matmul (:243-334): lower triangle of J^T J and rhs -= J^T r.
  int accumulate(size_t nrows, const double* r, size_t nb, const size_t* cols, const size_t* widths,
                 const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) override {
    damping_ready = false;
    for (size_t b = 0; b < nb; ++b)
      if (cols[b] + widths[b] < cols[b] || cols[b] + widths[b] > n) return DIMENSION_MISMATCH;
    auto J = [&](size_t b, size_t k, size_t c) { return jac[b][(ptrdiff_t)k * rs[b] + (ptrdiff_t)c * cs[b]]; };
    for (size_t i = 0; i < nb; ++i) {
      const size_t off = cols[i], w = widths[i];
      for (size_t c = 0; c < w; ++c) {
        double g = 0;
        for (size_t k = 0; k < nrows; ++k) g += J(i, k, c) * r[k];
        rhs[off + c] -= g;
        for (size_t rr = c; rr < w; ++rr) {
          double p = 0;
          for (size_t k = 0; k < nrows; ++k) p += J(i, k, rr) * J(i, k, c);
          N(off + rr, off + c) += p;
        }
      }
      for (size_t o = 0; o < i; ++o) {
        // Lower block first: (row offset, col offset, lhs block, rhs block).
        size_t ro, co, lb, rb;
        if (off > cols[o]) {
          ro = off; co = cols[o]; lb = i; rb = o;
        } else {
          ro = cols[o]; co = off; lb = o; rb = i;
        }
        for (size_t c = 0; c < widths[rb]; ++c)
          for (size_t rr = 0; rr < widths[lb]; ++rr) {
            double p = 0;
            for (size_t k = 0; k < nrows; ++k) p += J(lb, k, rr) * J(rb, k, c);
            N(ro + rr, co + c) += p;
          }
      }
    }
    return OK;
  }
  int gradient_norm(double* out) const override { return norm_inf(rhs.data(), n, out); }
  int factorize() {  // :339-365
    damping_ready = false;
    if (factorized) return OK;
    if (n == 0) {
      factorized = true;
      return OK;
    }
    for (size_t c = 0; c < n; ++c) {
      diagonal[c] = N(c, c);
      for (size_t r = c; r < n; ++r)
        if (!is_fin(N(r, c))) return INVALID_EVALUATION;
    }
    if (!chol_lower(normal.data(), n, n)) return LINEAR_SOLVE_FAILED;
    factorized = true;
    return OK;
  }
  int solve() override {  // :137-152
    damping_ready = false;
    if (n == 0) {
      work.step.clear();
      return OK;
    }
    int s = factorize();
    if (s) return s;
    lsolve(normal.data(), n, n, rhs.data());
    ltsolve(normal.data(), n, n, rhs.data());
    work.step = rhs;
    return OK;
  }
  int prepare_damping(double floor) override {  // :154-177
    damping_ready = false;
    if (factorized || !is_fin(floor) || floor <= 0) return INVALID_OPTIONS;
    double tmp;
    if (norm_inf(rhs.data(), n, &tmp)) return INVALID_EVALUATION;
    damped.assign(n * n, 0.);
    scales.assign(n, 0.);
    for (size_t c = 0; c < n; ++c) {
      for (size_t r = c; r < n; ++r)
        if (!is_fin(N(r, c))) return INVALID_EVALUATION;
      if (N(c, c) < 0) return INVALID_EVALUATION;
      scales[c] = std::max(std::sqrt(N(c, c)), floor);
    }
    damping_ready = true;
    return OK;
  }
  int solve_damped(double lambda, double* predicted) override {  // :179-230
    if (!damping_ready || !is_fin(lambda) || lambda < 0) return INVALID_OPTIONS;
    ++solves;
    for (size_t c = 0; c < n; ++c) {
      for (size_t r = c; r < n; ++r) damped[c * n + r] = N(r, c);
      double d = std::sqrt(lambda) * scales[c];
      damped[c * n + c] += d * d;
      if (!is_fin(damped[c * n + c])) return LINEAR_SOLVE_FAILED;
    }
    work.step = rhs;
    if (n > 0) {
      if (!chol_lower(damped.data(), n, n)) return LINEAR_SOLVE_FAILED;
      lsolve(damped.data(), n, n, work.step.data());
      ltsolve(damped.data(), n, n, work.step.data());
    }
    double tmp;
    if (norm_inf(work.step.data(), n, &tmp)) return LINEAR_SOLVE_FAILED;
    double p = 0;
    for (size_t c = 0; c < n; ++c) {
      double d = work.step[c];
      p += rhs[c] * d - 0.5 * d * N(c, c) * d;
      for (size_t r = c + 1; r < n; ++r) p -= d * N(r, c) * work.step[r];
    }
    if (!is_fin(p)) return LINEAR_SOLVE_FAILED;
    *predicted = p;
    return OK;
  }
  // information_factor (:367-392): the Cholesky factor with a pivot rank screen.
  int information_factor(double tol) {
    int s = factorize();
    if (s == LINEAR_SOLVE_FAILED) return SINGULAR_INFORMATION;
    if (s) return INVALID_INFORMATION;
    for (size_t i = 0; i < n; ++i) {
      double pivot = N(i, i), d = diagonal[i];
      if (!is_fin(pivot) || !is_fin(d)) return INVALID_INFORMATION;
      double ratio = pivot / std::sqrt(d);
      if (d <= 0 || pivot <= 0 || ratio * ratio <= tol) return SINGULAR_INFORMATION;
    }
    return OK;
  }
};

// SelectedCovariance::compute_factor (covariance.rs:225-255): with L the lower
// factor of (scaled) information H = D Hs D, Sigma_sel = Y^T Y for
// L Y = D^-1 E_sel. `scales` empty = original coordinates.
int covariance_from_factor(const double* L, size_t n, const double* scales, const std::vector<size_t>& columns,
                           std::vector<double>& out) {
  for (size_t c : columns)
    if (c >= n) return UNSUPPORTED_STRUCTURE;
  const size_t k = columns.size();
  std::vector<double> Y(n * k, 0.);
  for (size_t j = 0; j < k; ++j) Y[j * n + columns[j]] = 1.0 / (scales ? scales[columns[j]] : 1.0);
  for (size_t j = 0; j < k; ++j) lsolve(L, n, n, &Y[j * n]);
  out.assign(k * k, 0.);
  for (size_t b = 0; b < k; ++b)
    for (size_t a = 0; a < k; ++a) {
      double s = 0;
      for (size_t i = 0; i < n; ++i) s += Y[a * n + i] * Y[b * n + i];
      out[b * k + a] = s;
    }
  for (double v : out)
    if (!is_fin(v)) return INVALID_INFORMATION;
  return OK;
}

// LinearizedModel::covariance (linear_model.rs:122-167): replay the cached
// Jacobian into a DenseNormalCholesky, one call per row group.
int model_covariance(const Model& m, DenseNormal& normal, const std::vector<size_t>& columns, double tol,
                     std::vector<double>& out) {
  normal.prepare(m.cols);
  normal.clear();
  size_t start = 0;
  while (start < m.blocks.size()) {
    const Block& first = m.blocks[start];
    if (first.rows == 0) {
      ++start;
      continue;
    }
    size_t end = start + 1;
    while (end < m.blocks.size() && m.blocks[end].row == first.row && m.blocks[end].rows == first.rows) ++end;
    std::vector<size_t> cols, widths;
    std::vector<const double*> ptrs;
    std::vector<ptrdiff_t> rs, cs;
    for (size_t b = start; b < end; ++b) {
      cols.push_back(m.blocks[b].col);
      widths.push_back(m.blocks[b].cols);
      ptrs.push_back(&m.values[m.blocks[b].start]);
      rs.push_back(1);
      cs.push_back((ptrdiff_t)m.blocks[b].rows);
    }
    int s = normal.accumulate(first.rows, &m.negative_residual[first.row], end - start, cols.data(), widths.data(),
                              ptrs.data(), rs.data(), cs.data());
    if (s) return s;
    start = end;
  }
  int s = normal.information_factor(tol);
  if (s) return s;
  return covariance_from_factor(normal.normal.data(), normal.n, nullptr, columns, out);
}

// ------------------------------------------------------------- DenseSchur
struct DenseSchur : Linear {
  size_t retained;
  std::vector<size_t> widths;
  std::vector<std::pair<size_t, size_t>> landmarks;  // [begin, end)
  std::vector<size_t> owners, starts;
  std::vector<double> gram, factors, retained_gram, cross, solved, reduced, rhs;
  size_t elim = 0;
  Model model;
  bool ready = false;

  double& RG(size_t r, size_t c) { return retained_gram[c * retained + r]; }
  double& RD(size_t r, size_t c) { return reduced[c * retained + r]; }
  double& CR(size_t l, size_t c) { return cross[c * elim + l]; }
  double& SV(size_t l, size_t c) { return solved[c * elim + l]; }

  int prepare(size_t dim) override {  // dense_schur.rs:211-271
    ready = false;
    solves = iterations = 0;
    if (dim < retained) return INVALID_OPTIONS;
    elim = dim - retained;
    landmarks.clear();
    starts.clear();
    size_t offset = retained, size = 0;
    for (size_t w : widths) {
      size_t end = offset + w;
      if (w == 0 || end > dim) return INVALID_OPTIONS;
      landmarks.push_back({offset, end});
      starts.push_back(size);
      size += w * w;
      offset = end;
    }
    if (offset != dim) return INVALID_OPTIONS;
    owners.assign(elim, 0);
    for (size_t id = 0; id < landmarks.size(); ++id)
      for (size_t c = landmarks[id].first; c < landmarks[id].second; ++c) owners[c - retained] = id;
    gram.assign(size, 0.);
    factors.assign(size, 0.);
    retained_gram.assign(retained * retained, 0.);
    reduced.assign(retained * retained, 0.);
    cross.assign(elim * retained, 0.);
    solved.assign(elim * (retained + 1), 0.);
    rhs.assign(retained, 0.);
    model.prepare(dim);
    work.step.assign(dim, 0.);
    return OK;
  }
  void clear() override {  // :273-276
    ready = false;
    model.clear();
  }
  int accumulate(size_t nrows, const double* r, size_t nb, const size_t* cols, const size_t* w,
                 const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) override {  // :278-306
    ready = false;
    bool has_landmark = false;
    for (size_t i = 0; i < nb; ++i) {
      size_t col = cols[i], end = col + w[i];
      if (end < col || end > model.cols) return DIMENSION_MISMATCH;
      if (w[i] == 0) continue;
      if (col >= retained) {
        size_t id = owners[col - retained];
        if (landmarks[id].first != col || landmarks[id].second != end || has_landmark) return UNSUPPORTED_STRUCTURE;
        has_landmark = true;
      } else if (end > retained) {
        return UNSUPPORTED_STRUCTURE;
      }
      for (size_t o = 0; o < i; ++o)
        if (col < cols[o] + w[o] && cols[o] < end) return DIMENSION_MISMATCH;
    }
    return model.accumulate(nrows, r, nb, cols, w, jac, rs, cs);
  }
  int gradient_norm(double* out) const override { return norm_inf(model.gradient.data(), model.cols, out); }
  void assemble() {  // :92-137
    std::fill(gram.begin(), gram.end(), 0.);
    std::fill(retained_gram.begin(), retained_gram.end(), 0.);
    std::fill(cross.begin(), cross.end(), 0.);
    const auto& B = model.blocks;
    for (size_t index = 0; index < B.size(); ++index) {
      const Block& left = B[index];
      if (left.rows == 0) continue;
      for (size_t other = index + 1; other-- > 0;) {
        const Block& right = B[other];
        if (right.row != left.row || right.rows != left.rows) break;
        for (size_t col = 0; col < right.cols; ++col)
          for (size_t row = 0; row < left.cols; ++row) {
            if (other == index && row < col) continue;
            size_t a = left.col + row, b = right.col + col;
            double value = 0;
            for (size_t k = 0; k < left.rows; ++k)
              value += (model.values[left.start + row * left.rows + k] / model.scales[a]) *
                       (model.values[right.start + col * right.rows + k] / model.scales[b]);
            if (a < retained && b < retained) {
              RG(std::max(a, b), std::min(a, b)) += value;
            } else if (a >= retained && b >= retained) {
              size_t id = owners[a - retained];
              size_t lo = landmarks[id].first, len = landmarks[id].second - lo;
              size_t aa = a - lo, bb = b - lo;
              gram[starts[id] + std::min(aa, bb) * len + std::max(aa, bb)] += value;
            } else {
              size_t lm = a >= retained ? a : b, rt = a >= retained ? b : a;
              CR(lm - retained, rt) += value;
            }
          }
      }
    }
  }
  static int factorize_dense(double* m, size_t n, size_t lda) {  // :415-444
    for (size_t c = 0; c < n; ++c)
      for (size_t r = c; r < n; ++r)
        if (!is_fin(m[c * lda + r])) return INVALID_EVALUATION;
    if (n == 0) return OK;
    return chol_lower(m, n, lda) ? OK : LINEAR_SOLVE_FAILED;
  }
  static int check_rank(const double* L, size_t n, size_t lda, const std::vector<double>& diag, double tol) {
    for (size_t i = 0; i < n; ++i) {  // :452-460
      double pivot = L[i * lda + i], d = diag[i];
      if (!is_fin(pivot) || !is_fin(d)) return INVALID_INFORMATION;
      double q = pivot / std::sqrt(d);
      if (d <= 0 || pivot <= 0 || q * q <= tol) return SINGULAR_INFORMATION;
    }
    return OK;
  }
  int solve_landmarks(double lambda, const double* tol) {  // :139-172
    const size_t r = retained;
    factors = gram;
    for (size_t id = 0; id < landmarks.size(); ++id) {
      size_t w = landmarks[id].second - landmarks[id].first, st = starts[id];
      double* f = &factors[st];
      for (size_t i = 0; i < w; ++i) f[i * w + i] += lambda;
      int s = factorize_dense(f, w, w);
      if (s) return s;
      if (tol) {
        std::vector<double> d(w);
        for (size_t i = 0; i < w; ++i) d[i] = gram[st + i * w + i];
        if ((s = check_rank(f, w, w, d, *tol))) return s;
      }
      size_t off = landmarks[id].first - r;
      for (size_t row = 0; row < w; ++row) {
        for (size_t c = 0; c < r; ++c) SV(off + row, c) = CR(off + row, c);
        size_t gi = landmarks[id].first + row;
        SV(off + row, r) = -model.gradient[gi] / model.scales[gi];
      }
      std::vector<double> tmp(w);
      for (size_t c = 0; c <= r; ++c) {
        for (size_t row = 0; row < w; ++row) tmp[row] = SV(off + row, c);
        lsolve(f, w, w, tmp.data());
        ltsolve(f, w, w, tmp.data());
        for (size_t row = 0; row < w; ++row) SV(off + row, c) = tmp[row];
      }
    }
    return OK;
  }
  int reduce(double lambda, const double* tol) {  // :174-209
    int s = solve_landmarks(lambda, tol);
    if (s) return s;
    const size_t r = retained;
    for (size_t c = 0; c < r; ++c) {
      rhs[c] = -model.gradient[c] / model.scales[c];
      for (size_t row = c; row < r; ++row) RD(row, c) = RG(row, c);
      RD(c, c) += lambda;
    }
    for (size_t c = 0; c < r; ++c)
      for (size_t row = c; row < r; ++row) {
        double p = 0;
        for (size_t l = 0; l < elim; ++l) p += CR(l, row) * SV(l, c);
        RD(row, c) -= p;
      }
    for (size_t c = 0; c < r; ++c) {
      double p = 0;
      for (size_t l = 0; l < elim; ++l) p += CR(l, c) * SV(l, r);
      rhs[c] -= p;
    }
    if ((s = factorize_dense(reduced.data(), r, r))) return s;
    if (tol) {
      std::vector<double> d(r);
      for (size_t i = 0; i < r; ++i) d[i] = RG(i, i);
      if ((s = check_rank(reduced.data(), r, r, d, *tol))) return s;
    }
    return OK;
  }
  int solve() override {  // :312-315
    int s = prepare_damping(1e-6);
    if (s) return s;
    double p;
    return solve_damped(0., &p);
  }
  int prepare_damping(double floor) override {  // :317-326
    ready = false;
    int s = model.prepare_scales(floor);
    if (s) return s;
    double tmp;
    if (norm_inf(model.gradient.data(), model.cols, &tmp)) return INVALID_EVALUATION;
    work.prepare_verification(model.rows, model.cols);
    assemble();
    ready = true;
    return OK;
  }
  int solve_damped(double lambda, double* predicted) override {  // :328-356
    if (!ready || !is_fin(lambda) || lambda < 0) return INVALID_OPTIONS;
    ++solves;
    int s = reduce(lambda, nullptr);
    if (s) return s;
    const size_t r = retained;
    lsolve(reduced.data(), r, r, rhs.data());
    ltsolve(reduced.data(), r, r, rhs.data());
    for (size_t i = 0; i < r; ++i) work.step[i] = rhs[i] / model.scales[i];
    for (auto& lm : landmarks)
      for (size_t i = lm.first; i < lm.second; ++i) {
        size_t row = i - r;
        double v = SV(row, r);
        for (size_t c = 0; c < r; ++c) v -= SV(row, c) * rhs[c];
        work.step[i] = v / model.scales[i];
      }
    Verification v = verify_step(model, work, lambda);
    if (!v.finite_step || !is_fin(v.predicted)) return LINEAR_SOLVE_FAILED;
    *predicted = v.predicted;
    return OK;
  }
  // CovarianceBackend::covariance (:359-377), retained selections only.
  int covariance(const std::vector<size_t>& columns, double tol, std::vector<double>& out) {
    for (size_t c : columns)
      if (c >= retained) return UNSUPPORTED_STRUCTURE;
    int s = prepare_damping(1e-6);
    if (!s) s = reduce(0., &tol);
    if (s == LINEAR_SOLVE_FAILED) return SINGULAR_INFORMATION;
    if (s == INVALID_EVALUATION) return INVALID_INFORMATION;
    if (s) return s;
    return covariance_from_factor(reduced.data(), retained, model.scales.data(), columns, out);
  }
};

// ------------------------------------------------------------------ DenseQr
struct DenseQr : Linear {
  double relative_rank_tolerance = 64. * std::numeric_limits<double>::epsilon();
  Model model;
  std::vector<double> mat, product;
  std::vector<size_t> perm;
  bool damping_ready = false;

  int validate() const {
    return (relative_rank_tolerance >= 0 && relative_rank_tolerance < 1) ? OK : INVALID_OPTIONS;
  }
  int factor_solve(bool damped, double lambda) {  // qr.rs:65-176
    int s = validate();
    if (s) return s;
    const size_t n = model.cols;
    if (n == 0) return OK;
    const size_t m = model.rows, height = m + (damped ? n : 0), width = n + 1;
    if (height < n) return LINEAR_SOLVE_FAILED;
    mat.assign(height * width, 0.);
    for (const Block& b : model.blocks)
      for (size_t c = 0; c < b.cols; ++c) {
        double sc = damped ? model.scales[b.col + c] : 1.0;
        for (size_t r = 0; r < b.rows; ++r)
          mat[(b.col + c) * height + b.row + r] = model.values[b.start + c * b.rows + r] / sc;
      }
    for (size_t r = 0; r < m; ++r) mat[n * height + r] = model.negative_residual[r];
    if (damped)
      for (size_t c = 0; c < n; ++c) mat[c * height + m + c] = std::sqrt(lambda);
    double largest = 0;
    for (size_t c = 0; c < width; ++c)
      for (size_t r = 0; r < height; ++r) {
        double v = mat[c * height + r];
        if (!is_fin(v)) return LINEAR_SOLVE_FAILED;
        if (c < n) largest = std::max(largest, std::fabs(v));
      }
    if (largest == 0) return LINEAR_SOLVE_FAILED;
    qr_pivoted(mat.data(), height, height, width, 0, 0, n, perm);
    largest = 0;
    for (size_t c = 0; c < n; ++c) {
      double p = std::fabs(mat[c * height + c]);
      if (!is_fin(p)) return LINEAR_SOLVE_FAILED;
      largest = std::max(largest, p);
    }
    for (size_t c = n; c-- > 0;) {
      double pivot = mat[c * height + c];
      if (std::fabs(pivot) <= relative_rank_tolerance * largest) return LINEAR_SOLVE_FAILED;
      double v = mat[n * height + c];
      for (size_t j = c + 1; j < n; ++j) v -= mat[j * height + c] * work.step[perm[j]];
      work.step[perm[c]] = v / pivot;
    }
    if (damped)
      for (size_t j = 0; j < n; ++j) work.step[j] /= model.scales[j];
    double tmp;
    if (norm_inf(work.step.data(), n, &tmp)) return LINEAR_SOLVE_FAILED;
    return OK;
  }
  int prepare(size_t dim) override {  // :180-186
    damping_ready = false;
    solves = iterations = 0;
    int s = validate();
    if (s) return s;
    model.prepare(dim);
    work.step.assign(dim, 0.);
    return OK;
  }
  void clear() override {
    damping_ready = false;
    model.clear();
  }
  int accumulate(size_t nrows, const double* r, size_t nb, const size_t* cols, const size_t* w,
                 const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) override {
    damping_ready = false;
    for (size_t i = 0; i < nb; ++i)
      if (cols[i] + w[i] < cols[i] || cols[i] + w[i] > model.cols) return DIMENSION_MISMATCH;
    return model.accumulate(nrows, r, nb, cols, w, jac, rs, cs);
  }
  int gradient_norm(double* out) const override { return norm_inf(model.gradient.data(), model.cols, out); }
  int solve() override { return factor_solve(false, 0.); }
  int prepare_damping(double floor) override {
    damping_ready = false;
    int s = model.prepare_scales(floor);
    if (s) return s;
    product.assign(model.rows, 0.);
    damping_ready = true;
    return OK;
  }
  int solve_damped(double lambda, double* predicted) override {  // :220-236
    if (!damping_ready || !is_fin(lambda) || lambda < 0) return INVALID_OPTIONS;
    ++solves;
    int s = factor_solve(true, lambda);
    if (s) return s;
    double p = model.predicted_reduction(work.step.data(), product.data());
    if (!is_fin(p)) return LINEAR_SOLVE_FAILED;
    *predicted = p;
    return OK;
  }
};

// ----------------------------------------------- square-root elimination
// Elimination::reduce (marginalization.rs:458-513) on the row-major m x (n+1)
// system [J | r] whose first `removed` columns are eliminated. Outputs the
// prior rows A (rows x separator, column-major) and b, the constant term and
// the eliminated rank. tol < 0 selects eps * max(m, removed, 1).
struct EliminationResult {
  std::vector<double> a, b;
  double constant = 0;
  size_t rank = 0, rows = 0;
};
int eliminate(size_t m, size_t n, const double* rowmajor, size_t removed, double tol, EliminationResult& out) {
  const size_t width = n + 1;
  std::vector<double> M(m * width);
  for (size_t r = 0; r < m; ++r)
    for (size_t c = 0; c < width; ++c) M[c * m + r] = rowmajor[r * width + c];
  std::vector<size_t> perm;
  auto block_qr = [&](size_t row, size_t column, size_t w) {  // Elimination::qr, :412-455
    perm.resize(w);
    for (size_t i = 0; i < w; ++i) perm[i] = i;
    if (m - row == 0 || w == 0) return;
    bool zero = true;
    for (size_t j = column; j < column + w && zero; ++j)
      for (size_t i = row; i < m; ++i)
        if (M[j * m + i] != 0) {
          zero = false;
          break;
        }
    if (zero) return;
    qr_pivoted(M.data(), m, m, width, row, column, w, perm);
  };
  block_qr(0, 0, removed);
  if (tol < 0) tol = std::numeric_limits<double>::epsilon() * (double)std::max<size_t>(std::max(m, removed), 1);
  const double scale = (m > 0 && removed > 0) ? std::fabs(M[0]) : 0.0;
  size_t rank = 0;
  while (rank < std::min(m, removed) && std::fabs(M[rank * m + rank]) > scale * tol) ++rank;
  const size_t sep = n - removed;
  block_qr(rank, removed, sep);
  const size_t rows = std::min(m - rank, sep);
  out.a.assign(rows * sep, 0.);
  out.b.assign(rows, 0.);
  for (size_t row = 0; row < rows; ++row) {
    out.b[row] = M[n * m + rank + row];
    for (size_t col = row; col < sep; ++col) out.a[perm[col] * rows + row] = M[(removed + col) * m + rank + row];
  }
  double constant = 0;
  for (size_t row = rank + rows; row < m; ++row) {
    double r = M[n * m + row];
    constant += (0.5 * r) * r;
  }
  for (double v : out.a)
    if (!is_fin(v)) return INVALID_EVALUATION;
  for (double v : out.b)
    if (!is_fin(v)) return INVALID_EVALUATION;
  if (!is_fin(constant)) return INVALID_EVALUATION;
  for (size_t i = 0; i < std::min(m, removed); ++i)
    if (!is_fin(M[i * m + i])) return INVALID_EVALUATION;
  out.constant = constant;
  out.rank = rank;
  out.rows = rows;
  return OK;
}
