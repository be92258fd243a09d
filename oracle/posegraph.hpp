// ORACLE — test infrastructure only (included by oracle.cpp).
//
// SE(3) geometry of examples/slam/geometry.rs:13-212 (Pose: unit quaternion +
// translation, body-frame tangent [v, w], right increments), the PosePrior of
// examples/slam.rs:26-56, and the pose-graph window of the batched-window
// workload: poses x_0..x_{n-1}, an anchor PosePrior on x_0 and relative-pose
// factors r = Log(z^-1 x_i^-1 x_j). The reference defines no relative-pose
// factor; this one is composed from its primitives (local, log_jacobian,
// adjoint): dr/d(delta_j) = Jr^-1(r), dr/d(delta_i) = -Jr^-1(r) Ad((x_i^-1 x_j)^-1).
// A window is solved by LevenbergMarquardt over DenseSchur(6n, []) and its
// oldest poses are then eliminated by the square-root reduction of
// src/marginalization.rs:458-513 into a prior on the separator poses.

struct Pose3 {
  double q[4];  // w, x, y, z (unit)
  double t[3];
};
void qmul(const double* a, const double* b, double* o) {
  double w = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  double x = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  double y = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  double z = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
  o[0] = w; o[1] = x; o[2] = y; o[3] = z;
}
void qrot(const double* q, const double* v, double* o) {  // q v q^*
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  // t = 2 (u x v); o = v + w t + u x t
  double tx = 2 * (y * v[2] - z * v[1]), ty = 2 * (z * v[0] - x * v[2]), tz = 2 * (x * v[1] - y * v[0]);
  o[0] = v[0] + w * tx + (y * tz - z * ty);
  o[1] = v[1] + w * ty + (z * tx - x * tz);
  o[2] = v[2] + w * tz + (x * ty - y * tx);
}
void qmat(const double* q, double* R) {  // row-major 3x3
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z); R[2] = 2 * (x * z + w * y);
  R[3] = 2 * (x * y + w * z); R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
  R[6] = 2 * (x * z - w * y); R[7] = 2 * (y * z + w * x); R[8] = 1 - 2 * (x * x + y * y);
}
Pose3 compose(const Pose3& a, const Pose3& b) {  // geometry.rs:29-34
  Pose3 o;
  qmul(a.q, b.q, o.q);
  double rt[3];
  qrot(a.q, b.t, rt);
  for (int i = 0; i < 3; ++i) o.t[i] = rt[i] + a.t[i];
  return o;
}
Pose3 inverse(const Pose3& a) {  // :36-42
  Pose3 o;
  o.q[0] = a.q[0]; o.q[1] = -a.q[1]; o.q[2] = -a.q[2]; o.q[3] = -a.q[3];
  double rt[3];
  qrot(o.q, a.t, rt);
  for (int i = 0; i < 3; ++i) o.t[i] = -rt[i];
  return o;
}
void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
Pose3 pose_exp(const double* d) {  // :44-79
  const double* v = d;
  const double* w = d + 3;
  double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double qw, a, b, dd;
  if (t2 < 1e-2) {
    qw = 1 + t2 * (-1.0 / 8.0 + t2 * (1.0 / 384.0 - t2 * (1.0 / 46080.0)));
    a = 0.5 + t2 * (-1.0 / 48.0 + t2 * (1.0 / 3840.0 - t2 * (1.0 / 645120.0)));
    b = 0.5 + t2 * (-1.0 / 24.0 + t2 * (1.0 / 720.0 - t2 * (1.0 / 40320.0)));
    dd = 1.0 / 6.0 + t2 * (-1.0 / 120.0 + t2 * (1.0 / 5040.0 - t2 * (1.0 / 362880.0)));
  } else {
    double angle = std::sqrt(t2), half = angle * 0.5;
    a = std::sin(half) / angle;
    qw = std::cos(half);
    b = 2.0 * a * a;
    dd = (angle - std::sin(angle)) / (angle * t2);
  }
  Pose3 p;
  double qn = std::sqrt(qw * qw + a * a * t2);
  p.q[0] = qw / qn;
  for (int i = 0; i < 3; ++i) p.q[1 + i] = w[i] * a / qn;
  double c[3], wc[3];
  cross3(w, v, c);
  cross3(w, c, wc);
  for (int i = 0; i < 3; ++i) p.t[i] = v[i] + c[i] * b + wc[i] * dd;
  return p;
}
void pose_log(const Pose3& p, double* out) {  // :81-111
  double q[4] = {p.q[0], p.q[1], p.q[2], p.q[3]};
  if (q[0] < 0)
    for (double& e : q) e = -e;
  double s2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  double scale;
  if (s2 < 1e-4) {
    scale = 2.0 + s2 * (1.0 / 3.0 + s2 * (3.0 / 20.0 + s2 * (5.0 / 56.0)));
  } else {
    double s = std::sqrt(s2);
    scale = 2.0 * std::atan2(s, q[0]) / s;
  }
  double w[3] = {q[1] * scale, q[2] * scale, q[3] * scale};
  double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double coef;
  if (t2 < 1e-2) {
    coef = 1.0 / 12.0 + t2 * (1.0 / 720.0 + t2 * (1.0 / 30240.0 + t2 * (1.0 / 1209600.0)));
  } else {
    double half = std::sqrt(t2) * 0.5;
    coef = (1.0 - half / std::tan(half)) / t2;
  }
  double c[3], wc[3];
  cross3(w, p.t, c);
  cross3(w, c, wc);
  for (int i = 0; i < 3; ++i) {
    out[i] = p.t[i] - c[i] * 0.5 + wc[i] * coef;
    out[3 + i] = w[i];
  }
}
// 6x6 matrices below are row-major.
void pose_adjoint(const Pose3& p, double* A) {  // :113-127
  double R[9];
  qmat(p.q, R);
  std::fill(A, A + 36, 0.);
  double tx[9] = {0, -p.t[2], p.t[1], p.t[2], 0, -p.t[0], -p.t[1], p.t[0], 0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      A[i * 6 + j] = R[i * 3 + j];
      A[(3 + i) * 6 + 3 + j] = R[i * 3 + j];
      double s = 0;
      for (int k = 0; k < 3; ++k) s += tx[i * 3 + k] * R[k * 3 + j];
      A[i * 6 + 3 + j] = s;
    }
}
void so3_coefficients(double t2, double* b, double* c) {  // :141-161
  if (t2 < 0.25) {
    *b = 0.5 + t2 * (-1.0 / 24.0 + t2 * (1.0 / 720.0 + t2 * (-1.0 / 40320.0 + t2 * (1.0 / 3628800.0 - t2 * (1.0 / 479001600.0)))));
    *c = 1.0 / 6.0 + t2 * (-1.0 / 120.0 + t2 * (1.0 / 5040.0 + t2 * (-1.0 / 362880.0 + t2 * (1.0 / 39916800.0 - t2 * (1.0 / 6227020800.0)))));
  } else {
    double angle = std::sqrt(t2);
    double a = std::sin(angle * 0.5) / angle;
    *b = 2.0 * a * a;
    *c = (1.0 - std::sin(angle) / angle) / t2;
  }
}
void mat3mul_rm(const double* A, const double* B, double* C) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += A[i * 3 + k] * B[k * 3 + j];
      C[i * 3 + j] = s;
    }
}
void skew_rm(const double* v, double* K) {
  K[0] = 0; K[1] = -v[2]; K[2] = v[1];
  K[3] = v[2]; K[4] = 0; K[5] = -v[0];
  K[6] = -v[1]; K[7] = v[0]; K[8] = 0;
}
// right_jacobian_blocks (:169-206): J (3x3) and Q (3x3), row-major.
void right_jacobian_blocks(const double* d, double* J, double* Q) {
  const double* v = d;
  const double* w = d + 3;
  double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double b, dd;
  so3_coefficients(t2, &b, &dd);
  double db, ddd;
  if (t2 < 0.25) {
    db = -1.0 / 12.0 + t2 * (1.0 / 180.0 + t2 * (-1.0 / 6720.0 + t2 * (1.0 / 453600.0 - t2 * (1.0 / 47900160.0))));
    ddd = -1.0 / 60.0 + t2 * (1.0 / 1260.0 + t2 * (-1.0 / 60480.0 + t2 * (1.0 / 4989600.0 - t2 * (1.0 / 622702080.0))));
  } else {
    db = (1.0 - t2 * dd - 2.0 * b) / t2;
    ddd = (b - 3.0 * dd) / t2;
  }
  double W[9], W2[9];
  skew_rm(w, W);
  mat3mul_rm(W, W, W2);
  for (int i = 0; i < 9; ++i) J[i] = (i % 4 == 0 ? 1.0 : 0.0) - W[i] * b + W2[i] * dd;
  double c[3], wc[3];
  cross3(w, v, c);
  cross3(w, c, wc);
  double V[9];
  skew_rm(v, V);
  double wv = w[0] * v[0] + w[1] * v[1] + w[2] * v[2];
  double D[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double x = -V[i * 3 + j] * b;
      x += (w[i] * v[j] + (i == j ? wv : 0.0) - v[i] * w[j] * 2.0) * dd;
      x += (c[i] * db + wc[i] * ddd) * w[j];
      D[i * 3 + j] = x;
    }
  double Rinv[9];
  for (int i = 0; i < 9; ++i) Rinv[i] = (i % 4 == 0 ? 1.0 : 0.0) - W[i] * (1.0 - t2 * dd) + W2[i] * b;
  mat3mul_rm(Rinv, D, Q);
}
void assemble6(const double* J, const double* Q, double* out) {  // :208-217
  std::fill(out, out + 36, 0.);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      out[i * 6 + j] = J[i * 3 + j];
      out[(3 + i) * 6 + 3 + j] = J[i * 3 + j];
      out[i * 6 + 3 + j] = Q[i * 3 + j];
    }
}
void pose_right_jacobian(const double* d, double* out) {
  double J[9], Q[9];
  right_jacobian_blocks(d, J, Q);
  assemble6(J, Q, out);
}
bool inv3(const double* A, double* I) {
  double c00 = A[4] * A[8] - A[5] * A[7], c01 = A[5] * A[6] - A[3] * A[8], c02 = A[3] * A[7] - A[4] * A[6];
  double det = A[0] * c00 + A[1] * c01 + A[2] * c02;
  if (det == 0 || !is_fin(det)) return false;
  double id = 1.0 / det;
  I[0] = c00 * id; I[1] = (A[2] * A[7] - A[1] * A[8]) * id; I[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  I[3] = c01 * id; I[4] = (A[0] * A[8] - A[2] * A[6]) * id; I[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  I[6] = c02 * id; I[7] = (A[1] * A[6] - A[0] * A[7]) * id; I[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return true;
}
// log_jacobian (:289-304): Jr^-1 = [J^-1, -J^-1 Q J^-1; 0, J^-1].
int log_jacobian(const double* d, double* out) {
  for (int i = 0; i < 6; ++i)
    if (!is_fin(d[i])) return INVALID_EVALUATION;
  double J[9], Q[9], Ji[9], T[9], U[9];
  right_jacobian_blocks(d, J, Q);
  if (!inv3(J, Ji)) return INVALID_EVALUATION;
  mat3mul_rm(Ji, Q, T);
  mat3mul_rm(T, Ji, U);
  for (double& e : U) e = -e;
  assemble6(Ji, U, out);
  for (int i = 0; i < 36; ++i)
    if (!is_fin(out[i])) return INVALID_EVALUATION;
  return OK;
}
void pose_local(const Pose3& a, const Pose3& b, double* out) { pose_log(compose(inverse(a), b), out); }

// ------------------------------------------------------- pose-graph window
struct RelativeFactor {
  uint32_t i, j;
  Pose3 z;
};
// A prior on the window's first s poses, Priors::update (marginalization.rs:
// 157-231): r = b + sum_i A_i Log(ref_i^-1 x_i) (anchors in order, columns in
// order), J_i = A_i Jr^-1(Log(ref_i^-1 x_i)); A is m x 6s column-major. The
// anchor PosePrior (examples/slam.rs:26-56, r = Log(z^-1 x_0), J = Jr^-1(r))
// is the case s = 1, A = I, b = 0, ref = z, and gives its values exactly.
struct WindowPriorFactor {
  size_t s = 0, m = 0;
  std::vector<double> A, b;
  std::vector<Pose3> ref;
  void anchor(const Pose3& z) {
    s = 1;
    m = 6;
    A.assign(36, 0.0);
    for (int k = 0; k < 6; ++k) A[k * 6 + k] = 1.0;
    b.assign(6, 0.0);
    ref.assign(1, z);
  }
};
struct PoseWindow : Problem {
  std::vector<Pose3> x, tx;
  WindowPriorFactor prior;
  std::vector<RelativeFactor> rel;
  bool trial = false;

  size_t dimension() override { return 6 * x.size(); }
  // r (m values) and, with J, the m x 6s Jacobian (column-major).
  int prior_residual(const std::vector<Pose3>& X, double* r, double* J) const {
    const size_t m = prior.m;
    for (size_t row = 0; row < m; ++row) r[row] = prior.b[row];
    for (size_t i = 0; i < prior.s; ++i) {
      double d[6], jr[36];
      pose_local(prior.ref[i], X[i], d);
      for (int k = 0; k < 6; ++k)
        if (!is_fin(d[k])) return INVALID_EVALUATION;
      for (size_t row = 0; row < m; ++row)
        for (int col = 0; col < 6; ++col) r[row] += prior.A[(6 * i + col) * m + row] * d[col];
      if (J) {
        int st = log_jacobian(d, jr);
        if (st) return st;
        for (int col = 0; col < 6; ++col)
          for (size_t row = 0; row < m; ++row) {
            double v = 0;
            for (int k = 0; k < 6; ++k) v += prior.A[(6 * i + k) * m + row] * jr[k * 6 + col];
            J[(6 * i + col) * m + row] = v;
          }
      }
    }
    for (size_t row = 0; row < m; ++row)
      if (!is_fin(r[row])) return INVALID_EVALUATION;
    return OK;
  }
  int rel_residual(const std::vector<Pose3>& X, const RelativeFactor& f, double* r, double* Ji, double* Jj) const {
    Pose3 T = compose(inverse(X[f.i]), X[f.j]);
    pose_local(f.z, T, r);
    if (!Ji) {
      for (int k = 0; k < 6; ++k)
        if (!is_fin(r[k])) return INVALID_EVALUATION;
      return OK;
    }
    int s = log_jacobian(r, Jj);
    if (s) return s;
    double A[36];
    pose_adjoint(inverse(T), A);
    for (int a = 0; a < 6; ++a)
      for (int b = 0; b < 6; ++b) {
        double v = 0;
        for (int k = 0; k < 6; ++k) v += Jj[a * 6 + k] * A[k * 6 + b];
        Ji[a * 6 + b] = -v;
      }
    return OK;
  }
  int cost(bool t, double* out) override {
    const std::vector<Pose3>& X = t ? tx : x;
    double total = 0, r[6];
    std::vector<double> rp(prior.m);
    int s = prior_residual(X, rp.data(), nullptr);
    if (s) return s;
    double c = 0;
    for (double e : rp) c += 0.5 * e * e;
    if ((s = checked(OK, c))) return s;
    total += c;
    for (const auto& f : rel) {
      if ((s = rel_residual(X, f, r, nullptr, nullptr))) return s;
      c = 0;
      for (double e : r) c += 0.5 * e * e;
      if ((s = checked(OK, c))) return s;
      total += c;
    }
    *out = total;
    return checked(OK, total);
  }
  // Emission order: the prior pool, then the relative factors in insertion order.
  int linearize(Linear& s) override {
    s.clear();
    double r[6], Ji[36], Jj[36];
    size_t cols[2], widths[2] = {6, 6};
    ptrdiff_t rs[2] = {6, 6}, cs[2] = {1, 1};
    {  // the prior: one emission with a block per anchored pose (marginalization.rs:249-277)
      const size_t m = prior.m, np = prior.s;
      std::vector<double> rp(m), jp(m * 6 * np);
      int st = prior_residual(x, rp.data(), jp.data());
      if (st) return st;
      std::vector<size_t> pc(np), pw(np, 6);
      std::vector<const double*> pj(np);
      std::vector<ptrdiff_t> prs(np, 1), pcs(np, (ptrdiff_t)m);
      for (size_t i = 0; i < np; ++i) {
        pc[i] = 6 * i;
        pj[i] = jp.data() + 6 * i * m;
      }
      if ((st = s.accumulate(m, rp.data(), np, pc.data(), pw.data(), pj.data(), prs.data(), pcs.data()))) return st;
    }
    int st = OK;
    for (const auto& f : rel) {
      if ((st = rel_residual(x, f, r, Ji, Jj))) return st;
      cols[0] = 6 * (size_t)f.i;
      cols[1] = 6 * (size_t)f.j;
      const double* jj[2] = {Ji, Jj};
      if ((st = s.accumulate(6, r, 2, cols, widths, jj, rs, cs))) return st;
    }
    return OK;
  }
  int stage(const double* d) override {  // retract x (+) d = x Exp(d)
    tx.resize(x.size());
    for (size_t k = 0; k < x.size(); ++k) tx[k] = compose(x[k], pose_exp(d + 6 * k));
    trial = true;
    return OK;
  }
  void accept() override {
    if (trial) {
      x.swap(tx);
      trial = false;
    }
  }
  void reject() override { trial = false; }
};

// Square-root marginalization of poses [0, removed) of a window at its current
// estimate: rows of every factor touching a removed pose, columns = removed
// poses then the separator poses (touched poses >= removed, increasing index).
struct WindowPrior {
  std::vector<uint32_t> separator;
  EliminationResult elim;
};
int marginalize_window(const PoseWindow& w, size_t removed_poses, WindowPrior& out) {
  std::vector<char> touched(w.x.size(), 0);
  std::vector<const RelativeFactor*> facs;
  // the window prior touches its poses [0, s), pose 0 among the removed ones
  for (size_t k = 0; k < w.prior.s && k < w.x.size(); ++k) touched[k] = 1;
  for (const auto& f : w.rel)
    if (f.i < removed_poses || f.j < removed_poses) {
      facs.push_back(&f);
      touched[f.i] = touched[f.j] = 1;
    }
  out.separator.clear();
  for (size_t k = removed_poses; k < w.x.size(); ++k)
    if (touched[k]) out.separator.push_back((uint32_t)k);
  std::vector<size_t> column(w.x.size(), NONE);
  for (size_t k = 0; k < removed_poses && k < w.x.size(); ++k) column[k] = 6 * k;
  for (size_t s = 0; s < out.separator.size(); ++s) column[out.separator[s]] = 6 * (removed_poses + s);
  const size_t n = 6 * (removed_poses + out.separator.size()), width = n + 1;
  const size_t mp = w.prior.m, m = mp + 6 * facs.size();
  std::vector<double> rows(m * width, 0.);
  double r[6], Ji[36], Jj[36];
  {
    std::vector<double> rp(mp), jp(mp * 6 * w.prior.s);
    int st = w.prior_residual(w.x, rp.data(), jp.data());
    if (st) return st;
    for (size_t a = 0; a < mp; ++a) {
      for (size_t i = 0; i < w.prior.s; ++i)
        for (int b = 0; b < 6; ++b) rows[a * width + column[i] + b] = jp[(6 * i + b) * mp + a];
      rows[a * width + n] = rp[a];
    }
  }
  int st = OK;
  for (size_t k = 0; k < facs.size(); ++k) {
    if ((st = w.rel_residual(w.x, *facs[k], r, Ji, Jj))) return st;
    size_t base = mp + 6 * k;
    for (int a = 0; a < 6; ++a) {
      for (int b = 0; b < 6; ++b) {
        rows[(base + a) * width + column[facs[k]->i] + b] += Ji[a * 6 + b];
        rows[(base + a) * width + column[facs[k]->j] + b] += Jj[a * 6 + b];
      }
      rows[(base + a) * width + n] = r[a];
    }
  }
  return eliminate(m, n, rows.data(), 6 * removed_poses, -1.0, out.elim);
}
