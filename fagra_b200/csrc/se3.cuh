// SE(3) on the device, following fagra's examples/slam/geometry.rs:13-212:
// unit quaternion (w, x, y, z) + translation, body-frame tangents [v, w],
// right increments x (+) d = x Exp(d). 6x6 matrices are row-major.
#pragma once
#include <cmath>

namespace fg {

struct Pose7 {
  double q[4];
  double t[3];
};

__device__ __forceinline__ Pose7 load_pose(const double* p) {
  Pose7 o;
  o.q[0] = p[0]; o.q[1] = p[1]; o.q[2] = p[2]; o.q[3] = p[3];
  o.t[0] = p[4]; o.t[1] = p[5]; o.t[2] = p[6];
  return o;
}
__device__ __forceinline__ void store_pose(const Pose7& p, double* o) {
  o[0] = p.q[0]; o[1] = p.q[1]; o[2] = p.q[2]; o[3] = p.q[3];
  o[4] = p.t[0]; o[5] = p.t[1]; o[6] = p.t[2];
}
__device__ __forceinline__ void se3_qmul(const double* a, const double* b, double* o) {
  double w = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  double x = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  double y = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  double z = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
  o[0] = w; o[1] = x; o[2] = y; o[3] = z;
}
__device__ __forceinline__ void se3_qrot(const double* q, const double* v, double* o) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  double tx = 2 * (y * v[2] - z * v[1]), ty = 2 * (z * v[0] - x * v[2]), tz = 2 * (x * v[1] - y * v[0]);
  o[0] = v[0] + w * tx + (y * tz - z * ty);
  o[1] = v[1] + w * ty + (z * tx - x * tz);
  o[2] = v[2] + w * tz + (x * ty - y * tx);
}
__device__ __forceinline__ void se3_cross(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ Pose7 se3_compose(const Pose7& a, const Pose7& b) {
  Pose7 o;
  se3_qmul(a.q, b.q, o.q);
  double rt[3];
  se3_qrot(a.q, b.t, rt);
  for (int i = 0; i < 3; ++i) o.t[i] = rt[i] + a.t[i];
  return o;
}
__device__ __forceinline__ Pose7 se3_inverse(const Pose7& a) {
  Pose7 o;
  o.q[0] = a.q[0]; o.q[1] = -a.q[1]; o.q[2] = -a.q[2]; o.q[3] = -a.q[3];
  double rt[3];
  se3_qrot(o.q, a.t, rt);
  for (int i = 0; i < 3; ++i) o.t[i] = -rt[i];
  return o;
}
// Pose::exp (geometry.rs:44-79), series below 1e-2 squared angle.
__device__ inline Pose7 se3_exp(const double* d) {
  const double* v = d;
  const double* w = d + 3;
  const double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double qw, a, b, dd;
  if (t2 < 1e-2) {
    qw = 1 + t2 * (-1.0 / 8.0 + t2 * (1.0 / 384.0 - t2 * (1.0 / 46080.0)));
    a = 0.5 + t2 * (-1.0 / 48.0 + t2 * (1.0 / 3840.0 - t2 * (1.0 / 645120.0)));
    b = 0.5 + t2 * (-1.0 / 24.0 + t2 * (1.0 / 720.0 - t2 * (1.0 / 40320.0)));
    dd = 1.0 / 6.0 + t2 * (-1.0 / 120.0 + t2 * (1.0 / 5040.0 - t2 * (1.0 / 362880.0)));
  } else {
    const double angle = sqrt(t2), half = angle * 0.5;
    a = sin(half) / angle;
    qw = cos(half);
    b = 2.0 * a * a;
    dd = (angle - sin(angle)) / (angle * t2);
  }
  Pose7 p;
  const double qn = sqrt(qw * qw + a * a * t2);
  p.q[0] = qw / qn;
  for (int i = 0; i < 3; ++i) p.q[1 + i] = w[i] * a / qn;
  double c[3], wc[3];
  se3_cross(w, v, c);
  se3_cross(w, c, wc);
  for (int i = 0; i < 3; ++i) p.t[i] = v[i] + c[i] * b + wc[i] * dd;
  return p;
}
// Pose::log (geometry.rs:81-111).
__device__ inline void se3_log(const Pose7& p, double* out) {
  double q[4] = {p.q[0], p.q[1], p.q[2], p.q[3]};
  if (q[0] < 0)
    for (int i = 0; i < 4; ++i) q[i] = -q[i];
  const double s2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  double scale;
  if (s2 < 1e-4) {
    scale = 2.0 + s2 * (1.0 / 3.0 + s2 * (3.0 / 20.0 + s2 * (5.0 / 56.0)));
  } else {
    const double s = sqrt(s2);
    scale = 2.0 * atan2(s, q[0]) / s;
  }
  double w[3] = {q[1] * scale, q[2] * scale, q[3] * scale};
  const double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double coef;
  if (t2 < 1e-2) {
    coef = 1.0 / 12.0 + t2 * (1.0 / 720.0 + t2 * (1.0 / 30240.0 + t2 * (1.0 / 1209600.0)));
  } else {
    const double half = sqrt(t2) * 0.5;
    coef = (1.0 - half / tan(half)) / t2;
  }
  double c[3], wc[3];
  se3_cross(w, p.t, c);
  se3_cross(w, c, wc);
  for (int i = 0; i < 3; ++i) {
    out[i] = p.t[i] - c[i] * 0.5 + wc[i] * coef;
    out[3 + i] = w[i];
  }
}
__device__ __forceinline__ void se3_qmat(const double* q, double* R) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z); R[2] = 2 * (x * z + w * y);
  R[3] = 2 * (x * y + w * z); R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
  R[6] = 2 * (x * z - w * y); R[7] = 2 * (y * z + w * x); R[8] = 1 - 2 * (x * x + y * y);
}
// Pose::adjoint (geometry.rs:113-127): [R, [t]x R; 0, R].
__device__ inline void se3_adjoint(const Pose7& p, double* A) {
  double R[9];
  se3_qmat(p.q, R);
  const double tx[9] = {0, -p.t[2], p.t[1], p.t[2], 0, -p.t[0], -p.t[1], p.t[0], 0};
  for (int i = 0; i < 36; ++i) A[i] = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      A[i * 6 + j] = R[i * 3 + j];
      A[(3 + i) * 6 + 3 + j] = R[i * 3 + j];
      double s = 0;
      for (int k = 0; k < 3; ++k) s += tx[i * 3 + k] * R[k * 3 + j];
      A[i * 6 + 3 + j] = s;
    }
}
__device__ __forceinline__ void se3_mm3(const double* A, const double* B, double* C) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += A[i * 3 + k] * B[k * 3 + j];
      C[i * 3 + j] = s;
    }
}
__device__ __forceinline__ void se3_skew(const double* v, double* K) {
  K[0] = 0; K[1] = -v[2]; K[2] = v[1];
  K[3] = v[2]; K[4] = 0; K[5] = -v[0];
  K[6] = -v[1]; K[7] = v[0]; K[8] = 0;
}
// so3_coefficients and right_jacobian_blocks (geometry.rs:141-206).
__device__ inline void se3_right_jacobian_blocks(const double* d, double* J, double* Q) {
  const double* v = d;
  const double* w = d + 3;
  const double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double b, dd, db, ddd;
  if (t2 < 0.25) {
    b = 0.5 + t2 * (-1.0 / 24.0 + t2 * (1.0 / 720.0 + t2 * (-1.0 / 40320.0 + t2 * (1.0 / 3628800.0 - t2 * (1.0 / 479001600.0)))));
    dd = 1.0 / 6.0 + t2 * (-1.0 / 120.0 + t2 * (1.0 / 5040.0 + t2 * (-1.0 / 362880.0 + t2 * (1.0 / 39916800.0 - t2 * (1.0 / 6227020800.0)))));
    db = -1.0 / 12.0 + t2 * (1.0 / 180.0 + t2 * (-1.0 / 6720.0 + t2 * (1.0 / 453600.0 - t2 * (1.0 / 47900160.0))));
    ddd = -1.0 / 60.0 + t2 * (1.0 / 1260.0 + t2 * (-1.0 / 60480.0 + t2 * (1.0 / 4989600.0 - t2 * (1.0 / 622702080.0))));
  } else {
    const double angle = sqrt(t2);
    const double a = sin(angle * 0.5) / angle;
    b = 2.0 * a * a;
    dd = (1.0 - sin(angle) / angle) / t2;
    db = (1.0 - t2 * dd - 2.0 * b) / t2;
    ddd = (b - 3.0 * dd) / t2;
  }
  double W[9], W2[9];
  se3_skew(w, W);
  se3_mm3(W, W, W2);
  for (int i = 0; i < 9; ++i) J[i] = (i % 4 == 0 ? 1.0 : 0.0) - W[i] * b + W2[i] * dd;
  double c[3], wc[3];
  se3_cross(w, v, c);
  se3_cross(w, c, wc);
  double V[9];
  se3_skew(v, V);
  const double wv = w[0] * v[0] + w[1] * v[1] + w[2] * v[2];
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
  se3_mm3(Rinv, D, Q);
}
// log_jacobian (geometry.rs:289-304): Jr^-1 = [J^-1, -J^-1 Q J^-1; 0, J^-1];
// false on a nonfinite input, a singular J or a nonfinite result.
__device__ inline bool se3_log_jacobian(const double* d, double* out) {
  for (int i = 0; i < 6; ++i)
    if (!isfinite(d[i])) return false;
  double J[9], Q[9];
  se3_right_jacobian_blocks(d, J, Q);
  const double c00 = J[4] * J[8] - J[5] * J[7], c01 = J[5] * J[6] - J[3] * J[8], c02 = J[3] * J[7] - J[4] * J[6];
  const double det = J[0] * c00 + J[1] * c01 + J[2] * c02;
  if (det == 0 || !isfinite(det)) return false;
  const double id = 1.0 / det;
  double Ji[9] = {c00 * id, (J[2] * J[7] - J[1] * J[8]) * id, (J[1] * J[5] - J[2] * J[4]) * id,
                  c01 * id, (J[0] * J[8] - J[2] * J[6]) * id, (J[2] * J[3] - J[0] * J[5]) * id,
                  c02 * id, (J[1] * J[6] - J[0] * J[7]) * id, (J[0] * J[4] - J[1] * J[3]) * id};
  double T[9], U[9];
  se3_mm3(Ji, Q, T);
  se3_mm3(T, Ji, U);
  for (int i = 0; i < 36; ++i) out[i] = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      out[i * 6 + j] = Ji[i * 3 + j];
      out[(3 + i) * 6 + 3 + j] = Ji[i * 3 + j];
      out[i * 6 + 3 + j] = -U[i * 3 + j];
    }
  for (int i = 0; i < 36; ++i)
    if (!isfinite(out[i])) return false;
  return true;
}

}  // namespace fg
