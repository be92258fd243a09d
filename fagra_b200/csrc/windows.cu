// Batched pose-graph windows: thousands of independent SE(3) windows of
// uneven size solved in one persistent launch, one CTA per window at a time.
//
// Per window (n poses, N = 6n coordinates) the CTA runs fagra's
// LevenbergMarquardt (src/optimization/levenberg_marquardt.rs:330-472) over
// a DenseSchur backend with an all-retained partition (src/dense_schur.rs:
// scaled normal equations, LM damping lambda I in scaled coordinates, dense
// Cholesky, DenseSchur::solve_damped's prediction -g.d - |J d|^2 / 2), then
// eliminates the window's oldest poses by the square-root reduction of
// src/marginalization.rs:458-513 (column-pivoted Householder QR of [J | r]
// over the factors that touch them) into a prior on the separator poses.
//
// Factors, in emission order: the window prior and relative-pose factors
// r = Log(z^-1 x_i^-1 x_j) with dr/dd_j = Jr^-1(r), dr/dd_i = -Jr^-1(r)
// Ad((x_i^-1 x_j)^-1), composed from the reference's SE(3) primitives. The
// window prior is Priors::update (src/marginalization.rs:157-231) on the
// window's first s poses, r = b + sum_i A_i Log(ref_i^-1 x_i) with Jacobian
// blocks A_i Jr^-1(Log(ref_i^-1 x_i)): by default the anchor PosePrior of
// examples/slam.rs:26-56 (s = 1, A = I, b = 0, ref = z: r = Log(z^-1 x_0)),
// or a marginal prior from an earlier window's elimination
// (fg_windows_set_priors), which is how a window's marginal prior feeds the
// next window's device LM solve.
//
// Dense work stays inside the CTA: a right-looking blocked Cholesky (panel
// CB, trailing tiles of 64 x 64 with 4 x 4 register blocks from shared
// memory), blocked triangular solves, and the pivoted QR. The factorization
// runs in TF = double (the reference arithmetic) or TF = float with FP64
// iterative refinement of every solve against the FP64 scaled normal matrix.
// Windows are taken from an atomic queue in decreasing size; the CTA count per
// SM and the panel width are chosen by an autotuner that times a sample of
// the batch once per handle.
#include "common.cuh"
#include "se3.cuh"
#include "dense.cuh"
#include <algorithm>
#include <cstring>
#include <numeric>
#include <type_traits>

namespace fg {

struct WinOptions {
  double gradient_tolerance, step_tolerance, cost_tolerance;
  double initial_damping, min_damping, max_damping, min_column_norm, acceptance_threshold;
  unsigned max_iterations, max_trials;
  int removed;  // poses to eliminate per window
  int refine;   // FP64 refinement passes per solve (FP32 factorization)
};

struct WinDev {
  int W;
  const int64_t* pose_off;  // W+1
  const int64_t* rel_off;   // W+1
  const uint32_t* rel_ij;   // 2 per relative factor, window-local
  const double* rel_z;      // 7 per relative factor
  const int32_t* pr_s;      // W: prior poses (the window's first s)
  const int32_t* pr_m;      // W: prior rows
  const int64_t* pr_aoff;   // W: start of the window's A (m x 6s, column-major) in pr_A
  const int64_t* pr_boff;   // W: start of its b (m) in pr_b
  const int64_t* pr_roff;   // W: first reference pose (7 each) in pr_ref
  const int64_t* pf_off;    // W: scratch start: r (m) | J (m x 6s) | u (m) | d (6s) | Jr^-1 (36s)
  const double* pr_A;
  const double* pr_b;
  const double* pr_ref;
  double* x;                // 7 per pose (in/out)
  double* xt;               // 7 per pose (trial)
  const int64_t* inc_off;   // per global pose, CSR of incident relative factors
  const int32_t* inc;       // (factor << 1) | side, side 1 = j
  double* fac;              // FS per relative factor: r, Ji, Jj, J d
  double* pfac;             // prior scratch (pf_off)
  const int64_t* tile_off;  // W+1: 64-row tiles of each window's coordinates
  const int32_t* tile_cmin; // per tile: first 64-column tile of its rows' envelope
  const int64_t* mf_off;    // W+1: relative factors touching the eliminated poses
  const int32_t* mf;        // global factor indices
  const int64_t* sep_off;   // W+1: separator poses (window-local, increasing)
  const uint32_t* sep;
  const int64_t* a_off;     // W+1: prior A capacity (separator columns squared)
  double* prior_a;
  double* prior_b;          // 6 * sep_off[w] + row
  fg_window_report* reports;
  const int32_t* order;     // window schedule
  unsigned* queue;
  double* G;                // per CTA: Nmax^2 symmetric scaled normal matrix
  void* F;                  // per CTA: Nmax^2 factor (TF)
  double* M;                // per CTA: marginalization system, column-major
  double* V;                // per CTA: 4 x Nmax doubles (gradient, scales, step, residual)
  void* TV;                 // per CTA: Nmax TF (factor-precision solve vector)
  size_t g_stride, m_stride;
  int nmax;
};

constexpr int FS = 84;    // doubles per relative factor in the scratch
constexpr int PR_MAX_POSES = 64;  // poses a window prior may cover
constexpr int PR_MAX_ROWS = 384;  // rows a window prior may have

// ------------------------------------------------------------ factors
// Residual (and Jacobians) of relative factor f at poses X; false if nonfinite.
__device__ inline bool rel_eval(const WinDev& D, int64_t f, const double* X, double* r, double* Ji, double* Jj) {
  const uint32_t i = D.rel_ij[2 * f], j = D.rel_ij[2 * f + 1];
  const Pose7 T = se3_compose(se3_inverse(load_pose(X + 7 * (size_t)i)), load_pose(X + 7 * (size_t)j));
  se3_log(se3_compose(se3_inverse(load_pose(D.rel_z + 7 * f)), T), r);
  if (!Ji) {
    for (int k = 0; k < 6; ++k)
      if (!isfinite(r[k])) return false;
    return true;
  }
  if (!se3_log_jacobian(r, Jj)) return false;
  double A[36];
  se3_adjoint(se3_inverse(T), A);
  for (int a = 0; a < 6; ++a)
    for (int b = 0; b < 6; ++b) {
      double v = 0;
      for (int k = 0; k < 6; ++k) v += Jj[a * 6 + k] * A[k * 6 + b];
      Ji[a * 6 + b] = -v;
    }
  return true;
}
// The window prior of window w at poses X, all threads of the CTA:
// d_i = Log(ref_i^-1 x_i) (and Jr^-1(d_i) with `jac`), then r = b + sum_i A_i
// d_i and, with `jac`, J = [A_i Jr^-1(d_i)]_i into the window's scratch, in
// the order of Priors::update (anchors in order, columns in order). False if
// any value is nonfinite (uniform across the CTA).
struct WinPrior {
  int s, m;
  const double *A, *b, *ref;
  double *r, *J, *u, *d, *jr;
};
__device__ inline WinPrior win_prior(const WinDev& D, int w) {
  WinPrior P;
  P.s = D.pr_s[w];
  P.m = D.pr_m[w];
  P.A = D.pr_A + D.pr_aoff[w];
  P.b = D.pr_b + D.pr_boff[w];
  P.ref = D.pr_ref + 7 * D.pr_roff[w];
  P.r = D.pfac + D.pf_off[w];
  P.J = P.r + P.m;
  P.u = P.J + (size_t)P.m * 6 * P.s;
  P.d = P.u + P.m;
  P.jr = P.d + 6 * P.s;
  return P;
}
__device__ inline bool prior_terms(const WinPrior& P, const double* X, bool jac, double* red) {
  double bad = 0;
  for (int i = threadIdx.x; i < P.s; i += WNT) {
    se3_log(se3_compose(se3_inverse(load_pose(P.ref + 7 * (size_t)i)), load_pose(X + 7 * (size_t)i)), P.d + 6 * i);
    for (int k = 0; k < 6; ++k)
      if (!isfinite(P.d[6 * i + k])) bad = 1;
    if (jac && !se3_log_jacobian(P.d + 6 * i, P.jr + 36 * i)) bad = 1;
  }
  __syncthreads();
  for (int row = threadIdx.x; row < P.m; row += WNT) {
    double v = P.b[row];
    for (int i = 0; i < P.s; ++i)
      for (int col = 0; col < 6; ++col) v += P.A[(size_t)(6 * i + col) * P.m + row] * P.d[6 * i + col];
    P.r[row] = v;
    if (!isfinite(v)) bad = 1;
  }
  if (jac)
    for (int e = threadIdx.x; e < P.m * 6 * P.s; e += WNT) {
      const int row = e % P.m, cc = e / P.m, i = cc / 6, col = cc % 6;
      double v = 0;
      for (int k = 0; k < 6; ++k) v += P.A[(size_t)(6 * i + k) * P.m + row] * P.jr[36 * i + k * 6 + col];
      P.J[(size_t)cc * P.m + row] = v;
      if (!isfinite(v)) bad = 1;
    }
  __syncthreads();
  return wmax(bad, red) == 0;
}

// Cost of window w at poses X (pose base pb); bad = 1 if any factor is nonfinite.
__device__ inline double window_cost(const WinDev& D, int w, const double* X, double* red, int* bad) {
  const int64_t f0 = D.rel_off[w], f1 = D.rel_off[w + 1];
  double c = 0, nb = 0, r[6];
  for (int64_t f = f0 + threadIdx.x; f < f1; f += WNT) {
    if (!rel_eval(D, f, X, r, nullptr, nullptr)) {
      nb = 1;
      continue;
    }
    double e = 0;
    for (int k = 0; k < 6; ++k) e += 0.5 * r[k] * r[k];
    c += e;
  }
  const WinPrior P = win_prior(D, w);
  const bool pok = prior_terms(P, X, false, red);
  if (threadIdx.x == 0) {
    if (!pok) nb = 1;
    else
      for (int k = 0; k < P.m; ++k) c += 0.5 * P.r[k] * P.r[k];
  }
  const double tot = wsum(c, red);
  *bad = wmax(nb, red) != 0 || !isfinite(tot) || tot < 0;
  return tot;
}

// ------------------------------------------------------- window kernel
struct WinShared {
  double red[WNT / 32];
  int flag, bad;
};

template <class TF, int CB, int MINB>
__global__ void __launch_bounds__(WNT, MINB) k_windows(WinDev D, WinOptions O) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ WinShared S;
  __shared__ int next;
  double* g = D.V + (size_t)blockIdx.x * 4 * D.nmax;  // gradient
  double* sc = g + D.nmax;                              // column scales
  double* dv = sc + D.nmax;                             // scaled rhs / step (double)
  double* wv = dv + D.nmax;                             // refinement residual (double)
  TF* tv = reinterpret_cast<TF*>(D.TV) + (size_t)blockIdx.x * D.nmax;  // factor-precision vector
  TF* csm = reinterpret_cast<TF*>(smem_raw);            // Cholesky staging
  double* qnorms = reinterpret_cast<double*>(smem_raw);  // QR scratch (after the LM)
  int* qperm = reinterpret_cast<int*>(qnorms + D.nmax + 8);
  double* G = D.G + blockIdx.x * D.g_stride;
  TF* F = reinterpret_cast<TF*>(D.F) + blockIdx.x * D.g_stride;
  double* M = D.M + blockIdx.x * D.m_stride;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) next = (int)atomicAdd(D.queue, 1u);
    __syncthreads();
    const int slot = next;
    __syncthreads();
    if (slot >= D.W) break;
    const int w = D.order[slot];
    const int64_t p0 = D.pose_off[w];
    const int n = (int)(D.pose_off[w + 1] - p0), N = 6 * n;
    const int64_t f0 = D.rel_off[w], f1 = D.rel_off[w + 1];
    double* X = D.x + 7 * p0;
    double* XT = D.xt + 7 * p0;
    const int32_t* cmin = D.tile_cmin + D.tile_off[w];
    const int nT = (N + WCT - 1) / WCT;
    fg_window_report rep{};
    int status = FG_OK, term = 0;
    // ---- LevenbergMarquardt::optimize (levenberg_marquardt.rs:330-472)
    double lambda = O.initial_damping;
    rep.damping = lambda;
    int bad = 0;
    rep.cost_evaluations = 1;
    double current = window_cost(D, w, X, S.red, &bad);
    rep.initial_cost = current;
    bool stalled = false, tried_undamped = false;
    if (bad) status = FG_INVALID_EVALUATION;
    while (status == FG_OK && term == 0) {
      rep.linearizations += 1;
      // Linearize: factor residuals and Jacobians.
      double nb = 0;
      for (int64_t f = f0 + tid; f < f1; f += WNT) {
        double* o = D.fac + FS * f;
        if (!rel_eval(D, f, X, o, o + 6, o + 42)) nb = 1;
        for (int k = 0; k < 78; ++k)
          if (!isfinite(o[k])) nb = 1;
      }
      const WinPrior P = win_prior(D, w);
      if (!prior_terms(P, X, true, S.red)) nb = 1;
      if (wmax(nb, S.red) != 0) {
        status = FG_INVALID_EVALUATION;
        break;
      }
      // Gradient g = J^T r and column norms, per pose over its factors in emission order.
      double gmax = 0, gbad = 0;
      for (int p = tid; p < n; p += WNT) {
        double gg[6] = {0, 0, 0, 0, 0, 0}, ss[6] = {0, 0, 0, 0, 0, 0};
        if (p < P.s) {
          for (int c = 0; c < 6; ++c)
            for (int k = 0; k < P.m; ++k) {
              const double jv = P.J[(size_t)(6 * p + c) * P.m + k];
              gg[c] += jv * P.r[k];
              ss[c] += jv * jv;
            }
        }
        for (int64_t e = D.inc_off[p0 + p]; e < D.inc_off[p0 + p + 1]; ++e) {
          const int32_t code = D.inc[e];
          const double* o = D.fac + FS * (int64_t)(code >> 1);
          const double* J = o + ((code & 1) ? 42 : 6);
          for (int c = 0; c < 6; ++c)
            for (int k = 0; k < 6; ++k) {
              gg[c] += J[k * 6 + c] * o[k];
              ss[c] += J[k * 6 + c] * J[k * 6 + c];
            }
        }
        for (int c = 0; c < 6; ++c) {
          g[6 * p + c] = gg[c];
          if (!isfinite(gg[c])) gbad = 1;
          gmax = fmax(gmax, fabs(gg[c]));
          const double s = sqrt(ss[c]);
          if (!isfinite(s)) gbad = 1;
          sc[6 * p + c] = fmax(s, O.min_column_norm);
        }
      }
      gmax = wmax(gmax, S.red);
      if (wmax(gbad, S.red) != 0) {
        status = FG_INVALID_EVALUATION;
        break;
      }
      rep.gradient_norm = gmax;
      if (gmax <= O.gradient_tolerance) {
        term = 2;
        break;
      }
      if (stalled && (tried_undamped || rep.iterations == O.max_iterations)) {
        status = FG_NO_PROGRESS;
        break;
      }
      if (rep.iterations == O.max_iterations) {
        status = FG_NO_CONVERGENCE;
        break;
      }
      // prepare_damping: lower triangle of the scaled normal matrix
      // G = D^-1 J^T J D^-1 over the envelope tiles.
      for (int T = 0; T < nT; ++T)
        for (int C = cmin[T]; C <= T; ++C)
          for (int e = tid; e < WCT * WCT; e += WNT) {
            const int r = T * WCT + (e % WCT), c = C * WCT + (e / WCT);
            if (r < N && c <= r) G[(size_t)c * N + r] = 0;
          }
      __syncthreads();
      for (int p = tid; p < n; p += WNT) {
        double blk[36];
        for (int k = 0; k < 36; ++k) blk[k] = 0;
        if (p < P.s) {
          const double* J = P.J + (size_t)6 * p * P.m;
          for (int a = 0; a < 6; ++a)
            for (int b = 0; b <= a; ++b)
              for (int k = 0; k < P.m; ++k) blk[a * 6 + b] += J[(size_t)a * P.m + k] * J[(size_t)b * P.m + k];
        }
        for (int64_t e = D.inc_off[p0 + p]; e < D.inc_off[p0 + p + 1]; ++e) {
          const int32_t code = D.inc[e];
          const double* J = D.fac + FS * (int64_t)(code >> 1) + ((code & 1) ? 42 : 6);
          for (int a = 0; a < 6; ++a)
            for (int b = 0; b <= a; ++b)
              for (int k = 0; k < 6; ++k) blk[a * 6 + b] += J[k * 6 + a] * J[k * 6 + b];
        }
        for (int a = 0; a < 6; ++a)
          for (int b = 0; b <= a; ++b)
            G[(size_t)(6 * p + b) * N + 6 * p + a] = blk[a * 6 + b] / (sc[6 * p + a] * sc[6 * p + b]);
      }
      for (int64_t f = f0 + tid; f < f1; f += WNT) {
        const int i = (int)D.rel_ij[2 * f], j = (int)D.rel_ij[2 * f + 1];
        const double* Ji = D.fac + FS * f + 6;
        const double* Jj = D.fac + FS * f + 42;
        for (int a = 0; a < 6; ++a)
          for (int b = 0; b < 6; ++b) {
            double v = 0;
            for (int k = 0; k < 6; ++k) v += Ji[k * 6 + a] * Jj[k * 6 + b];
            v /= sc[6 * i + a] * sc[6 * j + b];
            const int row = i > j ? 6 * i + a : 6 * j + b, col = i > j ? 6 * j + b : 6 * i + a;
            atomicAdd(&G[(size_t)col * N + row], v);
          }
      }
      // the prior's blocks between its poses q < p (none for the anchor)
      for (int e = tid; e < 18 * P.s * (P.s - 1); e += WNT) {
        const int pq = e / 36, ab = e % 36, a = ab / 6, b = ab % 6;
        int p = 1, q = pq;
        while (q >= p) q -= p++;
        double v = 0;
        for (int k = 0; k < P.m; ++k) v += P.J[(size_t)(6 * p + a) * P.m + k] * P.J[(size_t)(6 * q + b) * P.m + k];
        v /= sc[6 * p + a] * sc[6 * q + b];
        atomicAdd(&G[(size_t)(6 * q + b) * N + 6 * p + a], v);
      }
      __syncthreads();
      const bool undamped = stalled;
      tried_undamped = tried_undamped || undamped;
      double growth = 2.0;
      bool accepted = false;
      for (unsigned t = 0; t < O.max_trials; ++t) {
        rep.attempts += 1;
        const double damping = undamped ? 0.0 : lambda;
        rep.damping = damping;
        int rejection = 0;
        // solve_damped: (G + damping I) z = -g / D, delta = z / D.
        for (int T = 0; T < nT; ++T)
          for (int C = cmin[T]; C <= T; ++C)
            for (int e = tid; e < WCT * WCT; e += WNT) {
              const int r = T * WCT + (e % WCT), c = C * WCT + (e / WCT);
              if (r < N && c <= r) {
                const size_t k = (size_t)c * N + r;
                F[k] = (TF)(G[k] + (r == c ? damping : 0.0));
              }
            }
        for (int c = tid; c < N; c += WNT) dv[c] = -g[c] / sc[c];
        if (tid == 0) S.flag = 0;
        __syncthreads();
        bool ok = cta_cholesky<TF, CB>(F, N, N, csm, &S.flag, cmin);
        __syncthreads();
        if (ok) {
          if (std::is_same<TF, double>::value) {
            cta_llt_solve<TF, CB>(F, N, N, reinterpret_cast<TF*>(dv), csm, cmin);
          } else {
            // FP32 factor, FP64 refinement: z += F^-1 (b - (G + damping I) z)
            // until the FP64 residual is below 1e-14 |b| or O.refine passes.
            double bn = 0;
            for (int c = tid; c < N; c += WNT) {
              wv[c] = dv[c];
              bn += dv[c] * dv[c];
              dv[c] = 0;
            }
            bn = wsum(bn, S.red);
            for (int it = 0; it <= O.refine; ++it) {
              for (int c = tid; c < N; c += WNT) tv[c] = (TF)wv[c];
              __syncthreads();
              cta_llt_solve<TF, CB>(F, N, N, tv, csm, cmin);
              for (int c = tid; c < N; c += WNT) dv[c] += (double)tv[c];
              __syncthreads();
              // Residual from the factor Jacobians: G z = D^-1 J^T (J (D^-1 z)).
              for (int64_t f = f0 + tid; f < f1; f += WNT) {
                const int i = (int)D.rel_ij[2 * f], j = (int)D.rel_ij[2 * f + 1];
                double* o = D.fac + FS * f;
                for (int a = 0; a < 6; ++a) {
                  double u = 0;
                  for (int k = 0; k < 6; ++k)
                    u += o[6 + a * 6 + k] * dv[6 * i + k] / sc[6 * i + k] + o[42 + a * 6 + k] * dv[6 * j + k] / sc[6 * j + k];
                  o[78 + a] = u;
                }
              }
              if (tid == 0)
                for (int a = 0; a < P.m; ++a) {
                  double u = 0;
                  for (int k = 0; k < 6 * P.s; ++k) u += P.J[(size_t)k * P.m + a] * dv[k] / sc[k];
                  P.u[a] = u;
                }
              __syncthreads();
              double rn = 0;
              for (int p = tid; p < n; p += WNT) {
                double y[6] = {0, 0, 0, 0, 0, 0};
                if (p < P.s)
                  for (int c = 0; c < 6; ++c)
                    for (int k = 0; k < P.m; ++k) y[c] += P.J[(size_t)(6 * p + c) * P.m + k] * P.u[k];
                for (int64_t e = D.inc_off[p0 + p]; e < D.inc_off[p0 + p + 1]; ++e) {
                  const int32_t code = D.inc[e];
                  const double* o = D.fac + FS * (int64_t)(code >> 1);
                  const double* J = o + ((code & 1) ? 42 : 6);
                  for (int c = 0; c < 6; ++c)
                    for (int k = 0; k < 6; ++k) y[c] += J[k * 6 + c] * o[78 + k];
                }
                for (int c = 0; c < 6; ++c) {
                  const int r = 6 * p + c;
                  const double s = -g[r] / sc[r] - damping * dv[r] - y[c] / sc[r];
                  wv[r] = s;
                  rn += s * s;
                }
              }
              rn = wsum(rn, S.red);
              if (!(rn > 1e-28 * bn)) break;
            }
          }
          // delta, prediction -g.d - |J d|^2 / 2 (DenseSchur::solve_damped + verify_step)
          double gd = 0, fin = 0, smax = 0;
          for (int c = tid; c < N; c += WNT) {
            const double d = dv[c] / sc[c];
            dv[c] = d;
            if (!isfinite(d)) fin = 1;
            smax = fmax(smax, fabs(d));
            gd += g[c] * d;
          }
          __syncthreads();
          double jd = 0;
          for (int64_t f = f0 + tid; f < f1; f += WNT) {
            const int i = (int)D.rel_ij[2 * f], j = (int)D.rel_ij[2 * f + 1];
            const double* Ji = D.fac + FS * f + 6;
            const double* Jj = D.fac + FS * f + 42;
            for (int a = 0; a < 6; ++a) {
              double u = 0;
              for (int k = 0; k < 6; ++k) u += Ji[a * 6 + k] * dv[6 * i + k] + Jj[a * 6 + k] * dv[6 * j + k];
              jd += u * u;
            }
          }
          if (tid == 0)
            for (int a = 0; a < P.m; ++a) {
              double u = 0;
              for (int k = 0; k < 6 * P.s; ++k) u += P.J[(size_t)k * P.m + a] * dv[k];
              jd += u * u;
            }
          gd = wsum(gd, S.red);
          jd = wsum(jd, S.red);
          fin = wmax(fin, S.red);
          smax = wmax(smax, S.red);
          const double predicted = -gd - 0.5 * jd;
          if (fin != 0 || !isfinite(predicted)) {
            rejection = 1;
          } else {
            rep.step_norm = smax;
            if (!(predicted > 0)) {
              rejection = 2;
            } else {
              // Stage x (+) delta and evaluate the trial cost.
              for (int p = tid; p < n; p += WNT)
                store_pose(se3_compose(load_pose(X + 7 * p), se3_exp(dv + 6 * p)), XT + 7 * p);
              __syncthreads();
              rep.cost_evaluations += 1;
              const double value = window_cost(D, w, XT, S.red, &bad);
              if (bad) {
                rejection = 3;
              } else {
                const double actual = current - value;
                const double ratio = fmin(actual / predicted, 2.0);
                if (actual > 0 && ratio >= O.acceptance_threshold) {
                  for (int e = tid; e < 7 * n; e += WNT) X[e] = XT[e];
                  __syncthreads();
                  rep.iterations += 1;
                  stalled = O.step_tolerance > 0 && smax <= O.step_tolerance &&
                            (O.cost_tolerance == 0 || actual / fmax(current, 1.0) <= O.cost_tolerance);
                  current = value;
                  const double cc = 2.0 * fmin(ratio, 1.0) - 1.0;
                  const double update = fmax(1.0 - cc * cc * cc, 1.0 / 3.0);
                  lambda = fmin(fmax(lambda * update, O.min_damping), O.max_damping);
                  accepted = true;
                  break;
                }
                rejection = 4;
              }
            }
          }
        } else {
          rejection = 1;
        }
        rep.rejected_steps += 1;
        rep.last_rejection = rejection;
        if (undamped || lambda == O.max_damping) break;
        lambda = fmin(lambda * growth, O.max_damping);
        growth = fmin(growth * 2.0, fmax(O.max_damping, 2.0));
      }
      if (!accepted) status = FG_NO_PROGRESS;
    }
    rep.final_cost = current;
    rep.status = status;
    rep.termination = term;
    // ---- square-root elimination of the oldest poses (marginalization.rs:458-513)
    int pstatus = FG_OK;
    const int removed = min(O.removed, n);
    if (removed > 0 && (status == FG_OK || status == FG_NO_PROGRESS || status == FG_NO_CONVERGENCE)) {
      const int64_t m0 = D.mf_off[w], m1 = D.mf_off[w + 1];
      const int64_t s0 = D.sep_off[w];
      const int nsep = (int)(D.sep_off[w + 1] - s0);
      const WinPrior P = win_prior(D, w);
      const int m = P.m + 6 * (int)(m1 - m0);
      const int ncol = 6 * (removed + nsep), width = ncol + 1;
      for (int64_t e = tid; e < (int64_t)m * width; e += WNT) M[e] = 0;
      const bool pok = prior_terms(P, X, true, S.red);  // r and J of the prior at the final estimate
      auto column = [&](int p) -> int {
        if (p < removed) return 6 * p;
        for (int s = 0; s < nsep; ++s)
          if ((int)D.sep[s0 + s] == p) return 6 * (removed + s);
        return -1;
      };
      double mbad = 0;
      for (int k = tid; k <= (int)(m1 - m0); k += WNT) {
        double r[6], Ji[36], Jj[36];
        const int base = P.m + 6 * (k - 1);
        if (k == 0) {  // the prior's rows first (its emission comes first)
          if (!pok) {
            mbad = 1;
            continue;
          }
          for (int i = 0; i < P.s; ++i) {
            const int ci = column(i);
            if (ci < 0) {
              mbad = 1;
              break;
            }
            for (int a = 0; a < P.m; ++a)
              for (int b = 0; b < 6; ++b) M[(size_t)(ci + b) * m + a] = P.J[(size_t)(6 * i + b) * P.m + a];
          }
          for (int a = 0; a < P.m; ++a) M[(size_t)ncol * m + a] = P.r[a];
        } else {
          const int64_t f = D.mf[m0 + k - 1];
          if (!rel_eval(D, f, X, r, Ji, Jj)) {
            mbad = 1;
            continue;
          }
          const int ci = column((int)D.rel_ij[2 * f]), cj = column((int)D.rel_ij[2 * f + 1]);
          if (ci < 0 || cj < 0) {
            mbad = 1;
            continue;
          }
          for (int a = 0; a < 6; ++a) {
            for (int b = 0; b < 6; ++b) {
              M[(size_t)(ci + b) * m + base + a] += Ji[a * 6 + b];
              M[(size_t)(cj + b) * m + base + a] += Jj[a * 6 + b];
            }
            M[(size_t)ncol * m + base + a] = r[a];
          }
        }
      }
      if (wmax(mbad, S.red) != 0) {
        pstatus = FG_INVALID_EVALUATION;
      } else {
        const int rem = 6 * removed, sepc = 6 * nsep;
        cta_qr(M, m, width, 0, 0, rem, qperm, qnorms, S.red, &S.flag);
        const double tol = 2.220446049250313e-16 * (double)max(max(m, rem), 1);
        const double scale = (m > 0 && rem > 0) ? fabs(M[0]) : 0.0;
        int rank = 0;
        while (rank < min(m, rem) && fabs(M[(size_t)rank * m + rank]) > scale * tol) ++rank;
        cta_qr(M, m, width, rank, rem, sepc, qperm, qnorms, S.red, &S.flag);
        const int rows = min(m - rank, sepc);
        double* A = D.prior_a + D.a_off[w];
        double* b = D.prior_b + 6 * s0;
        for (int e = tid; e < rows * sepc; e += WNT) A[e] = 0;
        __syncthreads();
        for (int e = tid; e < rows * sepc; e += WNT) {
          const int row = e % rows, col = e / rows;
          if (col >= row) A[(size_t)qperm[col] * rows + row] = M[(size_t)(rem + col) * m + rank + row];
        }
        for (int row = tid; row < rows; row += WNT) b[row] = M[(size_t)ncol * m + rank + row];
        double cst = 0, nf = 0;
        for (int row = rank + rows + tid; row < m; row += WNT) {
          const double r = M[(size_t)ncol * m + row];
          cst += (0.5 * r) * r;
        }
        for (int e = tid; e < rows * sepc; e += WNT)
          if (!isfinite(M[(size_t)(rem + e / rows) * m + rank + e % rows])) nf = 1;
        for (int i = tid; i < min(m, rem); i += WNT)
          if (!isfinite(M[(size_t)i * m + i])) nf = 1;
        cst = wsum(cst, S.red);
        nf = wmax(nf, S.red);
        if (nf != 0 || !isfinite(cst)) pstatus = FG_INVALID_EVALUATION;
        rep.prior_rows = rows;
        rep.eliminated_rank = rank;
        rep.prior_constant = cst;
        rep.separator_poses = nsep;
      }
    }
    rep.prior_status = pstatus;
    if (tid == 0) D.reports[w] = rep;
    __syncthreads();
  }
}

// ------------------------------------------------------------ host side
struct WindowsImpl {
  int dev = 0;
  cudaStream_t st = nullptr;
  int precision = FG_PRECISION_F64;
  size_t W = 0, P = 0, R = 0;
  int removed = 10;
  std::vector<int64_t> pose_off, rel_off, sep_off, a_off, mf_off, inc_off, tile_off;
  std::vector<int32_t> tile_cmin;
  std::vector<uint32_t> rel_ij, sep;
  std::vector<int32_t> inc, mf, order;
  // window priors (default: the anchor on pose 0): poses s and rows m per
  // window, A (m x 6s column-major), b (m), references (7 per prior pose)
  std::vector<int32_t> ps, pm;
  std::vector<int64_t> pr_aoff, pr_boff, pr_roff, pf_off;
  std::vector<double> prA, prb, pref;
  bool custom_priors = false;
  int nmax = 0;
  size_t mcap = 0;
  DBuf<int64_t> d_pose_off, d_rel_off, d_inc_off, d_mf_off, d_sep_off, d_a_off, d_tile_off;
  DBuf<int32_t> d_tile_cmin;
  DBuf<uint32_t> d_rel_ij, d_sep, d_queue;
  DBuf<int32_t> d_inc, d_mf, d_order, d_pr_s, d_pr_m;
  DBuf<int64_t> d_pr_aoff, d_pr_boff, d_pr_roff, d_pf_off;
  DBuf<double> d_prA, d_prb, d_pref;
  DBuf<double> d_x, d_xt, d_prior, d_rel_z, d_fac, d_pfac, d_pa, d_pb, d_G, d_M, d_V;
  DBuf<unsigned char> d_F, d_TV;
  DBuf<fg_window_report> d_reports;
  // autotuned launch
  int variant = -1, ctas_per_sm = 1;
  double tuned_ms[4] = {0, 0, 0, 0};
  int slots = 0;
  // The tuned launch (queue reset + persistent kernel) as a CUDA graph,
  // re-captured when the options change.
  cudaGraphExec_t graph = nullptr;
  WinOptions graph_opts{};
  ~WindowsImpl() {
    if (graph) cudaGraphExecDestroy(graph);
  }

  size_t smem_bytes(int cb) const {
    const size_t tf = precision == FG_PRECISION_F64 ? 8 : 4;
    const size_t chol = ((size_t)cb * (cb + 1) + 2 * (size_t)WCT * (cb + 1)) * tf;
    const size_t qr = ((size_t)nmax + 8) * 8 + (size_t)nmax * 4;
    return std::max(chol, qr) + 64;
  }
};

namespace {
// Raise the dynamic shared-memory cap of every variant once per handle
// (outside any stream capture).
template <class TF, int CB, int MINB>
fg_status prime_variant() {
  FG_CUDA(cudaFuncSetAttribute(k_windows<TF, CB, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 110 * 1024));
  return FG_OK;
}
template <class TF>
fg_status prime_all() {
  FG_TRY((prime_variant<TF, 32, 1>()));
  FG_TRY((prime_variant<TF, 32, 2>()));
  FG_TRY((prime_variant<TF, 16, 2>()));
  FG_TRY((prime_variant<TF, 16, 3>()));
  return FG_OK;
}
template <class TF, int CB, int MINB>
fg_status launch_variant(WindowsImpl& h, const WinDev& D, const WinOptions& O, int grid) {
  FG_LAUNCH((k_windows<TF, CB, MINB>), grid, WNT, h.smem_bytes(CB), h.st, D, O);
  return FG_OK;
}
// Variants: 0 = panel 32 / 1 CTA per SM, 1 = 32 / 2, 2 = 16 / 2, 3 = 16 / 3
// (register budgets follow the CTAs per SM).
template <class TF>
fg_status launch_tf(WindowsImpl& h, int variant, const WinDev& D, const WinOptions& O, int grid) {
  switch (variant) {
    case 0: return launch_variant<TF, 32, 1>(h, D, O, grid);
    case 1: return launch_variant<TF, 32, 2>(h, D, O, grid);
    case 2: return launch_variant<TF, 16, 2>(h, D, O, grid);
    default: return launch_variant<TF, 16, 3>(h, D, O, grid);
  }
}
fg_status launch(WindowsImpl& h, int variant, const WinDev& D, const WinOptions& O, int grid) {
  return h.precision == FG_PRECISION_F64 ? launch_tf<double>(h, variant, D, O, grid)
                                         : launch_tf<float>(h, variant, D, O, grid);
}
}  // namespace

}  // namespace fg

using namespace fg;

struct fg_windows {
  WindowsImpl impl;
};

namespace {
fg_status windows_view(WindowsImpl& h, const fg_optimize_options& o, const fg_lm_options& lo, WinDev* D,
                       WinOptions* O) {
  if (o.max_iterations == 0 || !std::isfinite(o.gradient_tolerance) || o.gradient_tolerance < 0 ||
      !std::isfinite(o.step_tolerance) || o.step_tolerance < 0 || !std::isfinite(o.cost_tolerance) ||
      o.cost_tolerance < 0) {
    set_error("invalid optimize options");
    return FG_INVALID_OPTIONS;
  }
  const double v[5] = {lo.initial_damping, lo.min_damping, lo.max_damping, lo.min_column_norm,
                       lo.acceptance_threshold};
  for (double x : v)
    if (!std::isfinite(x) || x <= 0) {
      set_error("invalid LM options");
      return FG_INVALID_OPTIONS;
    }
  if (lo.max_trials == 0 || lo.min_damping > lo.initial_damping || lo.initial_damping > lo.max_damping ||
      lo.acceptance_threshold >= 1) {
    set_error("invalid LM options");
    return FG_INVALID_OPTIONS;
  }
  O->gradient_tolerance = o.gradient_tolerance;
  O->step_tolerance = o.step_tolerance;
  O->cost_tolerance = o.cost_tolerance;
  O->initial_damping = lo.initial_damping;
  O->min_damping = lo.min_damping;
  O->max_damping = lo.max_damping;
  O->min_column_norm = lo.min_column_norm;
  O->acceptance_threshold = lo.acceptance_threshold;
  O->max_iterations = (unsigned)std::min<size_t>(o.max_iterations, 0xffffffffu);
  O->max_trials = (unsigned)std::min<size_t>(lo.max_trials, 0xffffffffu);
  O->removed = h.removed;
  O->refine = 8;
  WinDev d{};
  d.W = (int)h.W;
  d.pose_off = h.d_pose_off.get();
  d.rel_off = h.d_rel_off.get();
  d.rel_ij = h.d_rel_ij.get();
  d.rel_z = h.d_rel_z.get();
  d.pr_s = h.d_pr_s.get();
  d.pr_m = h.d_pr_m.get();
  d.pr_aoff = h.d_pr_aoff.get();
  d.pr_boff = h.d_pr_boff.get();
  d.pr_roff = h.d_pr_roff.get();
  d.pf_off = h.d_pf_off.get();
  d.pr_A = h.d_prA.get();
  d.pr_b = h.d_prb.get();
  d.pr_ref = h.custom_priors ? h.d_pref.get() : h.d_prior.get();
  d.x = h.d_x.get();
  d.xt = h.d_xt.get();
  d.inc_off = h.d_inc_off.get();
  d.inc = h.d_inc.get();
  d.fac = h.d_fac.get();
  d.pfac = h.d_pfac.get();
  d.mf_off = h.d_mf_off.get();
  d.mf = h.d_mf.get();
  d.sep_off = h.d_sep_off.get();
  d.sep = h.d_sep.get();
  d.a_off = h.d_a_off.get();
  d.tile_off = h.d_tile_off.get();
  d.tile_cmin = h.d_tile_cmin.get();
  d.prior_a = h.d_pa.get();
  d.prior_b = h.d_pb.get();
  d.reports = h.d_reports.get();
  d.order = h.d_order.get();
  d.queue = h.d_queue.get();
  d.G = h.d_G.get();
  d.F = h.d_F.get();
  d.M = h.d_M.get();
  d.g_stride = (size_t)h.nmax * h.nmax;
  d.m_stride = h.mcap;
  d.nmax = h.nmax;
  *D = d;
  return FG_OK;
}

// Per-slot workspace for `slots` concurrent CTAs.
fg_status ensure_slots(WindowsImpl& h, int slots) {
  if (slots <= h.slots) return FG_OK;
  const size_t g = (size_t)h.nmax * h.nmax;
  const size_t tf = h.precision == FG_PRECISION_F64 ? 8 : 4;
  FG_TRY(h.d_G.resize(std::max<size_t>(g * slots, 1)));
  FG_TRY(h.d_F.resize(std::max<size_t>(g * slots * tf, 1)));
  FG_TRY(h.d_M.resize(std::max<size_t>(h.mcap * slots, 1)));
  FG_TRY(h.d_V.resize(std::max<size_t>(4 * (size_t)h.nmax * slots, 1)));
  FG_TRY(h.d_TV.resize(std::max<size_t>((size_t)h.nmax * slots * tf, 1)));
  h.slots = slots;
  return FG_OK;
}

// One persistent launch over the first `windows` scheduled windows.
fg_status run_once(WindowsImpl& h, int variant, int per_sm, const WinDev& D0, const WinOptions& O, int windows,
                   float* ms) {
  const int sms = sm_count(h.dev);
  const int grid = std::max(1, std::min<int>(sms * per_sm, windows));
  FG_TRY(ensure_slots(h, grid));
  WinDev D = D0;
  D.W = windows;
  D.G = h.d_G.get();
  D.F = h.d_F.get();
  D.M = h.d_M.get();
  D.V = h.d_V.get();
  D.TV = h.d_TV.get();
  EventTimer t;
  if (ms) t.start(h.st);
  FG_CUDA(cudaMemsetAsync(h.d_queue.get(), 0, sizeof(unsigned), h.st));
  FG_TRY(launch(h, variant, D, O, grid));
  if (ms) *ms = (float)(t.stop(h.st) * 1e3);
  return FG_OK;
}

fg_status run_graph(WindowsImpl& h, const WinDev& D, const WinOptions& O) {
  if (h.graph && std::memcmp(&h.graph_opts, &O, sizeof(WinOptions)) != 0) {
    cudaGraphExecDestroy(h.graph);
    h.graph = nullptr;
  }
  if (!h.graph) {
    // Size the workspace before capture so no allocation happens inside it.
    const int grid = std::max(1, std::min<int>(sm_count(h.dev) * h.ctas_per_sm, (int)h.W));
    FG_TRY(ensure_slots(h, grid));
    cudaGraph_t g = nullptr;
    uint64_t before = g_launches.load();
    FG_CUDA(cudaStreamBeginCapture(h.st, cudaStreamCaptureModeThreadLocal));
    fg_status s = run_once(h, h.variant, h.ctas_per_sm, D, O, (int)h.W, nullptr);
    cudaError_t e = cudaStreamEndCapture(h.st, &g);
    g_launches.fetch_sub(g_launches.load() - before);
    if (s != FG_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    FG_CUDA(e);
    e = cudaGraphInstantiate(&h.graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      h.graph = nullptr;
      return cuda_status(e, "cudaGraphInstantiate");
    }
    h.graph_opts = O;
  }
  FG_CUDA(cudaGraphLaunch(h.graph, h.st));
  g_launches.fetch_add(1);
  return FG_OK;
}
}  // namespace

namespace {
// The per-window structure that depends on the factors and the window
// priors: incidence, the factors and separator of each elimination (the
// prior touches its poses [0, s), pose 0 among the removed ones), the
// normal-matrix envelope (the prior couples its poses densely) and the prior
// scratch; uploaded to the device.
fg_status plan_windows(WindowsImpl& h) {
  const size_t W = h.W;
  fg_status s = FG_OK;
  cudaStream_t st = h.st;
  // Validate factors, build incidence and the marginalization structure.
  std::vector<int64_t> cnt(h.P + 1, 0);
  h.mf_off.assign(W + 1, 0);
  h.sep_off.assign(W + 1, 0);
  h.a_off.assign(W + 1, 0);
  h.nmax = 0;
  h.mcap = 1;
  std::vector<int32_t> mf;
  std::vector<uint32_t> sep;
  for (size_t w = 0; w < W; ++w) {
    const int64_t n = h.pose_off[w + 1] - h.pose_off[w];
    if (6 * n > 6 * 4096) {
      set_error("windows hold at most 4096 poses");
      return FG_UNSUPPORTED_STRUCTURE;
    }
    h.nmax = std::max<int>(h.nmax, (int)(6 * n));
    const int rm = (int)std::min<int64_t>(h.removed, n);
    if (h.ps[w] > n) {
      set_error("a window prior covers more poses than its window holds");
      return FG_DIMENSION_MISMATCH;
    }
    std::vector<char> touched(n, 0);
    // the prior touches its poses [0, s); pose 0 is among the removed ones
    if (rm > 0)
      for (int k = 0; k < h.ps[w]; ++k) touched[k] = 1;
    std::vector<std::pair<uint32_t, uint32_t>> pairs;
    int64_t nmf = 0;
    for (int64_t f = h.rel_off[w]; f < h.rel_off[w + 1]; ++f) {
      const uint32_t i = h.rel_ij[2 * f], j = h.rel_ij[2 * f + 1];
      if (i >= (uint64_t)n || j >= (uint64_t)n) {
        set_error("relative factor pose index outside its window");
        return FG_DIMENSION_MISMATCH;
      }
      if (i == j) {
        set_error("relative factor between a pose and itself");
        return FG_UNSUPPORTED_STRUCTURE;
      }
      cnt[h.pose_off[w] + i + 1]++;
      cnt[h.pose_off[w] + j + 1]++;
      if ((int)i < rm || (int)j < rm) {
        mf.push_back((int32_t)f);
        ++nmf;
        touched[i] = touched[j] = 1;
      }
    }
    for (int64_t k = rm; k < n; ++k)
      if (touched[k]) sep.push_back((uint32_t)k);
    h.mf_off[w + 1] = (int64_t)mf.size();
    h.sep_off[w + 1] = (int64_t)sep.size();
    const int64_t nsep = h.sep_off[w + 1] - h.sep_off[w];
    h.a_off[w + 1] = h.a_off[w] + 36 * nsep * nsep;
    const size_t m = (size_t)h.pm[w] + 6 * (size_t)nmf, width = 6 * ((size_t)rm + (size_t)nsep) + 1;
    h.mcap = std::max(h.mcap, m * width);
    if (width - 1 > (size_t)6 * 4096) {
      set_error("marginalization system too wide");
      return FG_UNSUPPORTED_STRUCTURE;
    }
  }
  // Envelope of each window's normal matrix: row block p starts at pose
  // env[p] = min(p, lowest neighbour); per 64-row tile, its first 64-column tile.
  h.tile_off.assign(W + 1, 0);
  h.tile_cmin.clear();
  for (size_t w = 0; w < W; ++w) {
    const int64_t n = h.pose_off[w + 1] - h.pose_off[w], N = 6 * n;
    std::vector<int64_t> env(n);
    for (int64_t p = 0; p < n; ++p) env[p] = p < h.ps[w] ? 0 : p;  // the prior couples [0, s) densely
    for (int64_t f = h.rel_off[w]; f < h.rel_off[w + 1]; ++f) {
      const int64_t i = h.rel_ij[2 * f], j = h.rel_ij[2 * f + 1];
      const int64_t hi = std::max(i, j), lo = std::min(i, j);
      env[hi] = std::min(env[hi], lo);
    }
    const int64_t nT = (N + 63) / 64;
    for (int64_t T = 0; T < nT; ++T) {
      int64_t first = T * 64;
      for (int64_t r = T * 64; r < std::min(N, T * 64 + 64); ++r) first = std::min(first, 6 * env[r / 6]);
      h.tile_cmin.push_back((int32_t)(first / 64));
    }
    h.tile_off[w + 1] = (int64_t)h.tile_cmin.size();
  }
  for (size_t p = 0; p < h.P; ++p) cnt[p + 1] += cnt[p];
  h.inc_off = cnt;
  h.inc.assign(std::max<int64_t>(cnt[h.P], 1), 0);
  {
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (size_t w = 0; w < W; ++w)
      for (int64_t f = h.rel_off[w]; f < h.rel_off[w + 1]; ++f) {
        const uint32_t i = h.rel_ij[2 * f], j = h.rel_ij[2 * f + 1];
        h.inc[fill[h.pose_off[w] + i]++] = (int32_t)(f << 1);
        h.inc[fill[h.pose_off[w] + j]++] = (int32_t)((f << 1) | 1);
      }
  }
  if (h.R > (1u << 30)) {
    set_error("too many relative factors");
    return FG_UNSUPPORTED_STRUCTURE;
  }
  h.mf = mf;
  h.sep = sep;
  h.order.resize(W);
  std::iota(h.order.begin(), h.order.end(), 0);
  std::stable_sort(h.order.begin(), h.order.end(), [&](int a, int b) {
    return h.pose_off[a + 1] - h.pose_off[a] > h.pose_off[b + 1] - h.pose_off[b];
  });
  if ((s = upload(h.d_pose_off, h.pose_off.data(), h.pose_off.size(), st))) return s;
  if ((s = upload(h.d_rel_off, h.rel_off.data(), h.rel_off.size(), st))) return s;
  std::vector<uint32_t> ij = h.rel_ij;
  if (ij.empty()) ij.assign(2, 0);
  if ((s = upload(h.d_rel_ij, ij.data(), ij.size(), st))) return s;
  if ((s = upload(h.d_inc_off, h.inc_off.data(), h.inc_off.size(), st))) return s;
  if ((s = upload(h.d_inc, h.inc.data(), h.inc.size(), st))) return s;
  if ((s = upload(h.d_mf_off, h.mf_off.data(), h.mf_off.size(), st))) return s;
  std::vector<int32_t> mfv = h.mf;
  if (mfv.empty()) mfv.push_back(0);
  if ((s = upload(h.d_mf, mfv.data(), mfv.size(), st))) return s;
  if ((s = upload(h.d_sep_off, h.sep_off.data(), h.sep_off.size(), st))) return s;
  std::vector<uint32_t> sv = h.sep;
  if (sv.empty()) sv.push_back(0);
  if ((s = upload(h.d_sep, sv.data(), sv.size(), st))) return s;
  if ((s = upload(h.d_a_off, h.a_off.data(), h.a_off.size(), st))) return s;
  if ((s = upload(h.d_tile_off, h.tile_off.data(), h.tile_off.size(), st))) return s;
  std::vector<int32_t> tc = h.tile_cmin;
  if (tc.empty()) tc.push_back(0);
  if ((s = upload(h.d_tile_cmin, tc.data(), tc.size(), st))) return s;
  std::vector<int32_t> ord = h.order;
  if (ord.empty()) ord.push_back(0);
  if ((s = upload(h.d_order, ord.data(), ord.size(), st))) return s;
  // the window priors: shapes, data, scratch offsets
  h.pr_aoff.assign(W + 1, 0);
  h.pr_boff.assign(W + 1, 0);
  h.pr_roff.assign(W + 1, 0);
  h.pf_off.assign(W + 1, 0);
  for (size_t w = 0; w < W; ++w) {
  const int64_t ps = h.ps[w], pm = h.pm[w];
  h.pr_aoff[w + 1] = h.pr_aoff[w] + pm * 6 * ps;
  h.pr_boff[w + 1] = h.pr_boff[w] + pm;
  h.pr_roff[w + 1] = h.pr_roff[w] + ps;
  h.pf_off[w + 1] = h.pf_off[w] + pm + pm * 6 * ps + pm + 6 * ps + 36 * ps;
  }
  auto pad_i = [](std::vector<int32_t> v) {
    if (v.empty()) v.push_back(0);
    return v;
  };
  auto pad_d = [](std::vector<double> v) {
    if (v.empty()) v.push_back(0);
    return v;
  };
  const std::vector<int32_t> psv = pad_i(h.ps), pmv = pad_i(h.pm);
  const std::vector<double> pav = pad_d(h.prA), pbv = pad_d(h.prb), prv = pad_d(h.pref);
  if ((s = upload(h.d_pr_s, psv.data(), psv.size(), st))) return s;
  if ((s = upload(h.d_pr_m, pmv.data(), pmv.size(), st))) return s;
  if ((s = upload(h.d_pr_aoff, h.pr_aoff.data(), W + 1, st))) return s;
  if ((s = upload(h.d_pr_boff, h.pr_boff.data(), W + 1, st))) return s;
  if ((s = upload(h.d_pr_roff, h.pr_roff.data(), W + 1, st))) return s;
  if ((s = upload(h.d_pf_off, h.pf_off.data(), W + 1, st))) return s;
  if ((s = upload(h.d_prA, pav.data(), pav.size(), st))) return s;
  if ((s = upload(h.d_prb, pbv.data(), pbv.size(), st))) return s;
  if (h.custom_priors && (s = upload(h.d_pref, prv.data(), prv.size(), st))) return s;
  if ((s = h.d_pfac.resize(std::max<int64_t>(h.pf_off[W], 1)))) return s;
  if ((s = h.d_pa.resize(std::max<int64_t>(h.a_off[W], 1)))) return s;
  if ((s = h.d_pb.resize(std::max<int64_t>(6 * h.sep_off[W], 1)))) return s;
  h.slots = 0;  // the marginalization workspace (mcap) may have grown
  if (h.graph) {
  cudaGraphExecDestroy(h.graph);
  h.graph = nullptr;
  }
  FG_CUDA(cudaStreamSynchronize(st));
  return FG_OK;
}
}  // namespace

FG_API fg_status fg_windows_create(size_t windows, const uint64_t* pose_offset, const uint64_t* rel_offset,
                                   const uint32_t* rel_ij, size_t removed_poses, int precision, int device,
                                   fg_windows** out) {
  if (!out) return FG_NULL_ARGUMENT;
  *out = nullptr;
  if (windows && (!pose_offset || !rel_offset)) return FG_NULL_ARGUMENT;
  if (precision != FG_PRECISION_F64 && precision != FG_PRECISION_F32_REFINED) {
    set_error("unknown precision");
    return FG_INVALID_OPTIONS;
  }
  try {
    auto* H = new fg_windows();
    WindowsImpl& h = H->impl;
    auto fail = [&](fg_status s) {
      delete H;
      return s;
    };
    h.dev = device;
    h.precision = precision;
    h.W = windows;
    h.removed = (int)std::min<size_t>(removed_poses, 1u << 20);
    fg_status s = device_stream(device, &h.st);
    if (s) return fail(s);
    h.pose_off.assign(pose_offset, pose_offset + windows + 1);
    h.rel_off.assign(rel_offset, rel_offset + windows + 1);
    if (h.pose_off[0] != 0 || h.rel_off[0] != 0) {
      set_error("window offsets must start at 0");
      return fail(FG_DIMENSION_MISMATCH);
    }
    for (size_t w = 0; w < windows; ++w) {
      if (h.pose_off[w + 1] <= h.pose_off[w] || h.rel_off[w + 1] < h.rel_off[w]) {
        set_error("every window needs at least one pose and nondecreasing offsets");
        return fail(FG_DIMENSION_MISMATCH);
      }
    }
    h.P = (size_t)h.pose_off[windows];
    h.R = (size_t)h.rel_off[windows];
    if (h.R && !rel_ij) return fail(FG_NULL_ARGUMENT);
    h.rel_ij.assign(rel_ij, rel_ij + 2 * h.R);
    // default window priors: the anchor PosePrior on pose 0 (s = 1, A = I, b = 0)
    h.ps.assign(windows, 1);
    h.pm.assign(windows, 6);
    h.prA.assign(36 * windows, 0.0);
    h.prb.assign(6 * windows, 0.0);
    for (size_t w = 0; w < windows; ++w)
      for (int k = 0; k < 6; ++k) h.prA[36 * w + 7 * k] = 1.0;
    h.custom_priors = false;
    if ((s = plan_windows(h))) return fail(s);
    cudaStream_t st = h.st;
    if ((s = h.d_queue.resize(1))) return fail(s);
    if ((s = h.d_x.resize(std::max<size_t>(7 * h.P, 1)))) return fail(s);
    if ((s = h.d_xt.resize(std::max<size_t>(7 * h.P, 1)))) return fail(s);
    if ((s = h.d_prior.resize(std::max<size_t>(7 * windows, 1)))) return fail(s);
    if ((s = h.d_rel_z.resize(std::max<size_t>(7 * h.R, 1)))) return fail(s);
    if ((s = h.d_fac.resize(std::max<size_t>(FS * h.R, 1)))) return fail(s);
    if ((s = h.d_reports.resize(std::max<size_t>(windows, 1)))) return fail(s);
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(cuda_status(cudaGetLastError(), "create"));
    *out = H;
    return FG_OK;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return FG_OUT_OF_MEMORY;
  }
}

FG_API void fg_windows_destroy(fg_windows* h) { delete h; }

FG_API fg_status fg_windows_prior_layout(const fg_windows* H, uint64_t* separator_offset, uint64_t* a_offset,
                                         uint32_t* separators) {
  if (!H) return FG_NULL_ARGUMENT;
  const WindowsImpl& h = H->impl;
  for (size_t w = 0; w <= h.W; ++w) {
    if (separator_offset) separator_offset[w] = (uint64_t)h.sep_off[w];
    if (a_offset) a_offset[w] = (uint64_t)h.a_off[w];
  }
  if (separators) std::copy(h.sep.begin(), h.sep.end(), separators);
  return FG_OK;
}

FG_API fg_status fg_windows_set_priors(fg_windows* H, const uint32_t* prior_poses, const uint32_t* prior_rows,
                                       const double* A, const double* b, const double* refs) {
  if (!H) return FG_NULL_ARGUMENT;
  WindowsImpl& h = H->impl;
  if (h.W && (!prior_poses || !prior_rows || !A || !b || !refs)) return FG_NULL_ARGUMENT;
  try {
    std::vector<int32_t> ps(h.W), pm(h.W);
    size_t na = 0, nb = 0, nr = 0;
    for (size_t w = 0; w < h.W; ++w) {
      const int64_t n = h.pose_off[w + 1] - h.pose_off[w];
      if (prior_poses[w] < 1 || prior_poses[w] > (uint32_t)PR_MAX_POSES || prior_poses[w] > n) {
        set_error("a window prior covers 1 to min(64, window poses) poses");
        return FG_DIMENSION_MISMATCH;
      }
      if (prior_rows[w] < 1 || prior_rows[w] > (uint32_t)PR_MAX_ROWS) {
        set_error("a window prior has 1 to 384 rows");
        return FG_DIMENSION_MISMATCH;
      }
      ps[w] = (int32_t)prior_poses[w];
      pm[w] = (int32_t)prior_rows[w];
      na += (size_t)pm[w] * 6 * ps[w];
      nb += (size_t)pm[w];
      nr += 7 * (size_t)ps[w];
    }
    for (size_t k = 0; k < na; ++k)
      if (!std::isfinite(A[k])) {
        set_error("nonfinite window prior matrix");
        return FG_INVALID_EVALUATION;
      }
    for (size_t k = 0; k < nb; ++k)
      if (!std::isfinite(b[k])) {
        set_error("nonfinite window prior vector");
        return FG_INVALID_EVALUATION;
      }
    FG_TRY(select_device(h.dev));
    // keep the current priors until the new plan is known to be valid
    auto keep_ps = h.ps, keep_pm = h.pm;
    auto keep_a = h.prA, keep_b = h.prb, keep_r = h.pref;
    const bool keep_custom = h.custom_priors;
    h.ps = ps;
    h.pm = pm;
    h.prA.assign(A, A + na);
    h.prb.assign(b, b + nb);
    h.pref.assign(refs, refs + nr);
    h.custom_priors = true;
    fg_status s = plan_windows(h);
    if (s != FG_OK) {
      h.ps = keep_ps;
      h.pm = keep_pm;
      h.prA = keep_a;
      h.prb = keep_b;
      h.pref = keep_r;
      h.custom_priors = keep_custom;
      const fg_status s2 = plan_windows(h);
      return s2 != FG_OK ? s2 : s;
    }
    return FG_OK;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return FG_OUT_OF_MEMORY;
  }
}

FG_API fg_status fg_windows_upload(fg_windows* H, const double* poses, const double* priors, const double* rel_z) {
  if (!H || (H->impl.P && !poses) || (H->impl.W && !priors) || (H->impl.R && !rel_z)) return FG_NULL_ARGUMENT;
  WindowsImpl& h = H->impl;
  FG_TRY(select_device(h.dev));
  if (h.P) FG_CUDA(cudaMemcpyAsync(h.d_x.get(), poses, 7 * h.P * sizeof(double), cudaMemcpyHostToDevice, h.st));
  if (h.W)
    FG_CUDA(cudaMemcpyAsync(h.d_prior.get(), priors, 7 * h.W * sizeof(double), cudaMemcpyHostToDevice, h.st));
  if (h.R)
    FG_CUDA(cudaMemcpyAsync(h.d_rel_z.get(), rel_z, 7 * h.R * sizeof(double), cudaMemcpyHostToDevice, h.st));
  FG_CUDA(cudaStreamSynchronize(h.st));
  return FG_OK;
}

FG_API fg_status fg_windows_run(fg_windows* H, const fg_optimize_options* o, const fg_lm_options* lo) {
  if (!H || !o || !lo) return FG_NULL_ARGUMENT;
  WindowsImpl& h = H->impl;
  if (h.W == 0) return FG_OK;
  FG_TRY(select_device(h.dev));
  WinDev D;
  WinOptions O;
  FG_TRY(windows_view(h, *o, *lo, &D, &O));
  if (h.smem_bytes(32) > 100 * 1024) {
    set_error("window too large for the shared-memory working set");
    return FG_UNSUPPORTED_STRUCTURE;
  }
  if (h.variant < 0) {
    FG_TRY(prime_all<double>());
    FG_TRY(prime_all<float>());
    // Autotune on the largest scheduled windows (a sample of at most four
    // CTAs' worth per SM): time each (panel width, CTAs per SM) schedule once,
    // keep the fastest and restore the poses the sample moved.
    const int sample = std::min<int>((int)h.W, 4 * sm_count(h.dev));
    DBuf<double> saved;
    FG_TRY(saved.resize(std::max<size_t>(7 * h.P, 1)));
    FG_CUDA(cudaMemcpyAsync(saved.get(), h.d_x.get(), 7 * h.P * sizeof(double), cudaMemcpyDeviceToDevice, h.st));
    const int per_sm[4] = {1, 2, 2, 3};
    const int panel[4] = {32, 32, 16, 16};
    int best = 0;
    float best_ms = 0;
    for (int c = 0; c < 4; ++c) {
      const size_t sm = h.smem_bytes(panel[c]) + 2048;
      if ((size_t)per_sm[c] * sm > 220 * 1024) continue;
      float ms = 0;
      FG_CUDA(cudaMemcpyAsync(h.d_x.get(), saved.get(), 7 * h.P * sizeof(double), cudaMemcpyDeviceToDevice, h.st));
      FG_TRY(run_once(h, c, per_sm[c], D, O, sample, &ms));
      h.tuned_ms[c] = ms;
      if (best_ms == 0 || ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
    FG_CUDA(cudaMemcpyAsync(h.d_x.get(), saved.get(), 7 * h.P * sizeof(double), cudaMemcpyDeviceToDevice, h.st));
    FG_CUDA(cudaStreamSynchronize(h.st));
    h.variant = best;
    h.ctas_per_sm = per_sm[best];
  }
  return run_graph(h, D, O);
}

FG_API fg_status fg_windows_download(fg_windows* H, double* poses, fg_window_report* reports, double* prior_a,
                                     double* prior_b) {
  if (!H) return FG_NULL_ARGUMENT;
  WindowsImpl& h = H->impl;
  FG_TRY(select_device(h.dev));
  if (poses && h.P)
    FG_CUDA(cudaMemcpyAsync(poses, h.d_x.get(), 7 * h.P * sizeof(double), cudaMemcpyDeviceToHost, h.st));
  if (reports && h.W)
    FG_CUDA(cudaMemcpyAsync(reports, h.d_reports.get(), h.W * sizeof(fg_window_report), cudaMemcpyDeviceToHost,
                            h.st));
  if (prior_a && h.a_off[h.W])
    FG_CUDA(cudaMemcpyAsync(prior_a, h.d_pa.get(), h.a_off[h.W] * sizeof(double), cudaMemcpyDeviceToHost, h.st));
  if (prior_b && h.sep_off[h.W])
    FG_CUDA(cudaMemcpyAsync(prior_b, h.d_pb.get(), 6 * h.sep_off[h.W] * sizeof(double), cudaMemcpyDeviceToHost,
                            h.st));
  FG_CUDA(cudaStreamSynchronize(h.st));
  return FG_OK;
}

FG_API fg_status fg_windows_solve(fg_windows* H, double* poses, const double* priors, const double* rel_z,
                                  const fg_optimize_options* o, const fg_lm_options* lo, fg_window_report* reports,
                                  double* prior_a, double* prior_b) {
  FG_TRY(fg_windows_upload(H, poses, priors, rel_z));
  FG_TRY(fg_windows_run(H, o, lo));
  return fg_windows_download(H, poses, reports, prior_a, prior_b);
}

FG_API fg_status fg_windows_tuning(const fg_windows* H, int* panel, int* ctas_per_sm, double* ms4) {
  if (!H) return FG_NULL_ARGUMENT;
  const WindowsImpl& h = H->impl;
  if (panel) *panel = h.variant < 0 ? 0 : (h.variant < 2 ? 32 : 16);
  if (ctas_per_sm) *ctas_per_sm = h.ctas_per_sm;
  if (ms4)
    for (int k = 0; k < 4; ++k) ms4[k] = h.tuned_ms[k];
  return FG_OK;
}

FG_API fg_status fg_windows_stream(const fg_windows* H, void** stream) {
  if (!H || !stream) return FG_NULL_ARGUMENT;
  *stream = (void*)H->impl.st;
  return FG_OK;
}
