// Device kernels of the LSMR backend (fagra src/lsmr.rs over the block-sparse
// LinearizedModel of src/linear_model.rs).
//
// One LSMR iteration on A M, with A = [J D^-1; sqrt(lambda) I] (or
// [J; sqrt(lambda) D] unscaled) and M the block-Jacobi right preconditioner
// (src/lsmr/preconditioner.rs: M = L^-T per variable block), is three kernels:
//   k_lsmr_rows      u <- A M v - alpha u over the emission rows (J w) and the
//                    bottom rows (one per column), beta = ||u|| by last-block
//                    reduction
//   k_lsmr_segments  v <- M^T A^T u / beta - beta v per column segment,
//                    alpha = ||v||; the last block runs the scalar recurrences
//   k_lsmr_update    v /= alpha, the hbar / y / h updates and w = M v (/ D)
// Every scalar lives in LsmrState on the device, so a CUDA graph of several
// iterations replays with no host round trip.
//
// Data layout (int64 indices):
//   emissions  e_row[E+1] first row of each emission (rows = e_row[e+1]-e_row[e]),
//              e_blk[E+1] block range, e_val[E] value index of the emission's first
//              block; blocks b_col[nb], b_cols[nb]. An emission's values are
//              contiguous, block after block, each block column-major.
//   segments   s_col[S+1] column ranges partitioning [0, n) (width <= 32);
//              s_pc[S+1] CSR into pieces; a piece is the part of one block lying
//              in the segment: p_start (value index of its first column), p_row,
//              p_rows. Pieces keep emission order inside a segment.
//   Segments with many pieces (s_wide) get a CTA each, the rest a thread each.
#pragma once
#include "common.cuh"
#include "kernels.cuh"

namespace fg {

struct LsmrState {
  double alpha, beta, beta_next;  // normalizers of the stored raw v and u
  double alphabar, rho, rhobar, cbar, sbar, zetabar;
  double c_hbar, c_y, c_h;  // vector-update coefficients of the current iteration
  double normar, normar0, threshold, tolerance, root;
  unsigned long long min_scale_bits, max_scale_bits;  // positive doubles: ordered as integers
  int stop, upd, termination, nonfinite_scales;
  unsigned iterations, max_iterations;
  unsigned counter0, counter1, counter2, counter3;
  unsigned trips;  // loop trips of the single-launch solve graph (k_lsmr_continue)
};

struct LsmrVerify {
  double jd2, nr2, g2, gd, snr2, sg2;
  int nonfinite_step;
  unsigned counter0, counter1, pad;
};

template <class TS>
struct LsmrDev {
  const TS* values;
  int64_t m, n;
  int64_t E;
  const int64_t *e_row, *e_blk, *e_val, *b_col;
  const int32_t* b_cols;
  int64_t S;
  const int64_t *s_col, *s_pc, *p_start, *p_row;
  const int32_t* p_rows;
  const int32_t *s_wide, *s_narrow;
  int32_t n_wide, n_narrow;
  const double* factors;  // per segment: w*w lower Cholesky factor, column-major
  const int64_t* s_fac;   // factor offset per segment; -1 = identity
  const double* scales;   // null = unscaled operator
  // 1: the device BAL layout — emission e has rows 2e, 2e+1, blocks 2e (camera,
  // 2x9) and 2e+1 (point, 2x3), values [24e, 24e + 24), and every segment is
  // one whole block — so rows and pieces are read with 16-byte loads and the
  // row / row count of a piece follow from its start.
  int bal;
  // BAL: the point pieces' 6 values copied contiguously, in piece order from
  // piece pp0 on (null until copied for the current linearization)
  const TS* ptvals;
  int64_t pp0;
};

// ptvals[6 i + k] = values[p_start[pp0 + i] + k], the point halves of the BAL
// emissions in the segment pass's piece order (one pass per linearization).
template <class TS>
__global__ void k_lsmr_point_copy(int64_t npp, int64_t pp0, const int64_t* p_start, const TS* values, TS* ptvals) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= npp) return;
  const int64_t start = p_start[pp0 + i];
#pragma unroll
  for (int k = 0; k < 6; ++k) ptvals[6 * i + k] = values[start + k];
}

// n contiguous values at p into double (p 16-byte aligned when n is a
// multiple of 4 / 2 for float / double, 8-byte aligned otherwise).
template <int N>
__device__ __forceinline__ void load_vals(const float* p, double (&v)[N]) {
  if (N % 4 == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
#pragma unroll
    for (int i = 0; i < N / 4; ++i) {
      const float4 a = reinterpret_cast<const float4*>(p)[i];
      v[4 * i] = a.x; v[4 * i + 1] = a.y; v[4 * i + 2] = a.z; v[4 * i + 3] = a.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      const float2 a = reinterpret_cast<const float2*>(p)[i];
      v[2 * i] = a.x; v[2 * i + 1] = a.y;
    }
  }
}
template <int N>
__device__ __forceinline__ void load_vals(const double* p, double (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N / 2; ++i) {
    const double2 a = reinterpret_cast<const double2*>(p)[i];
    v[2 * i] = a.x; v[2 * i + 1] = a.y;
  }
}

// load_vals through the read-only path (the values do not change during a pass).
template <int N>
__device__ __forceinline__ void load_vals_ro(const float* p, double (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N / 4; ++i) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p) + i);
    v[4 * i] = a.x; v[4 * i + 1] = a.y; v[4 * i + 2] = a.z; v[4 * i + 3] = a.w;
  }
}
template <int N>
__device__ __forceinline__ void load_vals_ro(const double* p, double (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N / 2; ++i) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p) + i);
    v[2 * i] = a.x; v[2 * i + 1] = a.y;
  }
}

// emission_rows for the BAL layout, with the same summation order.
template <class TS, class F>
__device__ __forceinline__ void emission_rows_bal(const LsmrDev<TS>& D, int64_t e, const double* w, F f) {
  double v[24];
  load_vals<24>(D.values + 24 * e, v);
  const double* wc = w + D.b_col[2 * e];
  const double* wp = w + D.b_col[2 * e + 1];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double acc = 0;
#pragma unroll
    for (int j = 0; j < 9; ++j) acc += v[2 * j + i] * wc[j];
#pragma unroll
    for (int j = 0; j < 3; ++j) acc += v[18 + 2 * j + i] * wp[j];
    f(2 * e + i, acc);
  }
}

constexpr int LSMR_NT = 256;          // threads per block
constexpr int LSMR_WIDE_DEGREE = 48;  // pieces above which a segment gets a CTA
constexpr int LSMR_MAX_WIDTH = 32;    // widest segment

__device__ __forceinline__ double lsmr_inv(double x) { return x > 0 ? 1.0 / x : 0.0; }

// J rows of one emission times w; calls f(row, value) per row.
template <class TS, class F>
__device__ __forceinline__ void emission_rows(const LsmrDev<TS>& D, int64_t e, const double* w, F f) {
  const int64_t r0 = D.e_row[e], rows = D.e_row[e + 1] - r0;
  const int64_t b0 = D.e_blk[e], b1 = D.e_blk[e + 1];
  for (int64_t i = 0; i < rows; ++i) {
    double acc = 0;
    int64_t vs = D.e_val[e];
    for (int64_t b = b0; b < b1; ++b) {
      const int64_t col = D.b_col[b];
      const int cols = D.b_cols[b];
      const TS* v = D.values + vs + i;
      for (int j = 0; j < cols; ++j) acc += (double)v[(int64_t)j * rows] * w[col + j];
      vs += (int64_t)cols * rows;
    }
    f(r0 + i, acc);
  }
}

enum { ROWS_ITER = 0, ROWS_VERIFY = 1, ROWS_START = 2, ROWS_PRODUCT = 3 };

// Row pass. ITER: u <- A M v - alpha u with ||u||^2 (bottom rows included);
// VERIFY: pr = J d - negres with ||J d||^2; START: u = negres, ||u||^2;
// PRODUCT: pr = J w and ub = sqrt(lambda) D w (the Damped operator alone).
// Grid: [emission blocks | bottom-column blocks (ITER and PRODUCT)].
template <class TS, int MODE>
__global__ void __launch_bounds__(LSMR_NT) k_lsmr_rows(LsmrDev<TS> D, unsigned emission_blocks, const double* w,
                                                        TS* u, double* ub, const double* negres, double* pr,
                                                        double* partials, LsmrState* st, LsmrVerify* vs) {
  if (MODE == ROWS_ITER && st->stop) return;
  double f = 0, root = 0;
  if (MODE == ROWS_ITER) f = st->alpha * lsmr_inv(st->beta);
  if (MODE == ROWS_ITER || MODE == ROWS_PRODUCT) root = st->root;
  double sq[1] = {0.0};
  if (blockIdx.x < emission_blocks) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < D.E) {
      if (MODE == ROWS_START) {
        for (int64_t r = D.e_row[e]; r < D.e_row[e + 1]; ++r) {
          double x = negres[r];
          u[r] = (TS)x;
          sq[0] += x * x;
        }
      } else {
        auto body = [&](int64_t r, double acc) {
          if (MODE == ROWS_ITER) {
            double x = acc - f * (double)u[r];
            u[r] = (TS)x;
            sq[0] += x * x;
          } else if (MODE == ROWS_PRODUCT) {
            pr[r] = acc;
          } else {
            pr[r] = acc - negres[r];
            sq[0] += acc * acc;
          }
        };
        if (D.bal) emission_rows_bal(D, e, w, body);
        else emission_rows(D, e, w, body);
      }
    }
  } else if (MODE == ROWS_ITER || MODE == ROWS_PRODUCT) {
    int64_t j = (blockIdx.x - emission_blocks) * (int64_t)blockDim.x + threadIdx.x;
    if (j < D.n) {
      double s = D.scales ? D.scales[j] : 1.0;
      double x = root * s * w[j];
      if (MODE == ROWS_ITER) x -= f * ub[j];
      ub[j] = x;
      sq[0] += x * x;
    }
  }
  if (MODE == ROWS_PRODUCT) return;
  block_sums<1>(sq);
  if (threadIdx.x == 0) partials[blockIdx.x] = sq[0];
  unsigned* counter = MODE == ROWS_VERIFY ? &vs->counter0 : &st->counter0;
  if (arrive_last(counter)) {
    double tot[1];
    finish_sums<1>(partials, tot);
    if (threadIdx.x == 0) {
      if (MODE == ROWS_VERIFY) vs->jd2 = tot[0];
      else st->beta_next = sqrt(tot[0]);
      *counter = 0;
    }
  }
}

// ---------------------------------------------------------------- segments
// acc[j] += sum over this thread's share of the segment's pieces of
// J(:, j)^T vec (or of J(:, j)^2 with SQUARES).
template <class TS, int MAXW, bool SQUARES, class V>
__device__ __forceinline__ void segment_accumulate(const LsmrDev<TS>& D, int64_t s, int w, int64_t first,
                                                   int64_t stride, const V* vec, double (&acc)[MAXW]) {
  const int64_t p1 = D.s_pc[s + 1];
  if (D.bal && (w == 9 || w == 3) && MAXW >= 9) {
    // camera piece: 18 values at 24e; point piece: 6 values at 24e + 18; rows 2e, 2e + 1
    for (int64_t p = D.s_pc[s] + first; p < p1; p += stride) {
      const int64_t start = D.p_start[p], row = 2 * (start / 24);
      const double x0 = SQUARES ? 0.0 : (double)vec[row], x1 = SQUARES ? 0.0 : (double)vec[row + 1];
      double a[18];
      if (w == 9) {
        load_vals<18>(D.values + start, a);
      } else {
        double b[6];
        load_vals<6>(D.ptvals ? D.ptvals + 6 * (p - D.pp0) : D.values + start, b);
#pragma unroll
        for (int k = 0; k < 6; ++k) a[k] = b[k];
      }
#pragma unroll
      for (int j = 0; j < (MAXW < 9 ? MAXW : 9); ++j) {
        if (j < w) {
          acc[j] += SQUARES ? a[2 * j] * a[2 * j] : a[2 * j] * x0;
          acc[j] += SQUARES ? a[2 * j + 1] * a[2 * j + 1] : a[2 * j + 1] * x1;
        }
      }
    }
    return;
  }
  for (int64_t p = D.s_pc[s] + first; p < p1; p += stride) {
    const int64_t start = D.p_start[p], row = D.p_row[p];
    const int rows = D.p_rows[p];
    for (int i = 0; i < rows; ++i) {
      const double x = SQUARES ? 0.0 : (double)vec[row + i];
#pragma unroll
      for (int j = 0; j < MAXW; ++j) {
        if (j < w) {
          const double a = (double)D.values[start + (int64_t)j * rows + i];
          acc[j] += SQUARES ? a * a : a * x;
        }
      }
    }
  }
}

// q <- L^-1 q (forward substitution) with L the column-major w x w lower factor.
template <int MAXW>
__device__ __forceinline__ void lower_solve(const double* fac, int w, double (&q)[MAXW]) {
#pragma unroll
  for (int i = 0; i < MAXW; ++i) {
    if (i < w) {
      double s = q[i];
#pragma unroll
      for (int k = 0; k < MAXW; ++k)
        if (k < i) s -= fac[k * w + i] * q[k];
      q[i] = s / fac[i * w + i];
    }
  }
}
// q <- L^-T q (back substitution on L^T).
template <int MAXW>
__device__ __forceinline__ void upper_t_solve(const double* fac, int w, double (&q)[MAXW]) {
#pragma unroll
  for (int ii = MAXW - 1; ii >= 0; --ii) {
    if (ii < w) {
      double s = q[ii];
#pragma unroll
      for (int k = 0; k < MAXW; ++k)
        if (k > ii && k < w) s -= fac[ii * w + k] * q[k];
      q[ii] = s / fac[ii * w + ii];
    }
  }
}

enum { SEG_ITER = 0, SEG_START = 1, SEG_VERIFY = 2, SEG_SQUARES = 3, SEG_GRADIENT = 4, SEG_PRODUCT = 5 };
constexpr int SEG_K = 6;  // partial sums per block

struct SegArgs {
  const void* vec;     // u (TS) for ITER/START, pr (double) for VERIFY, negres for GRADIENT, y for PRODUCT
  const double* ub;    // bottom rows of u (ITER/START/PRODUCT)
  double* v;           // LSMR v (ITER/START): normalized on entry, raw on exit
  const double* step;  // VERIFY: the step in original coordinates
  const double* grad;  // VERIFY: the gradient J^T r
  double* out;         // SQUARES: scales; GRADIENT: gradient; PRODUCT: A^T y
  double lambda, floor;
  int scaled;          // D^-1 scaling active (non-identity modes)
};

// Finalization of one segment from its column sums; adds into part[].
template <class TS, int MAXW, int MODE>
__device__ __forceinline__ void segment_finish(const LsmrDev<TS>& D, int64_t s, int w, double (&acc)[MAXW],
                                               const SegArgs& a, const LsmrState* st, double (&part)[SEG_K],
                                               double& mn, double& mx) {
  const int64_t c0 = D.s_col[s];
  const int64_t fo = D.s_fac ? D.s_fac[s] : -1;
  if (MODE == SEG_ITER || MODE == SEG_START) {
    const double beta = st->beta_next, ib = lsmr_inv(beta), root = st->root;
#pragma unroll
    for (int j = 0; j < MAXW; ++j) {
      if (j < w) {
        const double sc = D.scales ? D.scales[c0 + j] : 1.0;
        const double ts = a.scaled ? 1.0 / sc : 1.0, td = a.scaled ? root : root * sc;
        acc[j] = (acc[j] * ts + td * a.ub[c0 + j]) * ib;
      }
    }
    if (fo >= 0) lower_solve<MAXW>(D.factors + fo, w, acc);
#pragma unroll
    for (int j = 0; j < MAXW; ++j) {
      if (j < w) {
        const double x = acc[j] - beta * a.v[c0 + j];
        a.v[c0 + j] = x;
        part[0] += x * x;
      }
    }
  } else if (MODE == SEG_VERIFY) {
    double g[MAXW];
#pragma unroll
    for (int j = 0; j < MAXW; ++j) {
      if (j < w) {
        const double sc = D.scales[c0 + j], d = a.step[c0 + j];
        if (!isfinite(d)) part[5] = 1.0;
        acc[j] += (a.lambda * (sc * d)) * sc;  // src/linear_model.rs:270-273
        g[j] = a.grad[c0 + j];
        part[0] += acc[j] * acc[j];
        part[1] += g[j] * g[j];
        part[2] += g[j] * d;
        if (a.scaled) {
          acc[j] /= sc;
          g[j] /= sc;
        }
      } else {
        g[j] = 0;
      }
    }
    if (fo >= 0) {
      lower_solve<MAXW>(D.factors + fo, w, acc);
      lower_solve<MAXW>(D.factors + fo, w, g);
    }
#pragma unroll
    for (int j = 0; j < MAXW; ++j) {
      if (j < w) {
        part[3] += acc[j] * acc[j];
        part[4] += g[j] * g[j];
      }
    }
  } else if (MODE == SEG_SQUARES) {
#pragma unroll
    for (int j = 0; j < MAXW; ++j) {
      if (j < w) {
        double r = sqrt(acc[j]);
        if (!isfinite(r)) part[5] = 1.0;
        r = fmax(r, a.floor);
        a.out[c0 + j] = r;
        mn = fmin(mn, r);
        mx = fmax(mx, r);
      }
    }
  } else if (MODE == SEG_PRODUCT) {  // src/lsmr.rs:200-211 transpose_apply
    const double root = st->root;
#pragma unroll
    for (int j = 0; j < MAXW; ++j) {
      if (j < w) {
        const double sc = D.scales ? D.scales[c0 + j] : 1.0;
        const double ts = a.scaled ? 1.0 / sc : 1.0, td = a.scaled ? root : root * sc;
        a.out[c0 + j] = acc[j] * ts + td * a.ub[c0 + j];
      }
    }
  } else {  // SEG_GRADIENT: g = J^T r = -J^T negres
#pragma unroll
    for (int j = 0; j < MAXW; ++j)
      if (j < w) a.out[c0 + j] = -acc[j];
  }
}

// The end of a segment pass: block sums of the partials, the last block's
// totals, and for ITER / START the scalar recurrences.
template <int MODE>
__device__ __forceinline__ void seg_tail(double (&part)[SEG_K], double* partials, LsmrState* st, LsmrVerify* vs) {
  block_sums<SEG_K>(part);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < SEG_K; ++k) partials[blockIdx.x * SEG_K + k] = part[k];
  unsigned* counter = MODE == SEG_VERIFY ? &vs->counter1 : &st->counter1;
  if (!arrive_last(counter)) return;
  double tot[SEG_K];
  finish_sums<SEG_K>(partials, tot);
  if (threadIdx.x != 0) return;
  *counter = 0;
  if (MODE == SEG_VERIFY) {
    vs->nr2 = tot[0];
    vs->g2 = tot[1];
    vs->gd = tot[2];
    vs->snr2 = tot[3];
    vs->sg2 = tot[4];
    vs->nonfinite_step = tot[5] != 0;
    return;
  }
  // Scalar recurrences (Fong & Saunders, Algorithm 1).
  const double alpha = sqrt(tot[0]), beta = st->beta_next;
  if (MODE == SEG_START) {
    st->alpha = alpha;
    st->beta = beta;
    st->alphabar = alpha;
    st->zetabar = alpha * beta;
    st->rho = 1;
    st->rhobar = 1;
    st->cbar = 1;
    st->sbar = 0;
    st->normar0 = alpha * beta;
    st->normar = st->normar0;
    st->threshold = st->tolerance * st->normar0;
    st->c_hbar = st->c_y = st->c_h = 0;
    st->iterations = 0;
    if (!isfinite(st->normar0)) {
      st->stop = 1;
      st->termination = 4;
    } else if (st->normar0 == 0) {
      st->stop = 1;
      st->termination = 1;
    }
    st->upd = 1;
    return;
  }
  const double rhoold = st->rho;
  const double rho = hypot(st->alphabar, beta);
  const double cs = st->alphabar / rho, sn = beta / rho;
  const double thetanew = sn * alpha;
  st->alphabar = cs * alpha;
  const double rhobarold = st->rhobar;
  const double thetabar = st->sbar * rho;
  const double crho = st->cbar * rho;
  const double rhobar = hypot(crho, thetanew);
  st->cbar = crho / rhobar;
  st->sbar = thetanew / rhobar;
  const double zeta = st->cbar * st->zetabar;
  st->zetabar = -st->sbar * st->zetabar;
  st->c_hbar = thetabar * rho / (rhoold * rhobarold);
  st->c_y = zeta / (rho * rhobar);
  st->c_h = thetanew / rho;
  st->rho = rho;
  st->rhobar = rhobar;
  st->alpha = alpha;
  st->beta = beta;
  st->normar = fabs(st->zetabar);
  st->iterations += 1;
  if (!isfinite(st->normar)) {
    st->stop = 1;
    st->termination = 4;
  } else if (st->iterations >= st->max_iterations) {
    st->stop = 1;
    st->termination = 2;
  } else if (st->normar <= st->threshold) {
    st->stop = 1;
    st->termination = 1;
  }
  st->upd = 1;
}

// Segment pass: blocks [0, n_wide) take one wide segment each with all their
// threads; the remaining blocks take one narrow segment per thread.
template <class TS, int MAXW, int MODE>
__global__ void __launch_bounds__(LSMR_NT) k_lsmr_segments(LsmrDev<TS> D, SegArgs a, double* partials,
                                                            LsmrState* st, LsmrVerify* vs) {
  if ((MODE == SEG_ITER) && st->stop) return;
  constexpr bool SQ = MODE == SEG_SQUARES;
  double part[SEG_K] = {0, 0, 0, 0, 0, 0};
  double mn = INFINITY, mx = 0;
  double acc[MAXW];
#pragma unroll
  for (int j = 0; j < MAXW; ++j) acc[j] = 0;
  if ((int)blockIdx.x < D.n_wide) {
    const int64_t s = D.s_wide[blockIdx.x];
    const int w = (int)(D.s_col[s + 1] - D.s_col[s]);
    if (MODE == SEG_VERIFY || MODE == SEG_GRADIENT || MODE == SEG_PRODUCT)
      segment_accumulate<TS, MAXW, SQ>(D, s, w, threadIdx.x, blockDim.x, (const double*)a.vec, acc);
    else
      segment_accumulate<TS, MAXW, SQ>(D, s, w, threadIdx.x, blockDim.x, (const TS*)a.vec, acc);
    __shared__ double red[LSMR_NT / 32][MAXW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < MAXW; ++j) {
      double x = warp_sum(acc[j]);
      if (lane == 0) red[warp][j] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int j = 0; j < MAXW; ++j) {
        double x = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) x += red[k][j];
        acc[j] = x;
      }
      segment_finish<TS, MAXW, MODE>(D, s, w, acc, a, st, part, mn, mx);
    }
  } else {
    const int64_t idx = (blockIdx.x - D.n_wide) * (int64_t)blockDim.x + threadIdx.x;
    if (idx < D.n_narrow) {
      const int64_t s = D.s_narrow[idx];
      const int w = (int)(D.s_col[s + 1] - D.s_col[s]);
      if (MODE == SEG_VERIFY || MODE == SEG_GRADIENT || MODE == SEG_PRODUCT)
        segment_accumulate<TS, MAXW, SQ>(D, s, w, 0, 1, (const double*)a.vec, acc);
      else
        segment_accumulate<TS, MAXW, SQ>(D, s, w, 0, 1, (const TS*)a.vec, acc);
      segment_finish<TS, MAXW, MODE>(D, s, w, acc, a, st, part, mn, mx);
    }
  }
  if (MODE == SEG_GRADIENT || MODE == SEG_PRODUCT) return;
  if (MODE == SEG_SQUARES) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
      mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
      if (mn < INFINITY) atomicMin(&((LsmrState*)st)->min_scale_bits, (unsigned long long)__double_as_longlong(mn));
      if (mx > 0) atomicMax(&((LsmrState*)st)->max_scale_bits, (unsigned long long)__double_as_longlong(mx));
      if (part[5] != 0) ((LsmrState*)st)->nonfinite_scales = 1;
    }
    return;
  }
  seg_tail<MODE>(part, partials, st, vs);
}

// ------------------------------------------------ fused BAL iteration pass
// For the device BAL layout with camera-major emissions (camera c's emissions
// are one contiguous range, the pieces of camera segment c) the row pass and
// the transposed pass of an ITER step read each emission's 24 values once:
// k_lsmr_fused_rows: one CTA per camera segment: u <- J w - alpha u for the
//   camera's emissions (u written back, ||u||^2), the camera's column sums of
//   J^T u (FP64, threads strided over the emissions, warp then CTA sums, as the
//   wide-segment pass), and each emission's point contribution J_p^T u (3
//   doubles at 3e); the remaining blocks update the bottom rows as k_lsmr_rows.
// k_lsmr_fused_segments: thread per segment: camera sums, or the point's
//   contributions summed in piece order, then segment_finish / seg_tail.
template <class TS>
__global__ void __launch_bounds__(LSMR_NT) k_lsmr_fused_rows(LsmrDev<TS> D, int ncam, const double* w, TS* u,
                                                              double* ub, double* csum, double* pcon,
                                                              double* partials, LsmrState* st) {
  if (st->stop) return;
  const double f = st->alpha * lsmr_inv(st->beta), root = st->root;
  double sq[1] = {0.0};
  if ((int)blockIdx.x < ncam) {
    const int64_t s = blockIdx.x;
    const int64_t p0 = D.s_pc[s], np = D.s_pc[s + 1] - p0;
    const int64_t e0 = np ? D.p_start[p0] / 24 : 0;
    __shared__ double wc[9];
    __shared__ double red[LSMR_NT / 32][9];
    if (threadIdx.x < 9) wc[threadIdx.x] = w[D.s_col[s] + threadIdx.x];
    __syncthreads();
    double acc[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) acc[j] = 0;
    for (int64_t i = threadIdx.x; i < np; i += LSMR_NT) {
      const int64_t e = e0 + i;
      double v[24];
      load_vals_ro<24>(D.values + 24 * e, v);
      const double* wp = w + __ldg(D.b_col + 2 * e + 1);
      const double wp0 = wp[0], wp1 = wp[1], wp2 = wp[2];
      double x[2];
#pragma unroll
      for (int r = 0; r < 2; ++r) {  // emission_rows_bal's summation order
        double a = 0;
#pragma unroll
        for (int j = 0; j < 9; ++j) a += v[2 * j + r] * wc[j];
        a += v[18 + r] * wp0;
        a += v[20 + r] * wp1;
        a += v[22 + r] * wp2;
        const double y = a - f * (double)u[2 * e + r];
        u[2 * e + r] = (TS)y;
        sq[0] += y * y;
        x[r] = (double)(TS)y;  // the transposed pass reads the stored u
      }
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        acc[j] += v[2 * j] * x[0];
        acc[j] += v[2 * j + 1] * x[1];
      }
      double* pc = pcon + 3 * e;
#pragma unroll
      for (int j = 0; j < 3; ++j) pc[j] = v[18 + 2 * j] * x[0] + v[18 + 2 * j + 1] * x[1];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      const double t = warp_sum(acc[j]);
      if (lane == 0) red[warp][j] = t;
    }
    __syncthreads();
    if (threadIdx.x < 9) {
      double t = 0;
      for (int k = 0; k < LSMR_NT / 32; ++k) t += red[k][threadIdx.x];
      csum[9 * s + threadIdx.x] = t;
    }
  } else {
    const int64_t j = (blockIdx.x - ncam) * (int64_t)blockDim.x + threadIdx.x;
    if (j < D.n) {
      const double sc = D.scales ? D.scales[j] : 1.0;
      const double x = root * sc * w[j] - f * ub[j];
      ub[j] = x;
      sq[0] += x * x;
    }
  }
  block_sums<1>(sq);
  if (threadIdx.x == 0) partials[blockIdx.x] = sq[0];
  if (arrive_last(&st->counter0)) {
    double tot[1];
    finish_sums<1>(partials, tot);
    if (threadIdx.x == 0) {
      st->beta_next = sqrt(tot[0]);
      st->counter0 = 0;
    }
  }
}

template <class TS, int MAXW>
__global__ void __launch_bounds__(LSMR_NT) k_lsmr_fused_segments(LsmrDev<TS> D, SegArgs a, int ncam,
                                                                  const double* csum, const double* pcon,
                                                                  double* partials, LsmrState* st) {
  if (st->stop) return;
  double part[SEG_K] = {0, 0, 0, 0, 0, 0};
  double mn = INFINITY, mx = 0;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s < D.S) {
    const int w = (int)(D.s_col[s + 1] - D.s_col[s]);
    double acc[MAXW];
#pragma unroll
    for (int j = 0; j < MAXW; ++j) acc[j] = 0;
    if (s < ncam) {
#pragma unroll
      for (int j = 0; j < (MAXW < 9 ? MAXW : 9); ++j) acc[j] = csum[9 * s + j];
    } else {
      for (int64_t p = D.s_pc[s]; p < D.s_pc[s + 1]; ++p) {
        const double* pc = pcon + 3 * (D.p_start[p] / 24);
#pragma unroll
        for (int j = 0; j < (MAXW < 3 ? MAXW : 3); ++j) acc[j] += pc[j];
      }
    }
    segment_finish<TS, MAXW, SEG_ITER>(D, s, w, acc, a, st, part, mn, mx);
  }
  seg_tail<SEG_ITER>(part, partials, st, nullptr);
}

// v /= alpha; hbar = h - c_hbar hbar; y += c_y hbar; h = v - c_h h; w = M v (/ D).
// RECOVER instead writes step = M y (/ D).
template <class TS, int MAXW, bool RECOVER>
__global__ void __launch_bounds__(LSMR_NT) k_lsmr_update(LsmrDev<TS> D, double* v, double* h, double* hbar,
                                                          double* y, double* w, int scaled, LsmrState* st) {
  if (!RECOVER && !st->upd) return;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s < D.S) {
    const int64_t c0 = D.s_col[s];
    const int wd = (int)(D.s_col[s + 1] - c0);
    const int64_t fo = D.s_fac ? D.s_fac[s] : -1;
    double z[MAXW];
    if (RECOVER) {
#pragma unroll
      for (int j = 0; j < MAXW; ++j) z[j] = j < wd ? y[c0 + j] : 0.0;
    } else {
      const double ia = lsmr_inv(st->alpha), ch = st->c_hbar, cy = st->c_y, chh = st->c_h;
#pragma unroll
      for (int j = 0; j < MAXW; ++j) {
        if (j < wd) {
          const int64_t c = c0 + j;
          const double vj = v[c] * ia;
          v[c] = vj;
          const double hb = h[c] - ch * hbar[c];
          hbar[c] = hb;
          y[c] += cy * hb;
          h[c] = vj - chh * h[c];
          z[j] = vj;
        } else {
          z[j] = 0;
        }
      }
    }
    if (fo >= 0) upper_t_solve<MAXW>(D.factors + fo, wd, z);
#pragma unroll
    for (int j = 0; j < MAXW; ++j)
      if (j < wd) w[c0 + j] = (scaled && D.scales) ? z[j] / D.scales[c0 + j] : z[j];
  }
  if (RECOVER) return;
  if (arrive_last(&st->counter2) && threadIdx.x == 0) {
    st->upd = 0;
    st->counter2 = 0;
  }
}

// BlockFactors::prepare Gram entries (src/linear_model/block_factors.rs:89-107):
// one thread per lower-triangle entry (r >= c) of every variable segment, in
// D-scaled coordinates, summed over the segment's pieces in emission order.
template <class TS>
__global__ void k_lsmr_gram(LsmrDev<TS> D, int64_t nentries, const int64_t* entry_seg, const int32_t* entry_rc,
                            double* gram) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nentries) return;
  const int64_t s = entry_seg[t];
  const int rc = entry_rc[t], c = rc >> 8, r = rc & 255;
  const int64_t c0 = D.s_col[s];
  const int w = (int)(D.s_col[s + 1] - c0);
  const double sc = D.scales[c0 + c], sr = D.scales[c0 + r];
  double sum = 0;
  for (int64_t p = D.s_pc[s]; p < D.s_pc[s + 1]; ++p) {
    const int64_t start = D.p_start[p];
    const int rows = D.p_rows[p];
    double b = 0;
    for (int k = 0; k < rows; ++k)
      b += ((double)D.values[start + (int64_t)c * rows + k] / sc) * ((double)D.values[start + (int64_t)r * rows + k] / sr);
    sum += b;
  }
  gram[D.s_fac[s] + (int64_t)c * w + r] = sum;
}

// BlockFactors::factor (block_factors.rs:113-138): gram + lambda I, in-place
// lower Cholesky; a failed or nonfinite block becomes the identity (s_fac = -1
// in the active offsets) and counts as a fallback.
__global__ void k_lsmr_factor(int64_t S, const int64_t* s_col, const int64_t* gram_off, const double* gram,
                              double lambda, double* factors, int64_t* active, unsigned* fallbacks) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= S) return;
  const int64_t o = gram_off[s];
  if (o < 0) {
    active[s] = -1;
    return;
  }
  const int w = (int)(s_col[s + 1] - s_col[s]);
  double* a = factors + o;
  const double* g = gram + o;
  bool ok = true;
  for (int j = 0; j < w; ++j)
    for (int i = j; i < w; ++i) {
      double x = g[j * w + i] + (i == j ? lambda : 0.0);
      if (!isfinite(x)) ok = false;
      a[j * w + i] = x;
    }
  for (int j = 0; j < w && ok; ++j) {
    double d = a[j * w + j];
    for (int k = 0; k < j; ++k) d -= a[k * w + j] * a[k * w + j];
    if (!(d > 0) || !isfinite(d)) {
      ok = false;
      break;
    }
    d = sqrt(d);
    a[j * w + j] = d;
    for (int i = j + 1; i < w; ++i) {
      double x = a[j * w + i];
      for (int k = 0; k < j; ++k) x -= a[k * w + i] * a[k * w + j];
      a[j * w + i] = x / d;
    }
  }
  active[s] = ok ? o : -1;
  if (!ok) atomicAdd(fallbacks, 1u);
}

}  // namespace fg
