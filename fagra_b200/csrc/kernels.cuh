// Device kernels of the Schur backend. Widths are template parameters for the
// common shapes (BAL 9/3 etc.); CW = 0 / PW = 0 selects runtime widths <= MAXW.
#pragma once
#include "common.cuh"
#include "schur.cuh"

namespace fg {

constexpr int MAXW = 16;
constexpr int NT = 256;  // threads per block for vector kernels

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sums of K doubles; result valid in thread 0.
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K]) {
  __shared__ double sh[32][K];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sh[warp][k] = v[k];
  __syncthreads();
  if (warp == 0) {
    int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double x = lane < nw ? sh[lane][k] : 0.0;
      v[k] = warp_sum(x);
    }
  }
  __syncthreads();
}

// Threadfence reduction: the last block to arrive sees every partial.
__device__ __forceinline__ bool arrive_last(unsigned* counter) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned prev = atomicAdd(counter, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Sums partials[b*K + k] over blocks in fixed order (deterministic); thread 0 result.
template <int K>
__device__ __forceinline__ void finish_sums(const double* partials, double (&out)[K]) {
  double v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += ((volatile const double*)partials)[b * K + k];
  block_sums<K>(v);
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = v[k];
}

// Coordinate -> (variable, offset). Variables: retained 0..nC-1, then eliminated.
struct Layout {
  int64_t retained, dim;
  int32_t cw, pw, nC, nP;
  __device__ __forceinline__ void locate(int64_t j, int64_t* var, int* off) const {
    if (j < retained) {
      *var = j / cw;
      *off = (int)(j % cw);
    } else {
      int64_t k = j - retained;
      *var = nC + k / pw;
      *off = (int)(k % pw);
    }
  }
  __device__ __forceinline__ int width(int64_t var) const { return var < nC ? cw : pw; }
  __device__ __forceinline__ int64_t gram_offset(int64_t var) const {
    return var < nC ? var * (int64_t)cw * cw : (int64_t)nC * cw * cw + (var - nC) * (int64_t)pw * pw;
  }
};

// ---------------------------------------------------------------- model
// g = J^T r with r = -negres (src/linear_model.rs:199-207), per coordinate over
// the variable's blocks in emission order.
template <class TS>
__global__ void k_gradient(Layout L, int64_t j0, const int64_t* var_off, const int64_t* var_blk,
                           const DBlockMeta* blocks, const TS* values, const double* negres, double* g) {
  int64_t j = j0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= L.dim) return;
  int64_t v;
  int off;
  L.locate(j, &v, &off);
  double sum = 0;
  for (int64_t k = var_off[v]; k < var_off[v + 1]; ++k) {
    DBlockMeta b = blocks[var_blk[k]];
    double s = 0;
    const TS* col = values + b.start + (int64_t)off * b.rows;
    for (int i = 0; i < b.rows; ++i) s += (double)col[i] * -negres[b.row + i];
    sum += s;
  }
  g[j] = sum;
}

// Column norms before flooring (src/linear_model.rs:211-224).
template <class TS>
__global__ void k_scales_raw(Layout L, int64_t j0, const int64_t* var_off, const int64_t* var_blk,
                             const DBlockMeta* blocks, const TS* values, double* scales) {
  int64_t j = j0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= L.dim) return;
  int64_t v;
  int off;
  L.locate(j, &v, &off);
  double sum = 0;
  for (int64_t k = var_off[v]; k < var_off[v + 1]; ++k) {
    DBlockMeta b = blocks[var_blk[k]];
    const TS* col = values + b.start + (int64_t)off * b.rows;
    for (int i = 0; i < b.rows; ++i) {
      double x = (double)col[i];
      sum += x * x;
    }
  }
  scales[j] = sqrt(sum);
}

static __global__ void k_floor(int64_t n, double* x, double floor) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < n) x[j] = fmax(x[j], floor);
}

// Infinity norm with a nonfinite flag (src/optimization.rs:653-662).
// out[0] = max |x|, out[1] = 1 if any value is nonfinite.
template <class T>
__global__ void k_norm_inf(int64_t n, const T* x, double* partials, unsigned* counter, double* out) {
  double m = 0, bad = 0;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    double v = (double)x[j];
    if (!isfinite(v)) bad = 1;
    else m = fmax(m, fabs(v));
  }
  // max-reduce via warp shuffles
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    bad = fmax(bad, __shfl_down_sync(0xffffffffu, bad, o));
  }
  __shared__ double sm[32], sb[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { sm[warp] = m; sb[warp] = bad; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int nw = (blockDim.x + 31) >> 5;
    for (int w = 1; w < nw; ++w) { m = fmax(m, sm[w]); bad = fmax(bad, sb[w]); }
    partials[2 * blockIdx.x] = m;
    partials[2 * blockIdx.x + 1] = bad;
  }
  if (arrive_last(counter)) {
    if (threadIdx.x == 0) {
      double M = 0, B = 0;
      for (unsigned b = 0; b < gridDim.x; ++b) {
        M = fmax(M, ((volatile double*)partials)[2 * b]);
        B = fmax(B, ((volatile double*)partials)[2 * b + 1]);
      }
      out[0] = M;
      out[1] = B;
      *counter = 0;
    }
  }
}

// Normalized Gram blocks, lower triangle, column major (block_factors.rs:87-99).
// One thread per (variable, c, r) with r >= c; `first` is the first variable.
template <class TS>
__global__ void k_gram(Layout L, int64_t first, int64_t count, int w, const int64_t* var_off, const int64_t* var_blk,
                       const DBlockMeta* blocks, const TS* values, const double* scales, TS* gram) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t ww = (int64_t)w * w;
  if (t >= count * ww) return;
  int64_t v = first + t / ww;
  int c = (int)((t % ww) / w), r = (int)(t % w);
  int64_t go = L.gram_offset(v);
  if (r < c) return;  // upper triangle untouched (zero)
  double sum = 0;
  for (int64_t k = var_off[v]; k < var_off[v + 1]; ++k) {
    DBlockMeta b = blocks[var_blk[k]];
    const TS* cc = values + b.start + (int64_t)c * b.rows;
    const TS* rr = values + b.start + (int64_t)r * b.rows;
    double dc = scales[b.col + c], dr = scales[b.col + r];
    double s = 0;
    for (int i = 0; i < b.rows; ++i) s += ((double)cc[i] / dc) * ((double)rr[i] / dr);
    sum += s;
  }
  gram[go + (int64_t)c * w + r] = (TS)sum;
}

// Cross blocks E_e[p,c] (src/schur.rs:504-519), layout (e*pw+p)*cw+c.
template <class TS>
__global__ void k_cross(int64_t nedges, int cw, int pw, const DEdgeMeta* edges, const DBlockMeta* blocks,
                        const TS* values, const double* scales, TS* cross) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t per = (int64_t)cw * pw;
  if (t >= nedges * per) return;
  int64_t e = t / per;
  int p = (int)((t % per) / cw), c = (int)(t % cw);
  DEdgeMeta ed = edges[e];
  DBlockMeta l = blocks[ed.lblk], r = blocks[ed.rblk];
  const TS* lc = values + l.start + (int64_t)c * l.rows;
  const TS* rp = values + r.start + (int64_t)p * r.rows;
  double dl = scales[l.col + c], dr = scales[r.col + p];
  double s = 0;
  for (int i = 0; i < l.rows; ++i) s += ((double)lc[i] / dl) * ((double)rp[i] / dr);
  cross[t] = (TS)s;
}

// ------------------------------------------------------------ small dense
template <int W>
__device__ __forceinline__ bool chol_inplace(double* a, int w) {  // column major, lower
  const int n = W ? W : w;
  for (int j = 0; j < n; ++j) {
    double d = a[j * n + j];
    for (int k = 0; k < j; ++k) d -= a[k * n + j] * a[k * n + j];
    if (!(d > 0)) return false;
    d = sqrt(d);
    a[j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double s = a[j * n + i];
      for (int k = 0; k < j; ++k) s -= a[k * n + i] * a[k * n + j];
      a[j * n + i] = s / d;
    }
  }
  return true;
}
// Solve (L L^T) x = b in place; L column major lower in storage type TS.
template <int W, class TS, class TV>
__device__ __forceinline__ void llt_solve(const TS* l, TV* x, int w) {
  const int n = W ? W : w;
  for (int i = 0; i < n; ++i) {
    TV s = x[i];
    for (int k = 0; k < i; ++k) s -= (TV)l[k * n + i] * x[k];
    x[i] = s / (TV)l[i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    TV s = x[i];
    for (int k = i + 1; k < n; ++k) s -= (TV)l[i * n + k] * x[k];
    x[i] = s / (TV)l[i * n + i];
  }
}

// Per-lambda block factorization (block_factors.rs:113-138) for `count`
// variables starting at `first` of width W; unobserved variables are skipped.
template <int W, class TS>
__global__ void k_factor(Layout L, int64_t first, int64_t count, int w_rt, const uint8_t* observed, const TS* gram,
                         TS* factors, double lambda, unsigned* fallbacks) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  int64_t v = first + t;
  if (!observed[v]) return;
  const int w = W ? W : w_rt;
  constexpr int WM = W ? W : MAXW;
  double a[WM * WM];
  int64_t go = L.gram_offset(v);
  bool bad = false;
  for (int c = 0; c < w; ++c)
    for (int r = 0; r < w; ++r) {
      double x = r >= c ? (double)gram[go + c * w + r] : 0.0;
      if (r == c) x += lambda;
      if (!isfinite(x)) bad = true;
      a[c * w + r] = x;
    }
  if (!bad) bad = !chol_inplace<W>(a, w);
  if (!bad)
    for (int j = 0; j < w; ++j)
      if (!isfinite(a[j * w + j]) || a[j * w + j] <= 0) bad = true;
  for (int c = 0; c < w; ++c)
    for (int r = 0; r < w; ++r) factors[go + c * w + r] = (TS)(r >= c ? a[c * w + r] : 0.0);
  if (bad) atomicAdd(fallbacks, 1u);
}

// ---------------------------------------------------------------- vectors
// A retained vector read either directly (pprev == nullptr) or as the PCG
// search direction p = z + beta * p_prev.
template <class TV>
struct PView {
  const TV* z;
  const TV* pprev;
  const double* beta;
  __device__ __forceinline__ TV at(int64_t i, TV b) const { return pprev ? z[i] + b * pprev[i] : z[i]; }
  __device__ __forceinline__ TV beta_value() const { return pprev ? (TV)*beta : (TV)0; }
};

// t_p = C_p^-1 sum_{e in p} E_e^T x_cam (first half of src/schur.rs:626-639).
template <int CW, int PW, class TS, class TV>
__global__ void k_points(Layout L, const int64_t* pt_edge_off, const int64_t* pt_edge, const DEdgeMeta* edges,
                         const TS* cross, const TS* factors, const uint8_t* observed, PView<TV> x, double lambda,
                         TV* t, const int* done) {
  if (done && *done) return;
  int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (pt >= L.nP) return;
  const int cw = CW ? CW : L.cw, pw = PW ? PW : L.pw;
  constexpr int PM = PW ? PW : MAXW;
  TV acc[PM];
  for (int p = 0; p < pw; ++p) acc[p] = 0;
  TV b = x.beta_value();
  for (int64_t k = pt_edge_off[pt]; k < pt_edge_off[pt + 1]; ++k) {
    int64_t e = pt_edge[k];
    int64_t cam = edges[e].cam;
    const TS* E = cross + e * (int64_t)cw * pw;
    TV xc[CW ? CW : MAXW];
    for (int c = 0; c < cw; ++c) xc[c] = x.at(cam * cw + c, b);
    for (int p = 0; p < pw; ++p) {
      TV s = 0;
      for (int c = 0; c < cw; ++c) s += (TV)E[p * cw + c] * xc[c];
      acc[p] += s;
    }
  }
  int64_t v = L.nC + pt;
  if (observed[v]) {
    llt_solve<PW, TS, TV>(factors + L.gram_offset(v), acc, pw);
  } else if (lambda != 0) {
    for (int p = 0; p < pw; ++p) acc[p] /= (TV)lambda;
  }
  for (int p = 0; p < pw; ++p) t[pt * pw + p] = acc[p];
}

// q_c = ax * x_c + [B x]_c - sum_{e in c} E_e t_p (src/schur.rs:608-648), one
// warp per retained variable. Optional: partial x.q into partials and, in the
// last block, alpha = rz / (p.q) with the positive-curvature test of CG.
template <int CW, int PW, class TS, class TV>
__global__ void k_cams(Layout L, const int64_t* cam_edge_off, const int64_t* cam_edge, const DEdgeMeta* edges,
                       const TS* cross, const TV* t, const TS* gram, const uint8_t* observed, PView<TV> x, double ax,
                       int use_gram, TV* q, double* partials, PcgState* st) {
  if (st && st->done) return;
  const int cw = CW ? CW : L.cw, pw = PW ? PW : L.pw;
  constexpr int CM = CW ? CW : MAXW;
  int lane = threadIdx.x & 31;
  int64_t cam = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  double dot = 0;
  if (cam < L.nC) {
    TV acc[CM];
    for (int c = 0; c < cw; ++c) acc[c] = 0;
    for (int64_t k = cam_edge_off[cam] + lane; k < cam_edge_off[cam + 1]; k += 32) {
      int64_t e = cam_edge[k];
      int64_t pt = edges[e].pt;
      const TS* E = cross + e * (int64_t)cw * pw;
      for (int p = 0; p < pw; ++p) {
        TV tp = t[pt * pw + p];
        for (int c = 0; c < cw; ++c) acc[c] += (TV)E[p * cw + c] * tp;
      }
    }
    for (int c = 0; c < cw; ++c) {
      double a = (double)acc[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      acc[c] = (TV)a;
    }
    TV b = x.beta_value();
    if (lane < cw) {
      int c = lane;
      TV xc = x.at(cam * cw + c, b);
      TV v = (TV)ax * xc;
      if (use_gram && observed[cam]) {
        const TS* g = gram + L.gram_offset(cam);
        for (int j = 0; j < cw; ++j) {
          TS gv = j >= c ? g[c * cw + j] : g[j * cw + c];
          v += (TV)gv * x.at(cam * cw + j, b);
        }
      }
      TV accc = acc[0];
      for (int k = 1; k < cw; ++k)
        if (k == c) accc = acc[k];
      v -= accc;
      q[cam * cw + c] = v;
      dot = (double)xc * (double)v;
    }
  }
  if (!partials) return;
  double s[1] = {dot};
  block_sums<1>(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s[0];
  if (arrive_last(&st->counter0)) {
    double tot[1];
    finish_sums<1>(partials, tot);
    if (threadIdx.x == 0) {
      st->pq = tot[0];
      if (!(tot[0] > 0)) {
        st->done = 1;
        st->termination = FG_TERM_NOT_POSITIVE_DEFINITE;
      } else {
        st->alpha = st->rz / tot[0];
      }
      st->counter0 = 0;
    }
  }
}

// Apply the retained block preconditioner z = M^-1 r for one variable.
template <int CW, class TS, class TV>
__device__ __forceinline__ void precondition_one(const TS* pre, bool observed, double lambda, TV* r, int cw) {
  if (observed) {
    llt_solve<CW, TS, TV>(pre, r, cw);
  } else if (lambda != 0) {
    for (int c = 0; c < cw; ++c) r[c] /= (TV)lambda;
  }
}

// PCG update for one retained variable per thread: x += alpha p;
// r -= alpha q; z = M^-1 r; partial r.r and r.z. The last block counts the
// iteration, applies the stopping rules of faer's CG and forms the next
// search direction p = z + beta p.
template <int CW, class TS, class TV>
__global__ void k_update(Layout L, TV* x, TV* r, TV* z, TV* p, const TV* q, const TS* pre,
                         const uint8_t* observed, double lambda, double* partials, PcgState* st) {
  if (st->done) return;
  const int cw = CW ? CW : L.cw;
  constexpr int CM = CW ? CW : MAXW;
  int64_t cam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double rr = 0, rz = 0;
  if (cam < L.nC) {
    TV alpha = (TV)st->alpha;
    TV rv[CM];
    for (int c = 0; c < cw; ++c) {
      int64_t i = cam * cw + c;
      x[i] += alpha * p[i];
      TV ri = r[i] - alpha * q[i];
      r[i] = ri;
      rv[c] = ri;
      rr += (double)ri * (double)ri;
    }
    TV zv[CM];
    for (int c = 0; c < cw; ++c) zv[c] = rv[c];
    precondition_one<CW, TS, TV>(pre + L.gram_offset(cam), observed[cam], lambda, zv, cw);
    for (int c = 0; c < cw; ++c) {
      z[cam * cw + c] = zv[c];
      rz += (double)rv[c] * (double)zv[c];
    }
  }
  double s[2] = {rr, rz};
  block_sums<2>(s);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = s[0];
    partials[2 * blockIdx.x + 1] = s[1];
  }
  if (arrive_last(&st->counter1)) {
    __shared__ int go_on;
    __shared__ double beta_s;
    double tot[2];
    finish_sums<2>(partials, tot);
    if (threadIdx.x == 0) {
      go_on = 0;
      st->iterations += 1;
      st->rr = tot[0];
      double rnorm = sqrt(tot[0]);
      if (rnorm < st->threshold) {
        st->done = 1;
        st->termination = FG_TERM_CONVERGED;
      } else if (!(st->rz > 0)) {
        st->done = 1;
        st->termination = FG_TERM_NOT_POSITIVE_DEFINITE;
      } else if (st->iterations >= st->max_iterations) {
        st->done = 1;
        st->termination = FG_TERM_ITERATION_LIMIT;
      } else {
        st->beta = tot[1] / st->rz;
        st->rz = tot[1];
        beta_s = st->beta;
        go_on = 1;
      }
      st->counter1 = 0;
    }
    __syncthreads();
    if (go_on) {
      TV b = (TV)beta_s;
      int64_t n = (int64_t)L.nC * cw;
      for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        TV zi = ((volatile TV*)z)[i];
        p[i] = zi + b * p[i];
      }
    }
  }
}

// PCG start: r = b, x = 0, p_prev = 0, ||b|| and the threshold.
template <class TV>
__global__ void k_pcg_init(int64_t n, const double* b, TV* x, TV* r, double* partials, PcgState* st,
                           double rel_tol) {
  double s = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    TV bi = (TV)b[i];
    r[i] = bi;
    x[i] = 0;
    s += (double)bi * (double)bi;
  }
  double v[1] = {s};
  block_sums<1>(v);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
  if (arrive_last(&st->counter2)) {
    double tot[1];
    finish_sums<1>(partials, tot);
    if (threadIdx.x == 0) {
      double bn = sqrt(tot[0]);
      st->bnorm = bn;
      st->threshold = rel_tol * bn;
      st->iterations = 0;
      st->beta = 0;
      st->alpha = 0;
      st->rr = tot[0];
      st->termination = FG_TERM_NONE;
      st->done = 0;
      if (bn == 0 || bn < st->threshold) {
        st->done = 1;
        st->termination = FG_TERM_CONVERGED;
      }
      st->counter2 = 0;
    }
  }
}

// z = M^-1 r, p = z and rz = r.z at the start of CG.
template <int CW, class TS, class TV>
__global__ void k_pcg_precond_init(Layout L, const TV* r, TV* z, TV* p, const TS* pre, const uint8_t* observed,
                                   double lambda, double* partials, PcgState* st) {
  if (st->done) return;
  const int cw = CW ? CW : L.cw;
  constexpr int CM = CW ? CW : MAXW;
  int64_t cam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double rz = 0;
  if (cam < L.nC) {
    TV zv[CM];
    for (int c = 0; c < cw; ++c) zv[c] = r[cam * cw + c];
    precondition_one<CW, TS, TV>(pre + L.gram_offset(cam), observed[cam], lambda, zv, cw);
    for (int c = 0; c < cw; ++c) {
      z[cam * cw + c] = zv[c];
      p[cam * cw + c] = zv[c];
      rz += (double)r[cam * cw + c] * (double)zv[c];
    }
  }
  double v[1] = {rz};
  block_sums<1>(v);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
  if (arrive_last(&st->counter2)) {
    double tot[1];
    finish_sums<1>(partials, tot);
    if (threadIdx.x == 0) {
      st->rz = tot[0];
      st->counter2 = 0;
    }
  }
}

}  // namespace fg
