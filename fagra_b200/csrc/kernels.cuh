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
    double M = 0, B = 0;  // thread-strided over the partials, then a block max
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
      M = fmax(M, ((volatile double*)partials)[2 * b]);
      B = fmax(B, ((volatile double*)partials)[2 * b + 1]);
    }
    for (int o = 16; o > 0; o >>= 1) {
      M = fmax(M, __shfl_down_sync(0xffffffffu, M, o));
      B = fmax(B, __shfl_down_sync(0xffffffffu, B, o));
    }
    __syncthreads();
    if (lane == 0) { sm[warp] = M; sb[warp] = B; }
    __syncthreads();
    if (threadIdx.x == 0) {
      int nw = (blockDim.x + 31) >> 5;
      for (int w = 1; w < nw; ++w) { M = fmax(M, sm[w]); B = fmax(B, sb[w]); }
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
                        const TS* values, const double* scales, TS* cross, int* bad) {
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
  if (!isfinite(s)) atomicOr(bad, 1);
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
                         TV* t, const int* done, const int* gate) {
  if (done && *done) return;
  if (gate && !*gate) return;
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
                       int use_gram, TV* q, double* partials, PcgState* st, const int* gate) {
  if (st && st->done) return;
  if (gate && !*gate) return;
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

// ---------------------------------------------------------------- PCG (wide)
// The retained preconditioner is applied through explicit inverses of its
// 9x9 (CW x CW) blocks, Minv = L^-T L^-1 from the block Cholesky factor
// (unobserved variables: I / lambda, as block_factors.rs:193-203), so the
// PCG kernels can run one thread per coordinate.
template <int CW, class TS>
__global__ void k_precond_inverse(Layout L, const uint8_t* observed, const TS* pre, double lambda, TS* minv) {
  int64_t cam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cam >= L.nC) return;
  const int cw = CW ? CW : L.cw;
  constexpr int CM = CW ? CW : MAXW;
  TS* out = minv + cam * (int64_t)cw * cw;
  if (!observed[cam]) {
    double v = lambda != 0 ? 1.0 / lambda : 1.0;
    for (int i = 0; i < cw * cw; ++i) out[i] = (TS)((i % (cw + 1)) == 0 ? v : 0.0);
    return;
  }
  const TS* l = pre + L.gram_offset(cam);  // column major lower
  double m[CM * CM];                        // M = L^-1, column major lower
  for (int j = 0; j < cw; ++j) {
    for (int i = 0; i < cw; ++i) m[j * cw + i] = 0;
    m[j * cw + j] = 1.0 / (double)l[j * cw + j];
    for (int i = j + 1; i < cw; ++i) {
      double s = 0;
      for (int k = j; k < i; ++k) s += (double)l[k * cw + i] * m[j * cw + k];
      m[j * cw + i] = -s / (double)l[i * cw + i];
    }
  }
  for (int i = 0; i < cw; ++i)
    for (int j = i; j < cw; ++j) {
      double s = 0;
      for (int k = j; k < cw; ++k) s += m[i * cw + k] * m[j * cw + k];  // (M^T M)_ij = sum_k M_ki M_kj
      out[i * cw + j] = (TS)s;
      out[j * cw + i] = (TS)s;
    }
}

// PCG update, one thread per retained coordinate, 32 variables per block:
// p = z + beta p; x += alpha p; r -= alpha q; z = Minv r (block local);
// partial r.r and r.z. The last block applies faer's stopping rules and sets
// beta for the next search direction, which its consumers form on the fly.
// XD: the iterate is FP64 (mixed-precision mode) and convergence is deferred
// to an FP64 residual replacement (see k_replace).
// Two-level preconditioning (CO): z = Minv r + W c with c = G W^T r, where
// W (nk <= MAXK rows of length 9C) spans a coarse space and G = (W^T S W)^-1.
// The kernels add the nk partial dots W^T r to their block sums; the last
// block forms c, adds d.c to r.z and leaves c for k_coarse_add, which adds
// W c to z before any consumer reads it.
constexpr int MAXK = 8;
// G staged in shared memory by every thread of the (last) block, so the
// coarse products below read it without one global round trip per entry.
__device__ __forceinline__ const double* stage_coarse(const double* G, int nk) {
  __shared__ double gs[MAXK * MAXK];
  for (int i = threadIdx.x; i < nk * nk; i += blockDim.x) gs[i] = G[i];
  __syncthreads();
  return gs;
}
__device__ __forceinline__ double coarse_finish(const double* G, int nk, const double* d, PcgState* st) {
  double extra = 0;
  for (int i = 0; i < nk; ++i) {
    double c = 0;
    for (int j = 0; j < nk; ++j) c += G[i * nk + j] * d[j];
    st->coarse[i] = c;
    extra += d[i] * c;
  }
  st->coarse_pending = 1;
  return extra;
}

template <int CW, class TS, class TX, bool MIXED, bool CO>
__global__ void k_update_wide(Layout L, TX* x, TS* r, TS* z, TS* p, const TS* q, const TS* minv,
                              double* partials, PcgState* st, const TS* W, const double* G, int nk) {
  pdl_wait();
  pdl_trigger();
  if (st->done) return;
  const int cw = CW ? CW : L.cw;
  extern __shared__ unsigned char sh_raw[];
  TS* rs = reinterpret_cast<TS*>(sh_raw);
  const int64_t n = (int64_t)L.nC * cw;
  const int64_t base = (int64_t)blockIdx.x * (blockDim.x / cw) * cw;
  const int lt = threadIdx.x;
  const int64_t i = base + lt;
  const bool active = lt < (int)(blockDim.x / cw) * cw && i < n;
  double rr = 0, rz = 0;
  TS ri = 0;
  if (active) {
    TS pc = z[i] + (TS)st->beta * p[i];
    double alpha = st->alpha;
    if (MIXED) x[i] += (TX)(alpha * (double)pc);
    else x[i] += (TX)((TS)alpha * pc);
    ri = r[i] - (TS)alpha * q[i];
    r[i] = ri;
    p[i] = pc;
    rr = (double)ri * (double)ri;
  }
  rs[lt] = ri;
  __syncthreads();
  if (active) {
    int64_t cam = i / cw;
    int c = (int)(i % cw);
    const TS* m = minv + cam * (int64_t)cw * cw + (int64_t)c * cw;
    const TS* rl = rs + (lt - c);
    TS zi = 0;
    for (int j = 0; j < cw; ++j) zi += m[j] * rl[j];
    z[i] = zi;
    rz = (double)ri * (double)zi;
  }
  constexpr int K = CO ? 2 + MAXK : 2;
  double s[K];
  s[0] = rr;
  s[1] = rz;
  if (CO)
#pragma unroll
    for (int j = 0; j < MAXK; ++j) s[2 + j] = (active && j < nk) ? (double)W[j * n + i] * (double)ri : 0.0;
  block_sums<K>(s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) partials[K * blockIdx.x + k] = s[k];
  if (arrive_last(&st->counter1)) {
    double tot[K];
    finish_sums<K>(partials, tot);
    const double* Gs = CO ? stage_coarse(G, nk) : G;
    if (threadIdx.x == 0) {
      if (CO) tot[1] += coarse_finish(Gs, nk, tot + 2, st);
      st->iterations += 1;
      st->rr = tot[0];
      bool conv = sqrt(tot[0]) < st->threshold;
      if (MIXED && (conv || st->iterations >= st->max_iterations)) {
        st->done = 2;
        st->replace = 1;
        // the search direction continues if the FP64 residual disagrees
        st->beta = st->rz > 0 ? tot[1] / st->rz : 0.0;
        st->rz = tot[1];
      } else if (!MIXED && conv) {
        st->done = 1;
        st->termination = FG_TERM_CONVERGED;
      } else if (!(st->rz > 0)) {
        st->done = 1;
        st->termination = FG_TERM_NOT_POSITIVE_DEFINITE;
      } else if (!MIXED && st->iterations >= st->max_iterations) {
        st->done = 1;
        st->termination = FG_TERM_ITERATION_LIMIT;
      } else {
        if (MIXED && tot[0] < st->delta2 * st->rr_last) st->replace = 1;
        st->beta = tot[1] / st->rz;
        st->rz = tot[1];
      }
      st->counter1 = 0;
    }
  }
}

// PCG start: r = b, x = 0, z = Minv r, p = 0, beta = 0, rz = r.z, ||b||.
template <int CW, class TS, class TX, bool CO>
__global__ void k_pcg_start(Layout L, const double* b, TX* x, TS* r, TS* z, TS* p, const TS* minv, double* partials,
                            PcgState* st, double rel_tol, const TS* W, const double* G, int nk) {
  const int cw = CW ? CW : L.cw;
  extern __shared__ unsigned char sh_raw[];
  TS* rs = reinterpret_cast<TS*>(sh_raw);
  const int64_t n = (int64_t)L.nC * cw;
  const int64_t base = (int64_t)blockIdx.x * (blockDim.x / cw) * cw;
  const int lt = threadIdx.x;
  const int64_t i = base + lt;
  const bool active = lt < (int)(blockDim.x / cw) * cw && i < n;
  double bb = 0, rz = 0;
  TS ri = 0;
  if (active) {
    ri = (TS)b[i];
    r[i] = ri;
    x[i] = 0;
    p[i] = 0;
    bb = (double)ri * (double)ri;
  }
  rs[lt] = ri;
  __syncthreads();
  if (active) {
    int64_t cam = i / cw;
    int c = (int)(i % cw);
    const TS* m = minv + cam * (int64_t)cw * cw + (int64_t)c * cw;
    const TS* rl = rs + (lt - c);
    TS zi = 0;
    for (int j = 0; j < cw; ++j) zi += m[j] * rl[j];
    z[i] = zi;
    rz = (double)ri * (double)zi;
  }
  constexpr int K = CO ? 2 + MAXK : 2;
  double s[K];
  s[0] = bb;
  s[1] = rz;
  if (CO)
#pragma unroll
    for (int j = 0; j < MAXK; ++j) s[2 + j] = (active && j < nk) ? (double)W[j * n + i] * (double)ri : 0.0;
  block_sums<K>(s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) partials[K * blockIdx.x + k] = s[k];
  if (arrive_last(&st->counter2)) {
    double tot[K];
    finish_sums<K>(partials, tot);
    const double* Gs = CO ? stage_coarse(G, nk) : G;
    if (threadIdx.x == 0) {
      st->coarse_pending = 0;
      st->counter4 = 0;
      if (CO) tot[1] += coarse_finish(Gs, nk, tot + 2, st);
      double bn = sqrt(tot[0]);
      st->bnorm = bn;
      st->threshold = rel_tol * bn;
      st->iterations = 0;
      st->beta = 0;
      st->alpha = 0;
      st->rr = tot[0];
      st->rr_last = tot[0];
      st->rz = tot[1];
      st->replace = 0;
      st->replacements = 0;
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

// FP64 residual replacement, gated by st->replace: r = b - S xd (qd = S xd in
// FP64 arithmetic), z = Minv r, rz = r.z. Ends the solve when the FP64 residual
// meets the threshold. When the recurrence had claimed convergence but the
// FP64 residual disagrees, the iteration goes on along the same search
// direction (beta from the recurrence, as after a periodic replacement):
// restarting from steepest descent would discard the Krylov space built so far.
template <int CW, class TS, bool CO>
__global__ void k_replace_wide(Layout L, const double* b, const double* qd, TS* r, TS* z, const TS* minv,
                               double* partials, PcgState* st, const TS* W, const double* G, int nk) {
  if (!st->replace) return;
  const int cw = CW ? CW : L.cw;
  extern __shared__ unsigned char sh_raw[];
  TS* rs = reinterpret_cast<TS*>(sh_raw);
  const int64_t n = (int64_t)L.nC * cw;
  const int64_t base = (int64_t)blockIdx.x * (blockDim.x / cw) * cw;
  const int lt = threadIdx.x;
  const int64_t i = base + lt;
  const bool active = lt < (int)(blockDim.x / cw) * cw && i < n;
  double rr = 0, rz = 0;
  TS ri = 0;
  if (active) {
    double rt = b[i] - qd[i];
    rr = rt * rt;
    ri = (TS)rt;
    r[i] = ri;
  }
  rs[lt] = ri;
  __syncthreads();
  if (active) {
    int64_t cam = i / cw;
    int c = (int)(i % cw);
    const TS* m = minv + cam * (int64_t)cw * cw + (int64_t)c * cw;
    const TS* rl = rs + (lt - c);
    TS zi = 0;
    for (int j = 0; j < cw; ++j) zi += m[j] * rl[j];
    z[i] = zi;
    rz = (double)ri * (double)zi;
  }
  constexpr int K = CO ? 2 + MAXK : 2;
  double s[K];
  s[0] = rr;
  s[1] = rz;
  if (CO)
#pragma unroll
    for (int j = 0; j < MAXK; ++j) s[2 + j] = (active && j < nk) ? (double)W[j * n + i] * (double)ri : 0.0;
  block_sums<K>(s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) partials[K * blockIdx.x + k] = s[k];
  if (arrive_last(&st->counter3)) {
    double tot[K];
    finish_sums<K>(partials, tot);
    const double* Gs = CO ? stage_coarse(G, nk) : G;
    if (threadIdx.x == 0) {
      if (CO) tot[1] += coarse_finish(Gs, nk, tot + 2, st);
      st->rr_last = tot[0];
      st->rr = tot[0];
      st->replacements += 1;
      st->replace = 0;
      st->rz = tot[1];
      if (sqrt(tot[0]) < st->threshold) {
        st->done = 1;
        st->termination = FG_TERM_CONVERGED;
      } else if (st->done == 2 && st->iterations >= st->max_iterations) {
        st->done = 1;
        st->termination = FG_TERM_ITERATION_LIMIT;
      } else if (st->done == 2) {
        st->done = 0;
      }
      st->counter3 = 0;
    }
  }
}

// z += W c for the pending coarse coefficients (see k_update_wide); the last
// block clears the flag after every block has read it.
template <class TS>
__global__ void k_coarse_add(int64_t n, int nk, const TS* W, PcgState* st, TS* z) {
  pdl_wait();
  pdl_trigger();
  if (!st->coarse_pending) return;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) {
    double acc = (double)z[i];
    for (int j = 0; j < nk; ++j) acc += (double)W[j * n + i] * st->coarse[j];
    z[i] = (TS)acc;
  }
  if (arrive_last(&st->counter4)) {
    if (threadIdx.x == 0) {
      st->coarse_pending = 0;
      st->counter4 = 0;
    }
  }
}

// W = D * basis (scaled coordinates) in f64 and in the storage type.
template <class TS>
__global__ void k_coarse_scale(int64_t n, int nk, const double* basis, const double* scales, double* wd, TS* wt) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n * nk) return;
  const double v = basis[k] * scales[k % n];
  wd[k] = v;
  wt[k] = (TS)v;
}

// G = E^-1 for the nk x nk coarse matrix (Cholesky of its symmetric part by
// one thread in shared memory, then one thread per column of the inverse);
// G = 0 — a one-level preconditioner — when E is not positive definite. *ok
// reports which. Launched with one warp.
static __global__ void k_coarse_factor(int nk, const double* E, double* G, int* ok) {
  __shared__ double L[MAXK][MAXK], Es[MAXK * MAXK];
  __shared__ int spd_s;
  const int t = threadIdx.x;
  for (int i = t; i < nk * nk; i += blockDim.x) Es[i] = E[i];  // one parallel round trip
  __syncwarp();
  if (t == 0) {
    int spd = 1;
    for (int j = 0; j < nk && spd; ++j)
      for (int i = j; i < nk; ++i) {
        double v = 0.5 * (Es[i * nk + j] + Es[j * nk + i]);
        for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k];
        if (i == j) {
          if (!(v > 0) || !isfinite(v)) {
            spd = 0;
            break;
          }
          L[j][j] = sqrt(v);
        } else {
          L[i][j] = v / L[j][j];
        }
      }
    spd_s = spd;
    *ok = spd;
  }
  __syncwarp();
  if (t >= nk) return;
  const int c = t;  // column c of L^-T L^-1
  double y[MAXK], x[MAXK];
#pragma unroll
  for (int i = 0; i < MAXK; ++i) {
    y[i] = 0;
    x[i] = 0;
  }
  if (spd_s) {
#pragma unroll
    for (int i = 0; i < MAXK; ++i) {
      if (i < nk) {
        double v = i == c ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < MAXK; ++k)
          if (k < i) v -= L[i][k] * y[k];
        y[i] = v / L[i][i];
      }
    }
#pragma unroll
    for (int i = MAXK - 1; i >= 0; --i) {
      if (i < nk) {
        double v = y[i];
#pragma unroll
        for (int k = 0; k < MAXK; ++k)
          if (k > i && k < nk) v -= L[k][i] * x[k];
        x[i] = v / L[i][i];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < MAXK; ++i)
    if (i < nk) G[i * nk + c] = x[i];
}

// E[a][b] = W_a . (S W)_b, one block per entry.
template <class TS>
__global__ void k_coarse_gram(int64_t n, int nk, const double* wd, const TS* sw, double* e) {
  const int a = blockIdx.x / nk, b = blockIdx.x % nk;
  double v[1] = {0};
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) v[0] += wd[a * n + i] * (double)sw[b * n + i];
  block_sums<1>(v);
  if (threadIdx.x == 0) e[a * nk + b] = v[0];
}

}  // namespace fg
