// CTA-level dense linear algebra shared by the batched pose-graph windows
// and the single-system dense backends: blocked lower Cholesky (panel CB,
// 64 x 64 trailing tiles, warp-level diagonal factorization, optional
// envelope-tile skipping), blocked triangular solves, column-pivoted
// Householder QR, and CTA reductions. Every routine is called by all WNT
// threads of a CTA with uniform arguments.
#pragma once
#include "common.cuh"

namespace fg {

constexpr int WNT = 256;  // threads per CTA
constexpr int WCT = 64;   // trailing-update tile

__device__ __forceinline__ double wsum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0;
  for (int w = 0; w < WNT / 32; ++w) t += red[w];
  return t;
}
__device__ __forceinline__ double wmax(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = red[0];
  for (int w = 1; w < WNT / 32; ++w) t = fmax(t, red[w]);
  return t;
}

// ------------------------------------------------------- dense kernels
// Warp 0 factors the kb x kb diagonal block held in shared memory (row-major,
// row stride CB+1; lane i owns row i); false on a non-positive or nonfinite
// pivot (the same answer in every lane).
template <class TF, int CB>
__device__ bool warp_potrf(TF* Dg, int kb) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < kb; ++j) {
    TF d = Dg[j * (CB + 1) + j];
    if (!(d > TF(0)) || !isfinite((double)d)) return false;
    d = sqrt(d);
    __syncwarp();
    if (lane == j) Dg[j * (CB + 1) + j] = d;
    TF lij = 0;
    if (lane > j && lane < kb) {
      lij = Dg[lane * (CB + 1) + j] / d;
      Dg[lane * (CB + 1) + j] = lij;
    }
    __syncwarp();
    if (lane > j && lane < kb)
      for (int c = j + 1; c <= lane; ++c) Dg[lane * (CB + 1) + c] -= lij * Dg[c * (CB + 1) + j];
    __syncwarp();
  }
  return true;
}

// In-place lower Cholesky of the n x n lower triangle of A (column-major,
// leading dimension lda) by the whole CTA; false on a non-positive or
// nonfinite pivot. sm holds CB x (CB+1) + 2 x WCT x (CB+1) TF values.
// cmin[T] (optional; null = dense) is the first 64-column tile that any row
// of 64-row tile T reaches (its envelope, which Cholesky fill never leaves):
// tiles left of it are exact zeros and are neither read nor written, so only
// the envelope tiles of A need to be initialized.
template <class TF, int CB>
__device__ bool cta_cholesky(TF* A, int n, int lda, TF* sm, int* flag, const int32_t* cmin) {
  TF* Dg = sm;
  TF* PI = Dg + CB * (CB + 1);
  TF* PJ = PI + WCT * (CB + 1);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int k0 = 0; k0 < n; k0 += CB) {
    const int kb = min(CB, n - k0);
    for (int e = tid; e < kb * kb; e += WNT) {
      const int r = e % kb, c = e / kb;
      if (r >= c) Dg[r * (CB + 1) + c] = A[(size_t)(k0 + c) * lda + k0 + r];
    }
    __syncthreads();
    if (warp == 0) {
      const bool ok = warp_potrf<TF, CB>(Dg, kb);
      if (lane == 0) *flag = ok ? 0 : 1;
    }
    __syncthreads();
    if (*flag) return false;
    for (int e = tid; e < kb * kb; e += WNT) {
      const int r = e % kb, c = e / kb;
      if (r >= c) A[(size_t)(k0 + c) * lda + k0 + r] = Dg[r * (CB + 1) + c];
    }
    const int t0 = k0 + kb;
    if (t0 >= n) break;  // kb == CB whenever rows remain below
    // Row tiles (64 rows, aligned at 0) whose rows' envelopes start right of
    // this panel hold exact zeros in it: skip them in the panel solve and the
    // trailing update.
    const int pc = k0 / WCT, T0 = t0 / WCT, nT = (n + WCT - 1) / WCT;
    // Panel: L[i, k0:k0+CB] = A[i, k0:k0+CB] L_kk^-T, one row per thread.
    for (int i = t0 + tid; i < n; i += WNT) {
      if (cmin && cmin[i / WCT] > pc) continue;
      TF x[CB];
#pragma unroll
      for (int q = 0; q < CB; ++q) x[q] = A[(size_t)(k0 + q) * lda + i];
#pragma unroll
      for (int c = 0; c < CB; ++c) {
        TF s = x[c];
#pragma unroll
        for (int q = 0; q < c; ++q) s -= x[q] * Dg[c * (CB + 1) + q];
        x[c] = s / Dg[c * (CB + 1) + c];
      }
#pragma unroll
      for (int q = 0; q < CB; ++q) A[(size_t)(k0 + q) * lda + i] = x[q];
    }
    __syncthreads();
    // Trailing update A[I, J] -= L[I, panel] L[J, panel]^T on lower tiles.
    const int tr = tid & 15, tc = tid >> 4;
    for (int JT = T0; JT < nT; ++JT) {
      if (cmin && cmin[JT] > pc) continue;  // uniform across the CTA
      const int J0 = max(JT * WCT, t0), nj = min(JT * WCT + WCT, n) - J0;
      for (int e = tid; e < WCT * CB; e += WNT) {
        const int r = e % WCT, q = e / WCT;
        PJ[r * (CB + 1) + q] = r < nj ? A[(size_t)(k0 + q) * lda + J0 + r] : TF(0);
      }
      for (int IT = JT; IT < nT; ++IT) {
        if (cmin && cmin[IT] > pc) continue;
        const int I0 = max(IT * WCT, t0), ni = min(IT * WCT + WCT, n) - I0;
        TF* P = PJ;
        if (IT != JT) {
          P = PI;
          for (int e = tid; e < WCT * CB; e += WNT) {
            const int r = e % WCT, q = e / WCT;
            PI[r * (CB + 1) + q] = r < ni ? A[(size_t)(k0 + q) * lda + I0 + r] : TF(0);
          }
        }
        __syncthreads();
        TF acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = 0;
#pragma unroll 8
        for (int q = 0; q < CB; ++q) {
          TF u[4], v[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            u[a] = P[(tr + 16 * a) * (CB + 1) + q];
            v[a] = PJ[(tc + 16 * a) * (CB + 1) + q];
          }
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] += u[a] * v[b];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int r = tr + 16 * a, c = tc + 16 * b;
            if (r < ni && c < nj && I0 + r >= J0 + c) A[(size_t)(J0 + c) * lda + I0 + r] -= acc[a][b];
          }
        __syncthreads();
      }
    }
  }
  return true;
}

// v <- L^-T L^-1 v for the lower factor L (whole CTA). The diagonal blocks are
// staged in shared memory (Dg, CB x (CB+1)) and solved by warp 0 with
// shuffles; the off-diagonal updates run one row per thread.
template <class TF, int CB>
__device__ void cta_llt_solve(const TF* L, int n, int lda, TF* v, TF* Dg, const int32_t* cmin) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int k0 = 0; k0 < n; k0 += CB) {
    const int kb = min(CB, n - k0);
    for (int e = tid; e < kb * kb; e += WNT) {
      const int r = e % kb, c = e / kb;
      if (r >= c) Dg[r * (CB + 1) + c] = L[(size_t)(k0 + c) * lda + k0 + r];
    }
    __syncthreads();
    if (warp == 0) {
      TF x = lane < kb ? v[k0 + lane] : TF(0);
      for (int c = 0; c < kb; ++c) {
        const TF xc = __shfl_sync(0xffffffffu, x, c) / Dg[c * (CB + 1) + c];
        if (lane == c) x = xc;
        else if (lane > c && lane < kb) x -= Dg[lane * (CB + 1) + c] * xc;
      }
      if (lane < kb) v[k0 + lane] = x;
    }
    __syncthreads();
    const int pc = k0 / WCT;
    for (int i = k0 + kb + tid; i < n; i += WNT) {
      if (cmin && cmin[i / WCT] > pc) continue;
      TF s = v[i];
      for (int q = 0; q < kb; ++q) s -= L[(size_t)(k0 + q) * lda + i] * v[k0 + q];
      v[i] = s;
    }
    __syncthreads();
  }
  const int last = n > 0 ? ((n - 1) / CB) * CB : -1;
  for (int k0 = last; k0 >= 0; k0 -= CB) {
    const int kb = min(CB, n - k0);
    for (int e = tid; e < kb * kb; e += WNT) {
      const int r = e % kb, c = e / kb;
      if (r >= c) Dg[r * (CB + 1) + c] = L[(size_t)(k0 + c) * lda + k0 + r];
    }
    __syncthreads();
    if (warp == 0) {
      TF x = lane < kb ? v[k0 + lane] : TF(0);
      for (int c = kb - 1; c >= 0; --c) {
        const TF xc = __shfl_sync(0xffffffffu, x, c) / Dg[c * (CB + 1) + c];
        if (lane == c) x = xc;
        else if (lane < c) x -= Dg[c * (CB + 1) + lane] * xc;
      }
      if (lane < kb) v[k0 + lane] = x;
    }
    __syncthreads();
    for (int q = (cmin ? WCT * cmin[k0 / WCT] : 0) + tid; q < k0; q += WNT) {
      TF s = v[q];
      const TF* col = L + (size_t)q * lda + k0;
      for (int i = 0; i < kb; ++i) s -= col[i] * v[k0 + i];
      v[q] = s;
    }
    __syncthreads();
  }
}

// Column-pivoted Householder QR of rows [r0, m) x columns [c0, c0+w) of the
// column-major m x ncols matrix M, transforming every column right of the
// block; perm (w entries) receives the pivot order (Elimination::qr,
// marginalization.rs:412-455). A zero block is left as it is.
static __device__ void cta_qr(double* M, int m, int ncols, int r0, int c0, int w, int* perm, double* norms, double* red,
                       int* flag) {
  const int tid = threadIdx.x;
  for (int k = tid; k < w; k += WNT) perm[k] = k;
  const int h = m - r0;
  double mx = 0;
  for (int e = tid; e < h * w; e += WNT) mx = fmax(mx, fabs(M[(size_t)(c0 + e / h) * m + r0 + e % h]));
  mx = wmax(mx, red);
  if (h <= 0 || w <= 0 || mx == 0) {
    __syncthreads();
    return;
  }
  const int steps = min(h, w);
  for (int k = 0; k < steps; ++k) {
    for (int j = k + tid; j < w; j += WNT) {
      const double* col = M + (size_t)(c0 + j) * m + r0;
      double s = 0;
      for (int i = k; i < h; ++i) s += col[i] * col[i];
      norms[j] = s;
    }
    __syncthreads();
    if (tid == 0) {
      int best = k;
      double bn = -1;
      for (int j = k; j < w; ++j)
        if (norms[j] > bn) {
          bn = norms[j];
          best = j;
        }
      *flag = best;
    }
    __syncthreads();
    const int best = *flag;
    if (best != k) {
      double* x = M + (size_t)(c0 + k) * m + r0;
      double* y = M + (size_t)(c0 + best) * m + r0;
      for (int i = tid; i < h; i += WNT) {
        const double t = x[i];
        x[i] = y[i];
        y[i] = t;
      }
      if (tid == 0) {
        const int t = perm[k];
        perm[k] = perm[best];
        perm[best] = t;
      }
    }
    __syncthreads();
    double* v = M + (size_t)(c0 + k) * m + r0;
    if (tid == 0) {
      const double alpha = v[k];
      double xn2 = 0;
      for (int i = k + 1; i < h; ++i) xn2 += v[i] * v[i];
      const double xn = sqrt(xn2);
      if (xn == 0) {
        red[0] = 0;  // H = I
      } else {
        const double beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        const double tau = (beta - alpha) / beta;
        const double scale = 1.0 / (alpha - beta);
        for (int i = k + 1; i < h; ++i) v[i] *= scale;
        v[k] = beta;
        red[0] = tau;
      }
    }
    __syncthreads();
    const double tau = red[0];
    if (tau != 0) {
      for (int j = c0 + k + 1 + tid; j < ncols; j += WNT) {
        double* cj = M + (size_t)j * m + r0;
        double s = cj[k];
        for (int i = k + 1; i < h; ++i) s += v[i] * cj[i];
        s *= tau;
        cj[k] -= s;
        for (int i = k + 1; i < h; ++i) cj[i] -= s * v[i];
      }
    }
    __syncthreads();
  }
}

}  // namespace fg
