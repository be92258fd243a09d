// Learned block preconditioner: a message-passing network over the camera
// covisibility graph of the reduced camera system, with BF16 tensor-core GEMMs
// (mma.sync m16n8k16, FP32 accumulation) for inference and training, Adam on
// the device, and the feature / probe kernels that turn a Schur backend's
// factors into training systems. fagra has no learned preconditioner; the
// network reshapes the retained block-Jacobi preconditioner of
// src/schur.rs:658-682 (block factors of src/linear_model/block_factors.rs:
// 113-138) and falls back to it.
//
// Math (whitened block-Jacobi coordinates, L_c L_c^T = B_c + lambda I):
//   features  P_c = L_c^-1 (sum_e E_e C_p^-1 E_e^T) L_c^-1^T, covisibility
//             s_ij = sqrt(sum_p ||G_ip G_jp^T||_F^2), G_e = L_c^-1 E_e L_p^-T,
//             row-normalized;
//   network   h0 = relu(X0 W_in + b_in); h_l = h_{l-1} + relu([h_{l-1}, A h_{l-1}] W_l + b_l), l = 1..3;
//             O = h_3 W_out + b_out;
//   head      A_c = I + 0.1 tril(O_c), M_c = L_c^-T (A_c A_c^T + 1e-3 I) L_c^-1 (SPD);
//   loss      mean ||x - M_hat S_hat x||^2 over whitened probes x.
#include "gnn.cuh"
#include <cuda_bf16.h>
#include <algorithm>
#include <memory>
#include <new>
#include <random>

namespace fg {
namespace {

constexpr int NF = 64;  // node features
constexpr int NH = 64;  // hidden width
constexpr int NLAYER = 3;
constexpr float OUT_SCALE = 0.1f;
constexpr float EPSILON = 1e-3f;

// flat parameter layout: W_in (64x64), b_in, {W_l (128x64), b_l} x 3, W_out (64x64), b_out
struct PLayout {
  size_t w_in, b_in, w[NLAYER], b[NLAYER], w_out, b_out, total;
  PLayout() {
    size_t o = 0;
    w_in = o; o += NF * NH;
    b_in = o; o += NH;
    for (int l = 0; l < NLAYER; ++l) {
      w[l] = o; o += 2 * NH * NH;
      b[l] = o; o += NH;
    }
    w_out = o; o += NH * NH;
    b_out = o; o += NH;
    total = o;
  }
};

// ------------------------------------------------------------------ GEMM
// C (M x N) = op(A) (M x K) * op(B) (K x N); A(m,k) = TRA ? A[k*lda+m] : A[m*lda+k],
// B(k,n) = TRB ? B[n*ldb+k] : B[k*ldb+n]. Operands are rounded to bf16 into
// shared memory; 64x64 CTA tile, 4 warps of 32x32, K step 32; split-K over
// gridDim.z (EPI_STORE only, atomic accumulation into C).
enum Epilogue { EPI_STORE = 0, EPI_BIAS_RELU = 1, EPI_BIAS = 2, EPI_SPLIT = 3, EPI_STORE_MASK = 4 };
struct Epi {
  const float* bias = nullptr;
  float* z = nullptr;        // BIAS_RELU: pre-activation out
  int ldz = 0;
  float* h = nullptr;        // BIAS_RELU: activation out; SPLIT: second half out
  int ldh = 0;
  const float* r = nullptr;  // BIAS_RELU: residual in (may be null); SPLIT: added to the first half
  int ldr = 0;
  const float* zmask = nullptr;  // STORE_MASK: pre-activation whose sign masks d2
  int ldzm = 0;
  float* d2 = nullptr;
  int ldd2 = 0;
  int accumulate = 0;  // STORE: C += result
  int split_at = 0;    // SPLIT: columns >= split_at go to h
};

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int GT = 64, GK = 32, GPAD = 40;

template <class TA, class TB, bool TRA, bool TRB, int EPI>
__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const TA* __restrict__ A, int lda,
                                              const TB* __restrict__ B, int ldb, float* __restrict__ Cm, int ldc,
                                              Epi ep, int kchunk) {
  __shared__ __align__(16) __nv_bfloat16 As[GT][GPAD];
  __shared__ __align__(16) __nv_bfloat16 Bs[GT][GPAD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.x * GT, n0 = blockIdx.y * GT;
  const int kb = blockIdx.z * kchunk;
  const int ke = min(K, kb + kchunk);
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;
  for (int k0 = kb; k0 < ke; k0 += GK) {
#pragma unroll 4
    for (int j = 0; j < GT * GK / 128; ++j) {
      const int i = tid + 128 * j;
      const int m = TRA ? (i & 63) : (i >> 5);
      const int k = TRA ? (i >> 6) : (i & 31);
      const int gm = m0 + m, gk = k0 + k;
      float v = 0.f;
      if (gm < M && gk < ke) v = to_f(TRA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk]);
      As[m][k] = __float2bfloat16_rn(v);
    }
#pragma unroll 4
    for (int j = 0; j < GT * GK / 128; ++j) {
      const int i = tid + 128 * j;
      const int n = TRB ? (i >> 5) : (i & 63);
      const int k = TRB ? (i & 31) : (i >> 6);
      const int gn = n0 + n, gk = k0 + k;
      float v = 0.f;
      if (gn < N && gk < ke) v = to_f(TRB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn]);
      Bs[n][k] = __float2bfloat16_rn(v);
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < GK; ks += 16) {
      uint32_t a[2][4], b[4][2];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        const int r = wm + mi * 16 + g;
        a[mi][0] = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * t]);
        a[mi][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * t]);
        a[mi][2] = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * t + 8]);
        a[mi][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int c = wn + ni * 8 + g;
        b[ni][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + 2 * t]);
        b[ni][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) mma_bf16(acc[mi][ni], a[mi], b[ni]);
    }
    __syncthreads();
  }
  const bool split = gridDim.z > 1;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = m0 + wm + mi * 16 + g + (q >> 1) * 8;
        const int n = n0 + wn + ni * 8 + 2 * t + (q & 1);
        if (m >= M || n >= N) continue;
        const float v = acc[mi][ni][q];
        if (EPI == EPI_STORE) {
          float* c = Cm + (size_t)m * ldc + n;
          if (split) atomicAdd(c, v);
          else *c = ep.accumulate ? *c + v : v;
        } else if (EPI == EPI_BIAS_RELU) {
          const float z = v + ep.bias[n];
          ep.z[(size_t)m * ep.ldz + n] = z;
          const float res = ep.r ? ep.r[(size_t)m * ep.ldr + n] : 0.f;
          ep.h[(size_t)m * ep.ldh + n] = res + fmaxf(z, 0.f);
        } else if (EPI == EPI_BIAS) {
          Cm[(size_t)m * ldc + n] = v + ep.bias[n];
        } else if (EPI == EPI_SPLIT) {
          if (n < ep.split_at) Cm[(size_t)m * ldc + n] = v + ep.r[(size_t)m * ep.ldr + n];
          else ep.h[(size_t)m * ep.ldh + (n - ep.split_at)] = v;
        } else if (EPI == EPI_STORE_MASK) {
          Cm[(size_t)m * ldc + n] = v;
          ep.d2[(size_t)m * ep.ldd2 + n] = ep.zmask[(size_t)m * ep.ldzm + n] > 0.f ? v : 0.f;
        }
      }
}

template <class TA, class TB, bool TRA, bool TRB, int EPI>
fg_status gemm(cudaStream_t st, int nsm, int M, int N, int K, const TA* A, int lda, const TB* B, int ldb, float* Cm,
               int ldc, const Epi& ep, bool allow_split) {
  if (M <= 0 || N <= 0) return FG_OK;
  const unsigned gx = (unsigned)((M + GT - 1) / GT), gy = (unsigned)((N + GT - 1) / GT);
  int splits = 1;
  if (allow_split && EPI == EPI_STORE && K > 256) {
    const int want = std::max(1, (2 * nsm) / (int)(gx * gy));
    splits = std::min(want, (K + 255) / 256);
  }
  int kchunk = (K + splits - 1) / splits;
  kchunk = std::max(GK, (kchunk + GK - 1) / GK * GK);
  splits = std::max(1, (K + kchunk - 1) / kchunk);
  if (K <= 0) {  // empty reduction: the product is zero
    splits = 1;
    kchunk = GK;
  }
  if (EPI == EPI_STORE && splits > 1 && !ep.accumulate)
    FG_CUDA(cudaMemset2DAsync(Cm, (size_t)ldc * sizeof(float), 0, (size_t)N * sizeof(float), (size_t)M, st));
  dim3 grid(gx, gy, (unsigned)splits);
  FG_LAUNCH((k_gemm<TA, TB, TRA, TRB, EPI>), grid, 128, 0, st, M, N, K, A, lda, B, ldb, Cm, ldc, ep, kchunk);
  return FG_OK;
}

// ------------------------------------------------------------------ small kernels
__global__ void k_colsum(int M, const float* X, int ld, float* out) {  // 64 columns, one block of 256
  const int c = threadIdx.x & 63, r0 = threadIdx.x >> 6;
  float s = 0.f;
  for (int r = r0; r < M; r += 4) s += X[(size_t)r * ld + c];
  __shared__ float sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < 64) out[c] = (sh[c] + sh[c + 64]) + (sh[c + 128] + sh[c + 192]);
}

__global__ void k_relu_mask(int64_t n, const float* dh, const float* z, float* dz) {  // contiguous C x 64
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dz[i] = z[i] > 0.f ? dh[i] : 0.f;
}

__global__ void k_adam(int64_t n, float* w, const float* grad, float* m, float* v, __nv_bfloat16* wbf, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  wbf[i] = __float2bfloat16_rn(wi);
}

__global__ void k_to_bf16(int64_t n, const float* x, __nv_bfloat16* y) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

__device__ __forceinline__ double lane_allsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Standard normal probes by Box-Muller over a counter-based hash.
__global__ void k_probe_fill(int64_t n, uint64_t seed, float* out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t h = splitmix(seed ^ splitmix((uint64_t)i));
  const double u1 = ((h >> 11) + 1.0) * (1.0 / 9007199254740993.0);  // (0, 1]
  const double u2 = (double)(splitmix(h) >> 11) * (1.0 / 9007199254740992.0);
  out[i] = (float)(sqrt(-2.0 * log(u1)) * cospi(2.0 * u2));
}

// Lower factor element L(i,k) in the Gram layout (column major).
template <class TS>
__device__ __forceinline__ double lf(const TS* l, int n, int i, int k) {
  return (double)l[k * n + i];
}
template <class TS>
__device__ __forceinline__ void fwd_solve(const TS* l, double* x, int n) {  // x = L^-1 x
  for (int i = 0; i < n; ++i) {
    double s = x[i];
    for (int k = 0; k < i; ++k) s -= lf(l, n, i, k) * x[k];
    x[i] = s / lf(l, n, i, i);
  }
}
template <class TS>
__device__ __forceinline__ void bwd_solve(const TS* l, double* x, int n) {  // x = L^-T x
  for (int i = n - 1; i >= 0; --i) {
    double s = x[i];
    for (int k = i + 1; k < n; ++k) s -= lf(l, n, k, i) * x[k];
    x[i] = s / lf(l, n, i, i);
  }
}

// Node features of observed cameras (warp per camera): U = sum_e E_e C_p^-1 E_e^T
// (as the exact Schur diagonal), P = L_c^-1 U L_c^-T; X0 row = [P lower
// (column major), ., ., log10(lambda)/12, trace(P)/cw, 1, 0...]. Columns 45
// and 46 are written by k_normalize.
template <class TS>
__global__ void k_node_features(Layout L, const int64_t* cam_edge_off, const int64_t* cam_edge,
                                const DEdgeMeta* edges, const TS* cross, const uint8_t* observed, const TS* factors,
                                double lambda, float* X0, uint8_t* mask) {
  const int cw = L.cw, pw = L.pw;
  constexpr int NL = GNN_MAX_CW * (GNN_MAX_CW + 1) / 2;
  const int lane = threadIdx.x & 31;
  const int64_t cam = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (cam >= L.nC) return;
  float* row = X0 + cam * NF;
  if (!observed[cam]) {
    if (lane == 0) mask[cam] = 0;
    for (int k = lane; k < NF; k += 32) row[k] = k == 49 ? 1.f : 0.f;
    return;
  }
  double acc[NL];
  const int nl = cw * (cw + 1) / 2;
  for (int k = 0; k < NL; ++k) acc[k] = 0;
  for (int64_t k = cam_edge_off[cam] + lane; k < cam_edge_off[cam + 1]; k += 32) {
    const int64_t e = cam_edge[k];
    const int pt = edges[e].pt;
    const TS* E = cross + e * (int64_t)cw * pw;
    const bool obs = observed[L.nC + pt];
    const TS* lp = factors + L.gram_offset(L.nC + pt);
    double y[GNN_MAX_CW][GNN_MAX_PW];
    for (int c = 0; c < cw; ++c) {
      double b[GNN_MAX_PW];
      for (int p = 0; p < pw; ++p) b[p] = (double)E[p * cw + c];
      if (obs) {
        fwd_solve(lp, b, pw);
        bwd_solve(lp, b, pw);
      } else {
        for (int p = 0; p < pw; ++p) b[p] /= lambda;
      }
      for (int p = 0; p < pw; ++p) y[c][p] = b[p];
    }
    int idx = 0;
    for (int c = 0; c < cw; ++c)
      for (int r = c; r < cw; ++r) {
        double s = 0;
        for (int p = 0; p < pw; ++p) s += (double)E[p * cw + r] * y[c][p];
        acc[idx++] += s;
      }
  }
  for (int k = 0; k < nl; ++k) acc[k] = lane_allsum(acc[k]);
  if (lane != 0) return;
  const TS* lc = factors + L.gram_offset(cam);
  double U[GNN_MAX_CW * GNN_MAX_CW];
  int idx = 0;
  for (int c = 0; c < cw; ++c)
    for (int r = c; r < cw; ++r) {
      U[c * cw + r] = acc[idx];
      U[r * cw + c] = acc[idx];
      ++idx;
    }
  // W = L^-1 U (columns), then P = L^-1 W^T (U symmetric)
  for (int c = 0; c < cw; ++c) fwd_solve(lc, U + c * cw, cw);  // column c of U (column major)
  double P[GNN_MAX_CW * GNN_MAX_CW];
  for (int c = 0; c < cw; ++c) {
    double col[GNN_MAX_CW];
    for (int r = 0; r < cw; ++r) col[r] = U[r * cw + c];  // row c of W = column c of W^T
    fwd_solve(lc, col, cw);
    for (int r = 0; r < cw; ++r) P[c * cw + r] = col[r];
  }
  double tr = 0;
  for (int c = 0; c < cw; ++c) tr += P[c * cw + c];
  for (int k = 0; k < NF; ++k) row[k] = 0.f;
  idx = 0;
  for (int c = 0; c < cw; ++c)
    for (int r = c; r < cw; ++r) row[idx++] = (float)(0.5 * (P[c * cw + r] + P[r * cw + c]));
  row[47] = (float)(log10(fmax(lambda, 1e-12)) / 12.0);
  row[48] = (float)(tr / cw);
  row[49] = 1.f;
  mask[cam] = 1;
}

// K_e = L_p^-1 (L_c^-1 E_e)^T (L_c^-1 E_e) L_p^-T, thread per edge (pw x pw, stride 16).
template <class TS>
__global__ void k_edge_k(Layout L, int64_t nedges, const DEdgeMeta* edges, const TS* cross, const uint8_t* observed,
                         const TS* factors, double lambda, float* Kout) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nedges) return;
  const int cw = L.cw, pw = L.pw;
  const DEdgeMeta m = edges[e];
  const TS* E = cross + e * (int64_t)cw * pw;
  float* out = Kout + e * 16;
  if (!observed[m.cam]) {
    for (int k = 0; k < 16; ++k) out[k] = 0.f;
    return;
  }
  const TS* lc = factors + L.gram_offset(m.cam);
  double Eb[GNN_MAX_PW][GNN_MAX_CW];
  for (int p = 0; p < pw; ++p) {
    for (int c = 0; c < cw; ++c) Eb[p][c] = (double)E[p * cw + c];
    fwd_solve(lc, Eb[p], cw);
  }
  double W[GNN_MAX_PW * GNN_MAX_PW];
  for (int p = 0; p < pw; ++p)
    for (int q = 0; q < pw; ++q) {
      double s = 0;
      for (int c = 0; c < cw; ++c) s += Eb[p][c] * Eb[q][c];
      W[p * pw + q] = s;
    }
  double K[GNN_MAX_PW * GNN_MAX_PW];
  if (observed[L.nC + m.pt]) {
    const TS* lp = factors + L.gram_offset(L.nC + m.pt);
    for (int q = 0; q < pw; ++q) {  // column q of W -> L_p^-1 W
      double col[GNN_MAX_PW];
      for (int p = 0; p < pw; ++p) col[p] = W[p * pw + q];
      fwd_solve(lp, col, pw);
      for (int p = 0; p < pw; ++p) W[p * pw + q] = col[p];
    }
    for (int p = 0; p < pw; ++p) {  // row p of (L_p^-1 W) -> L_p^-1 (.)^T
      double col[GNN_MAX_PW];
      for (int q = 0; q < pw; ++q) col[q] = W[p * pw + q];
      fwd_solve(lp, col, pw);
      for (int q = 0; q < pw; ++q) K[q * pw + p] = col[q];
    }
  } else {
    for (int k = 0; k < pw * pw; ++k) K[k] = W[k] / lambda;
  }
  for (int k = 0; k < 16; ++k) out[k] = k < pw * pw ? (float)K[k] : 0.f;
}

// Pair weights w_ij += <K_e, K_f> over the edge pairs of each point (warp per point).
__global__ void k_pairs(int64_t nP, int64_t nC, const int64_t* pt_edge_off, const int64_t* pt_edge,
                        const DEdgeMeta* edges, const float* Kin, int pw, float* adj) {
  const int lane = threadIdx.x & 31;
  const int64_t pt = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (pt >= nP) return;
  const int64_t o = pt_edge_off[pt], t = pt_edge_off[pt + 1] - o;
  const int nk = pw * pw;
  for (int64_t a = lane; a < t; a += 32) {
    const int64_t e = pt_edge[o + a];
    const int ci = edges[e].cam;
    float ka[16];
    for (int k = 0; k < 16; ++k) ka[k] = Kin[e * 16 + k];
    for (int64_t b = a + 1; b < t; ++b) {
      const int64_t f = pt_edge[o + b];
      const int cj = edges[f].cam;
      if (ci == cj) continue;
      float w = 0.f;
      for (int k = 0; k < nk; ++k) w += ka[k] * Kin[f * 16 + k];
      atomicAdd(adj + (int64_t)ci * nC + cj, w);
      atomicAdd(adj + (int64_t)cj * nC + ci, w);
    }
  }
}

// Row-normalized sqrt weights in bf16, plus features 45 (log1p degree / 4) and
// 46 (log1p coupling) of observed cameras. Block of 256 per row.
__global__ void k_normalize(int64_t nC, const float* adj, const uint8_t* mask, float* X0, __nv_bfloat16* Abf) {
  const int64_t i = blockIdx.x;
  const float* row = adj + i * nC;
  double s = 0;
  int cnt = 0;
  for (int64_t j = threadIdx.x; j < nC; j += blockDim.x) {
    const float w = row[j];
    if (w > 0.f) {
      s += sqrt((double)w);
      ++cnt;
    }
  }
  __shared__ double ss[256];
  __shared__ int sc[256];
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = cnt;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      ss[threadIdx.x] += ss[threadIdx.x + o];
      sc[threadIdx.x] += sc[threadIdx.x + o];
    }
    __syncthreads();
  }
  const double tot = ss[0];
  const double inv = tot > 0 ? 1.0 / tot : 0.0;
  for (int64_t j = threadIdx.x; j < nC; j += blockDim.x) {
    const float w = row[j];
    Abf[i * nC + j] = __float2bfloat16_rn(w > 0.f ? (float)(sqrt((double)w) * inv) : 0.f);
  }
  if (threadIdx.x == 0 && mask[i]) {
    X0[i * NF + 45] = (float)(log1p((double)sc[0]) / 4.0);
    X0[i * NF + 46] = (float)log1p(tot);
  }
}

__device__ __forceinline__ void head_factor(const float* o, int cw, double* A) {  // A = I + 0.1 tril(o)
  for (int k = 0; k < cw * cw; ++k) A[k] = 0;
  int idx = 0;
  for (int c = 0; c < cw; ++c)
    for (int r = c; r < cw; ++r) A[r * cw + c] = (double)OUT_SCALE * (double)o[idx++];
  for (int c = 0; c < cw; ++c) A[c * cw + c] += 1.0;
}
__device__ __forceinline__ void head_metric(const double* A, int cw, double* Mh) {  // A A^T + eps I (row major)
  for (int i = 0; i < cw; ++i)
    for (int j = 0; j < cw; ++j) {
      double s = 0;
      for (int k = 0; k < cw; ++k) s += A[i * cw + k] * A[j * cw + k];
      Mh[i * cw + j] = s + (i == j ? (double)EPSILON : 0.0);
    }
}

// Explicit M = L^-T Mh L^-1 into minv (storage type), thread per observed camera.
template <class TS>
__global__ void k_head_minv(Layout L, const float* O, const uint8_t* mask, const TS* factors, TS* minv,
                            unsigned* nonfinite) {
  const int64_t cam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cam >= L.nC || !mask[cam]) return;
  const int cw = L.cw;
  double A[GNN_MAX_CW * GNN_MAX_CW], Mh[GNN_MAX_CW * GNN_MAX_CW];
  head_factor(O + cam * NH, cw, A);
  head_metric(A, cw, Mh);
  const TS* l = factors + L.gram_offset(cam);
  double m[GNN_MAX_CW * GNN_MAX_CW];  // columns of L^-1 (m[j*cw+i] = (L^-1)_{ij})
  for (int j = 0; j < cw; ++j) {
    for (int i = 0; i < cw; ++i) m[j * cw + i] = i == j ? 1.0 : 0.0;
    fwd_solve(l, m + j * cw, cw);
  }
  double out[GNN_MAX_CW * GNN_MAX_CW];
  bool ok = true;
  for (int i = 0; i < cw; ++i)
    for (int j = i; j < cw; ++j) {
      double s = 0;  // sum_ab (L^-1)_{ai} Mh_ab (L^-1)_{bj}
      for (int a = 0; a < cw; ++a) {
        double t = 0;
        for (int b = 0; b < cw; ++b) t += Mh[a * cw + b] * m[j * cw + b];
        s += m[i * cw + a] * t;
      }
      ok = ok && isfinite(s);
      out[i * cw + j] = s;
      out[j * cw + i] = s;
    }
  if (!ok) {
    atomicAdd(nonfinite, 1u);
    return;
  }
  TS* dst = minv + cam * (int64_t)cw * cw;
  for (int k = 0; k < cw * cw; ++k) dst[k] = (TS)out[k];
}

// Training head: loss sum and dL/dO for probes PX, PY (K x C x cw), thread per camera.
__global__ void k_head_loss(int64_t nC, int cw, int K, const float* O, const float* PX, const float* PY,
                            const uint8_t* mask, double inv_kn, float* dO, double* loss) {
  const int64_t cam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cam >= nC) return;
  float* d = dO + cam * NH;
  for (int k = 0; k < NH; ++k) d[k] = 0.f;
  if (!mask[cam]) return;
  double A[GNN_MAX_CW * GNN_MAX_CW], Mh[GNN_MAX_CW * GNN_MAX_CW], G[GNN_MAX_CW * GNN_MAX_CW];
  head_factor(O + cam * NH, cw, A);
  head_metric(A, cw, Mh);
  for (int k = 0; k < cw * cw; ++k) G[k] = 0;
  double l2 = 0;
  const int64_t n = nC * cw;
  for (int k = 0; k < K; ++k) {
    const float* x = PX + k * n + cam * cw;
    const float* y = PY + k * n + cam * cw;
    for (int r = 0; r < cw; ++r) {
      double s = x[r];
      for (int c = 0; c < cw; ++c) s -= Mh[r * cw + c] * (double)y[c];
      l2 += s * s;
      for (int c = 0; c < cw; ++c) G[r * cw + c] += s * (double)y[c];
    }
  }
  atomicAdd(loss, l2 * inv_kn);
  const double gs = -2.0 * inv_kn;
  int idx = 0;
  for (int c = 0; c < cw; ++c)
    for (int r = c; r < cw; ++r) {
      double s = 0;  // dA = (G + G^T) A, G scaled by gs
      for (int k = 0; k < cw; ++k) s += (G[r * cw + k] + G[k * cw + r]) * A[k * cw + c];
      d[idx++] = (float)((double)OUT_SCALE * gs * s);
    }
}

// x = L_c^-T xh (unwhiten) and yh = L_c^-1 y (whiten), thread per camera;
// unobserved cameras use L = sqrt(lambda) I.
template <class TS>
__global__ void k_unwhiten(Layout L, const uint8_t* observed, const TS* factors, double lambda, const float* xh,
                           double* x) {
  const int64_t cam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cam >= L.nC) return;
  const int cw = L.cw;
  double v[GNN_MAX_CW];
  for (int c = 0; c < cw; ++c) v[c] = (double)xh[cam * cw + c];
  if (observed[cam]) bwd_solve(factors + L.gram_offset(cam), v, cw);
  else for (int c = 0; c < cw; ++c) v[c] /= sqrt(lambda);
  for (int c = 0; c < cw; ++c) x[cam * cw + c] = v[c];
}
// b = L_c v (kind 1 probes: right-hand sides of S z = L y_hat) and x_hat = L_c^T z.
template <class TS>
__global__ void k_mul_l(Layout L, const uint8_t* observed, const TS* factors, double lambda, const float* v, double* b) {
  const int64_t cam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cam >= L.nC) return;
  const int cw = L.cw;
  const TS* l = factors + L.gram_offset(cam);
  for (int i = 0; i < cw; ++i) {
    double s = 0;
    if (observed[cam]) for (int k = 0; k <= i; ++k) s += lf(l, cw, i, k) * (double)v[cam * cw + k];
    else s = sqrt(lambda) * (double)v[cam * cw + i];
    b[cam * cw + i] = s;
  }
}
template <class TS>
__global__ void k_mul_lt(Layout L, const uint8_t* observed, const TS* factors, double lambda, const double* z,
                         float* x) {
  const int64_t cam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cam >= L.nC) return;
  const int cw = L.cw;
  const TS* l = factors + L.gram_offset(cam);
  for (int i = 0; i < cw; ++i) {
    double s = 0;
    if (observed[cam]) for (int k = i; k < cw; ++k) s += lf(l, cw, k, i) * z[cam * cw + k];
    else s = sqrt(lambda) * z[cam * cw + i];
    x[cam * cw + i] = (float)s;
  }
}

template <class TS>
__global__ void k_whiten(Layout L, const uint8_t* observed, const TS* factors, double lambda, const double* y,
                         float* yh) {
  const int64_t cam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cam >= L.nC) return;
  const int cw = L.cw;
  double v[GNN_MAX_CW];
  for (int c = 0; c < cw; ++c) v[c] = y[cam * cw + c];
  if (observed[cam]) fwd_solve(factors + L.gram_offset(cam), v, cw);
  else for (int c = 0; c < cw; ++c) v[c] /= sqrt(lambda);
  for (int c = 0; c < cw; ++c) yh[cam * cw + c] = (float)v[c];
}

}  // namespace

// One training system: node features, covisibility (bf16), whitened probes.
struct GnnSystem {
  int64_t C = 0, observed = 0;
  int cw = 0, K = 0;
  double lambda = 0;
  DBuf<float> X0, PX, PY;
  DBuf<__nv_bfloat16> A;
  DBuf<uint8_t> mask;
};

class Gnn {
 public:
  int dev = 0, nsm = 148;
  cudaStream_t st = nullptr;
  PLayout P;
  DBuf<float> w, grad, am, av;
  DBuf<__nv_bfloat16> wbf;
  int64_t step = 0;
  std::vector<std::unique_ptr<GnnSystem>> systems;
  GnnSystem live;  // inference system of the attached backend
  // activations / gradients, sized to the largest C seen
  int64_t cap = 0;
  DBuf<float> Z[NLAYER + 1], HA[NLAYER], H3, O, dO, dHa, dHb, dA, dZ, adj, edgeK;
  DBuf<double> dloss;
  DBuf<unsigned> dcount;
  HBuf<double> hloss;
  HBuf<unsigned> hcount;
  std::mt19937_64 order_rng;

  fg_status init(uint64_t seed, int device) {
    dev = device;
    FG_TRY(select_device(dev));
    FG_TRY(device_stream(dev, &st));
    nsm = sm_count(dev);
    FG_TRY(w.resize(P.total));
    FG_TRY(grad.resize(P.total));
    FG_TRY(am.resize(P.total));
    FG_TRY(av.resize(P.total));
    FG_TRY(wbf.resize(P.total));
    FG_TRY(dloss.resize(1));
    FG_TRY(dcount.resize(1));
    FG_TRY(hloss.resize(1));
    FG_TRY(hcount.resize(1));
    order_rng.seed(seed ^ 0x5DEECE66Dull);
    // He-style initialization; the output layer starts at zero so the
    // untrained network is exactly block-Jacobi (times 1 + eps).
    std::vector<float> h(P.total, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (size_t i = 0; i < (size_t)NF * NH; ++i) h[P.w_in + i] = (float)(nd(rng) * std::sqrt(2.0 / NF));
    for (int l = 0; l < NLAYER; ++l)
      for (size_t i = 0; i < (size_t)2 * NH * NH; ++i) h[P.w[l] + i] = (float)(nd(rng) * 0.5 * std::sqrt(2.0 / (2 * NH)));
    return set_parameters(h.data());
  }

  fg_status set_parameters(const float* h) {
    FG_TRY(select_device(dev));
    FG_CUDA(cudaMemcpyAsync(w.get(), h, P.total * sizeof(float), cudaMemcpyHostToDevice, st));
    FG_CUDA(cudaMemsetAsync(am.get(), 0, P.total * sizeof(float), st));
    FG_CUDA(cudaMemsetAsync(av.get(), 0, P.total * sizeof(float), st));
    FG_LAUNCH(k_to_bf16, grid_for(P.total, 256), 256, 0, st, (int64_t)P.total, w.get(), wbf.get());
    FG_CUDA(cudaStreamSynchronize(st));
    step = 0;
    return FG_OK;
  }

  fg_status reserve(int64_t C) {
    if (C <= cap) return FG_OK;
    for (auto& z : Z) FG_TRY(z.resize(C * NH));
    for (auto& h : HA) FG_TRY(h.resize(C * 2 * NH));
    for (DBuf<float>* b : {&H3, &O, &dO, &dHa, &dHb, &dA, &dZ}) FG_TRY(b->resize(C * NH));
    cap = C;
    return FG_OK;
  }

  // ---- features of a Schur view into sys (X0, A, mask)
  template <class TS>
  fg_status features_t(const SchurView& v, GnnSystem& s) {
    const Layout& L = v.L;
    const int64_t C = L.nC;
    s.C = C;
    s.cw = L.cw;
    s.lambda = v.lambda;
    FG_TRY(s.X0.resize(C * NF));
    FG_TRY(s.A.resize(std::max<int64_t>(C * C, 1)));
    FG_TRY(s.mask.resize(std::max<int64_t>(C, 1)));
    FG_TRY(adj.resize(std::max<int64_t>(C * C, 1)));
    FG_TRY(edgeK.resize(std::max<int64_t>(v.nedges * 16, 1)));
    const TS* fac = (const TS*)v.factors;
    const TS* cr = (const TS*)v.cross;
    FG_LAUNCH(k_node_features<TS>, grid_for((size_t)C * 32, 128), 128, 0, st, L, v.cam_edge_off, v.cam_edge, v.edges,
              cr, v.observed, fac, v.lambda, s.X0.get(), s.mask.get());
    FG_CUDA(cudaMemsetAsync(adj.get(), 0, (size_t)C * C * sizeof(float), st));
    if (v.nedges) {
      FG_LAUNCH(k_edge_k<TS>, grid_for(v.nedges, 128), 128, 0, st, L, v.nedges, v.edges, cr, v.observed, fac,
                v.lambda, edgeK.get());
      if (L.nP)
        FG_LAUNCH(k_pairs, grid_for((size_t)L.nP * 32, 128), 128, 0, st, (int64_t)L.nP, C, v.pt_edge_off, v.pt_edge,
                  v.edges, edgeK.get(), L.pw, adj.get());
    }
    FG_LAUNCH(k_normalize, (unsigned)C, 256, 0, st, C, adj.get(), s.mask.get(), s.X0.get(), s.A.get());
    return FG_OK;
  }
  fg_status features(const SchurView& v, GnnSystem& s) {
    return v.f64 ? features_t<double>(v, s) : features_t<float>(v, s);
  }

  // ---- network
  fg_status forward(const GnnSystem& s) {
    const int C = (int)s.C;
    FG_TRY(reserve(s.C));
    const __nv_bfloat16* W = wbf.get();
    Epi e0;
    e0.bias = w.get() + P.b_in;
    e0.z = Z[0].get();
    e0.ldz = NH;
    e0.h = HA[0].get();
    e0.ldh = 2 * NH;
    FG_TRY((gemm<float, __nv_bfloat16, false, false, EPI_BIAS_RELU>(st, nsm, C, NH, NF, s.X0.get(), NF, W + P.w_in, NH,
                                                                     nullptr, 0, e0, false)));
    for (int l = 0; l < NLAYER; ++l) {
      Epi ea;
      FG_TRY((gemm<__nv_bfloat16, float, false, false, EPI_STORE>(st, nsm, C, NH, C, s.A.get(), C, HA[l].get(), 2 * NH,
                                                                   HA[l].get() + NH, 2 * NH, ea, true)));
      Epi ez;
      ez.bias = w.get() + P.b[l];
      ez.z = Z[l + 1].get();
      ez.ldz = NH;
      ez.h = l + 1 < NLAYER ? HA[l + 1].get() : H3.get();
      ez.ldh = l + 1 < NLAYER ? 2 * NH : NH;
      ez.r = HA[l].get();
      ez.ldr = 2 * NH;
      FG_TRY((gemm<float, __nv_bfloat16, false, false, EPI_BIAS_RELU>(st, nsm, C, NH, 2 * NH, HA[l].get(), 2 * NH,
                                                                       W + P.w[l], NH, nullptr, 0, ez, false)));
    }
    Epi eo;
    eo.bias = w.get() + P.b_out;
    FG_TRY((gemm<float, __nv_bfloat16, false, false, EPI_BIAS>(st, nsm, C, NH, NH, H3.get(), NH, W + P.w_out, NH,
                                                                O.get(), NH, eo, false)));
    return FG_OK;
  }

  // loss of s (accumulated into dloss) and dO
  fg_status head_loss(const GnnSystem& s) {
    const double inv_kn = 1.0 / ((double)std::max<int>(s.K, 1) * (double)std::max<int64_t>(s.observed * s.cw, 1));
    FG_LAUNCH(k_head_loss, grid_for(s.C, 128), 128, 0, st, s.C, s.cw, s.K, O.get(), s.PX.get(), s.PY.get(),
              s.mask.get(), inv_kn, dO.get(), dloss.get());
    return FG_OK;
  }
  fg_status backward(const GnnSystem& s) {
    const int C = (int)s.C;
    const __nv_bfloat16* W = wbf.get();
    float* G = grad.get();
    Epi none;
    // output layer
    FG_TRY((gemm<float, float, true, false, EPI_STORE>(st, nsm, NH, NH, C, H3.get(), NH, dO.get(), NH, G + P.w_out,
                                                        NH, none, true)));
    FG_LAUNCH(k_colsum, 1, 256, 0, st, C, dO.get(), NH, G + P.b_out);
    Epi em;
    em.zmask = Z[NLAYER].get();
    em.ldzm = NH;
    em.d2 = dZ.get();
    em.ldd2 = NH;
    FG_TRY((gemm<float, __nv_bfloat16, false, true, EPI_STORE_MASK>(st, nsm, C, NH, NH, dO.get(), NH, W + P.w_out, NH,
                                                                     dHa.get(), NH, em, false)));
    float* dh = dHa.get();
    float* dh2 = dHb.get();
    for (int l = NLAYER - 1; l >= 0; --l) {
      FG_TRY((gemm<float, float, true, false, EPI_STORE>(st, nsm, 2 * NH, NH, C, HA[l].get(), 2 * NH, dZ.get(), NH,
                                                          G + P.w[l], NH, none, true)));
      FG_LAUNCH(k_colsum, 1, 256, 0, st, C, dZ.get(), NH, G + P.b[l]);
      Epi es;
      es.split_at = NH;
      es.r = dh;
      es.ldr = NH;
      es.h = dA.get();
      es.ldh = NH;
      FG_TRY((gemm<float, __nv_bfloat16, false, true, EPI_SPLIT>(st, nsm, C, 2 * NH, NH, dZ.get(), NH, W + P.w[l], NH,
                                                                  dh2, NH, es, false)));
      Epi acc;
      acc.accumulate = 1;
      FG_TRY((gemm<__nv_bfloat16, float, true, false, EPI_STORE>(st, nsm, C, NH, C, s.A.get(), C, dA.get(), NH, dh2,
                                                                  NH, acc, true)));
      FG_LAUNCH(k_relu_mask, grid_for((size_t)C * NH, 256), 256, 0, st, (int64_t)C * NH, dh2, Z[l].get(), dZ.get());
      std::swap(dh, dh2);
    }
    FG_TRY((gemm<float, float, true, false, EPI_STORE>(st, nsm, NF, NH, C, s.X0.get(), NF, dZ.get(), NH, G + P.w_in,
                                                        NH, none, true)));
    FG_LAUNCH(k_colsum, 1, 256, 0, st, C, dZ.get(), NH, G + P.b_in);
    return FG_OK;
  }

  fg_status adam(double lr) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
    FG_LAUNCH(k_adam, grid_for(P.total, 256), 256, 0, st, (int64_t)P.total, w.get(), grad.get(), am.get(), av.get(),
              wbf.get(), (float)lr, b1, b2, 1e-8f, c1, c2);
    return FG_OK;
  }

  // ---- entry points
  template <class TS>
  fg_status precondition_t(const SchurView& v, void* minv, unsigned* nonfinite) {
    FG_TRY(features(v, live));
    FG_TRY(forward(live));
    FG_CUDA(cudaMemsetAsync(dcount.get(), 0, sizeof(unsigned), st));
    FG_LAUNCH(k_head_minv<TS>, grid_for(live.C, 64), 64, 0, st, v.L, O.get(), live.mask.get(), (const TS*)v.factors,
              (TS*)minv, dcount.get());
    FG_CUDA(cudaMemcpyAsync(hcount.get(), dcount.get(), sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    *nonfinite = hcount.get()[0];
    return FG_OK;
  }

  template <class TS>
  fg_status capture_t(const SchurView& v, size_t K, uint64_t seed, int kind, const ReducedApply& apply, double* xd,
                      double* yd, size_t* index) {
    if (!v.L.nC) {
      set_error("no retained variables to capture");
      return FG_INVALID_OPTIONS;
    }
    auto s = std::make_unique<GnnSystem>();
    FG_TRY(features(v, *s));
    const int64_t n = (int64_t)v.L.nC * v.L.cw;
    s->K = (int)K;
    FG_TRY(s->PX.resize(std::max<int64_t>(n * (int64_t)K, 1)));
    FG_TRY(s->PY.resize(std::max<int64_t>(n * (int64_t)K, 1)));
    // kind 0: x_hat Gaussian, y_hat = S_hat x_hat; kind 1: y_hat Gaussian,
    // x_hat = S_hat^-1 y_hat (apply is then the backend's solve)
    float* given = kind == 0 ? s->PX.get() : s->PY.get();
    float* derived = kind == 0 ? s->PY.get() : s->PX.get();
    if (n * (int64_t)K)
      FG_LAUNCH(k_probe_fill, grid_for((size_t)(n * K), 256), 256, 0, st, n * (int64_t)K, seed, given);
    const TS* fac = (const TS*)v.factors;
    for (size_t k = 0; k < K; ++k) {
      if (kind == 0)
        FG_LAUNCH(k_unwhiten<TS>, grid_for(v.L.nC, 128), 128, 0, st, v.L, v.observed, fac, v.lambda, given + k * n,
                  xd);
      else
        FG_LAUNCH(k_mul_l<TS>, grid_for(v.L.nC, 128), 128, 0, st, v.L, v.observed, fac, v.lambda, given + k * n, xd);
      FG_TRY(apply(xd, yd));
      if (kind == 0)
        FG_LAUNCH(k_whiten<TS>, grid_for(v.L.nC, 128), 128, 0, st, v.L, v.observed, fac, v.lambda, yd,
                  derived + k * n);
      else
        FG_LAUNCH(k_mul_lt<TS>, grid_for(v.L.nC, 128), 128, 0, st, v.L, v.observed, fac, v.lambda, yd,
                  derived + k * n);
    }
    std::vector<uint8_t> hm(v.L.nC);
    if (v.L.nC) FG_CUDA(cudaMemcpyAsync(hm.data(), s->mask.get(), v.L.nC, cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    for (uint8_t m : hm) s->observed += m ? 1 : 0;
    systems.push_back(std::move(s));
    *index = systems.size() - 1;
    return FG_OK;
  }

  fg_status train(size_t steps, double lr, double* mean_loss) {
    if (systems.empty()) {
      set_error("no training systems captured");
      return FG_INVALID_OPTIONS;
    }
    FG_TRY(select_device(dev));
    FG_CUDA(cudaMemsetAsync(dloss.get(), 0, sizeof(double), st));
    std::vector<size_t> order(systems.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    size_t pos = order.size();
    for (size_t s = 0; s < steps; ++s) {
      if (pos == order.size()) {
        std::shuffle(order.begin(), order.end(), order_rng);
        pos = 0;
      }
      const GnnSystem& sys = *systems[order[pos++]];
      FG_TRY(forward(sys));
      FG_TRY(head_loss(sys));
      FG_TRY(backward(sys));
      FG_TRY(adam(lr));
    }
    FG_CUDA(cudaMemcpyAsync(hloss.get(), dloss.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    *mean_loss = steps ? hloss.get()[0] / (double)steps : 0.0;
    return FG_OK;
  }

  fg_status evaluate(size_t index, double* loss, float* gradient, float* outputs) {
    if (index >= systems.size()) {
      set_error("system index out of range");
      return FG_INVALID_OPTIONS;
    }
    FG_TRY(select_device(dev));
    const GnnSystem& sys = *systems[index];
    FG_CUDA(cudaMemsetAsync(dloss.get(), 0, sizeof(double), st));
    FG_TRY(forward(sys));
    FG_TRY(head_loss(sys));
    if (gradient) FG_TRY(backward(sys));
    FG_CUDA(cudaMemcpyAsync(hloss.get(), dloss.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    if (gradient) FG_CUDA(cudaMemcpyAsync(gradient, grad.get(), P.total * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (outputs && sys.C)
      FG_CUDA(cudaMemcpyAsync(outputs, O.get(), (size_t)sys.C * NH * sizeof(float), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    *loss = hloss.get()[0];
    return FG_OK;
  }
};

}  // namespace fg

struct fg_gnn {
  fg::Gnn impl;
};

namespace fg {

fg_status gnn_check(const fg_gnn* g, size_t cw, size_t pw, size_t cameras, int device) {
  if (!g) return FG_OK;
  if (cw > (size_t)GNN_MAX_CW || pw > (size_t)GNN_MAX_PW || cw == 0 || pw == 0) {
    set_error("the learned preconditioner supports retained widths <= 9 and eliminated widths <= 4");
    return FG_UNSUPPORTED_STRUCTURE;
  }
  if ((int64_t)cameras > GNN_MAX_CAMERAS) {
    set_error("the learned preconditioner supports at most 16384 retained variables");
    return FG_UNSUPPORTED_STRUCTURE;
  }
  if (g->impl.dev != device) {
    set_error("the network and the backend live on different devices");
    return FG_INVALID_OPTIONS;
  }
  return FG_OK;
}

fg_status gnn_precondition(fg_gnn* g, const SchurView& v, void* minv, cudaStream_t, unsigned* nonfinite) {
  *nonfinite = 0;
  if (!v.L.nC) return FG_OK;
  return v.f64 ? g->impl.precondition_t<double>(v, minv, nonfinite)
               : g->impl.precondition_t<float>(v, minv, nonfinite);
}

fg_status gnn_capture(fg_gnn* g, const SchurView& v, size_t probes, uint64_t seed, int kind,
                      const ReducedApply& apply, double* x_dev, double* y_dev, cudaStream_t, size_t* index) {
  return v.f64 ? g->impl.capture_t<double>(v, probes, seed, kind, apply, x_dev, y_dev, index)
               : g->impl.capture_t<float>(v, probes, seed, kind, apply, x_dev, y_dev, index);
}

}  // namespace fg

using fg::set_error;

FG_API fg_status fg_gnn_create(uint64_t seed, int device, fg_gnn** out) {
  if (!out) {
    set_error("null output");
    return FG_NULL_ARGUMENT;
  }
  *out = nullptr;
  auto* g = new (std::nothrow) fg_gnn();
  if (!g) {
    set_error("host allocation failed");
    return FG_OUT_OF_MEMORY;
  }
  fg_status s = g->impl.init(seed, device);
  if (s != FG_OK) {
    delete g;
    return s;
  }
  *out = g;
  return FG_OK;
}

FG_API void fg_gnn_destroy(fg_gnn* g) {
  if (!g) return;
  fg::select_device(g->impl.dev);
  cudaStreamSynchronize(g->impl.st);
  delete g;
}

FG_API fg_status fg_gnn_parameter_count(const fg_gnn* g, size_t* count) {
  if (!g || !count) {
    set_error("null argument");
    return FG_NULL_ARGUMENT;
  }
  *count = g->impl.P.total;
  return FG_OK;
}

FG_API fg_status fg_gnn_get_parameters(fg_gnn* g, float* out) {
  if (!g || !out) {
    set_error("null argument");
    return FG_NULL_ARGUMENT;
  }
  FG_TRY(fg::select_device(g->impl.dev));
  FG_CUDA(cudaMemcpyAsync(out, g->impl.w.get(), g->impl.P.total * sizeof(float), cudaMemcpyDeviceToHost, g->impl.st));
  FG_CUDA(cudaStreamSynchronize(g->impl.st));
  return FG_OK;
}

FG_API fg_status fg_gnn_set_parameters(fg_gnn* g, const float* in) {
  if (!g || !in) {
    set_error("null argument");
    return FG_NULL_ARGUMENT;
  }
  return g->impl.set_parameters(in);
}

FG_API fg_status fg_gnn_system_count(const fg_gnn* g, size_t* count) {
  if (!g || !count) {
    set_error("null argument");
    return FG_NULL_ARGUMENT;
  }
  *count = g->impl.systems.size();
  return FG_OK;
}

FG_API fg_status fg_gnn_system_size(const fg_gnn* g, size_t index, size_t* cameras, size_t* width, size_t* probes) {
  if (!g || index >= g->impl.systems.size()) {
    set_error("system index out of range");
    return FG_INVALID_OPTIONS;
  }
  const fg::GnnSystem& s = *g->impl.systems[index];
  if (cameras) *cameras = (size_t)s.C;
  if (width) *width = (size_t)s.cw;
  if (probes) *probes = (size_t)s.K;
  return FG_OK;
}

FG_API fg_status fg_gnn_export_system(fg_gnn* g, size_t index, float* features, float* adjacency, float* probe_x,
                                      float* probe_y, uint8_t* mask, double* damping) {
  if (!g || index >= g->impl.systems.size()) {
    set_error("system index out of range");
    return FG_INVALID_OPTIONS;
  }
  FG_TRY(fg::select_device(g->impl.dev));
  cudaStream_t st = g->impl.st;
  const fg::GnnSystem& s = *g->impl.systems[index];
  const size_t C = (size_t)s.C, n = C * s.cw * (size_t)s.K;
  if (features && C) FG_CUDA(cudaMemcpyAsync(features, s.X0.get(), C * fg::NF * sizeof(float), cudaMemcpyDeviceToHost, st));
  if (adjacency && C) {
    std::vector<__nv_bfloat16> tmp(C * C);
    FG_CUDA(cudaMemcpyAsync(tmp.data(), s.A.get(), C * C * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < C * C; ++i) adjacency[i] = __bfloat162float(tmp[i]);
  }
  if (probe_x && n) FG_CUDA(cudaMemcpyAsync(probe_x, s.PX.get(), n * sizeof(float), cudaMemcpyDeviceToHost, st));
  if (probe_y && n) FG_CUDA(cudaMemcpyAsync(probe_y, s.PY.get(), n * sizeof(float), cudaMemcpyDeviceToHost, st));
  if (mask && C) FG_CUDA(cudaMemcpyAsync(mask, s.mask.get(), C, cudaMemcpyDeviceToHost, st));
  if (damping) *damping = s.lambda;
  FG_CUDA(cudaStreamSynchronize(st));
  return FG_OK;
}

FG_API fg_status fg_gnn_import_system(fg_gnn* g, size_t cameras, size_t width, size_t probes, const float* features,
                                      const float* adjacency, const float* probe_x, const float* probe_y,
                                      const uint8_t* mask, size_t* index) {
  if (!g || !index || (cameras && (!features || !adjacency || !mask)) ||
      (cameras * width * probes && (!probe_x || !probe_y))) {
    set_error("null argument");
    return FG_NULL_ARGUMENT;
  }
  if (width == 0 || width > (size_t)fg::GNN_MAX_CW || (int64_t)cameras > fg::GNN_MAX_CAMERAS) {
    set_error("system sizes out of range");
    return FG_INVALID_OPTIONS;
  }
  fg::Gnn& G = g->impl;
  FG_TRY(fg::select_device(G.dev));
  auto s = std::make_unique<fg::GnnSystem>();
  const size_t C = cameras, n = C * width * probes;
  s->C = (int64_t)C;
  s->cw = (int)width;
  s->K = (int)probes;
  FG_TRY(s->X0.resize(std::max<size_t>(C * fg::NF, 1)));
  FG_TRY(s->A.resize(std::max<size_t>(C * C, 1)));
  FG_TRY(s->mask.resize(std::max<size_t>(C, 1)));
  FG_TRY(s->PX.resize(std::max<size_t>(n, 1)));
  FG_TRY(s->PY.resize(std::max<size_t>(n, 1)));
  std::vector<__nv_bfloat16> tmp(C * C);
  for (size_t i = 0; i < C * C; ++i) tmp[i] = __float2bfloat16_rn(adjacency[i]);
  if (C) {
    FG_CUDA(cudaMemcpyAsync(s->X0.get(), features, C * fg::NF * sizeof(float), cudaMemcpyHostToDevice, G.st));
    FG_CUDA(cudaMemcpyAsync(s->A.get(), tmp.data(), C * C * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, G.st));
    FG_CUDA(cudaMemcpyAsync(s->mask.get(), mask, C, cudaMemcpyHostToDevice, G.st));
  }
  if (n) {
    FG_CUDA(cudaMemcpyAsync(s->PX.get(), probe_x, n * sizeof(float), cudaMemcpyHostToDevice, G.st));
    FG_CUDA(cudaMemcpyAsync(s->PY.get(), probe_y, n * sizeof(float), cudaMemcpyHostToDevice, G.st));
  }
  FG_CUDA(cudaStreamSynchronize(G.st));
  for (size_t i = 0; i < C; ++i) s->observed += mask[i] ? 1 : 0;
  G.systems.push_back(std::move(s));
  *index = G.systems.size() - 1;
  return FG_OK;
}

FG_API fg_status fg_gnn_clear_systems(fg_gnn* g) {
  if (!g) {
    set_error("null argument");
    return FG_NULL_ARGUMENT;
  }
  fg::select_device(g->impl.dev);
  cudaStreamSynchronize(g->impl.st);
  g->impl.systems.clear();
  return FG_OK;
}

FG_API fg_status fg_gnn_evaluate(fg_gnn* g, size_t index, double* loss, float* gradient, float* outputs) {
  if (!g || !loss) {
    set_error("null argument");
    return FG_NULL_ARGUMENT;
  }
  return g->impl.evaluate(index, loss, gradient, outputs);
}

FG_API fg_status fg_gnn_train(fg_gnn* g, size_t steps, double learning_rate, double* mean_loss) {
  if (!g || !mean_loss || !(learning_rate > 0) || !std::isfinite(learning_rate)) {
    set_error("invalid training arguments");
    return FG_INVALID_OPTIONS;
  }
  return g->impl.train(steps, learning_rate, mean_loss);
}
