// Retained-variable (camera) reductions: one warp per variable, lanes striding
// over the variable's Jacobian blocks or Schur edges. A BAL camera carries
// ~1,100 blocks, so these replace the per-coordinate loops used for points.
#pragma once
#include "kernels.cuh"

namespace fg {

__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

enum CamJtMode { CAM_GRADIENT = 0, CAM_SQUARES = 1, CAM_NORMAL = 2 };

// out[cam*cw + c] = sum over the camera's blocks of
//   GRADIENT: sum_i J[i,c] * r[row+i]                   (r = -negres)
//   SQUARES : sqrt(sum_i J[i,c]^2)                      (raw column norms)
//   NORMAL  : sum_i J[i,c] * (jd[row+i] - negres[row+i]) (J^T (J delta + r))
template <int CW, class TS, int MODE>
__global__ void k_cam_jt(Layout L, const int64_t* var_off, const int64_t* var_blk, const DBlockMeta* blocks,
                         const TS* values, const double* negres, const double* jd, double* out) {
  const int cw = CW ? CW : L.cw;
  constexpr int CM = CW ? CW : MAXW;
  int lane = threadIdx.x & 31;
  int64_t cam = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (cam >= L.nC) return;
  double acc[CM];
  for (int c = 0; c < cw; ++c) acc[c] = 0;
  for (int64_t k = var_off[cam] + lane; k < var_off[cam + 1]; k += 32) {
    DBlockMeta b = blocks[var_blk[k]];
    for (int i = 0; i < b.rows; ++i) {
      double v;
      if (MODE == CAM_GRADIENT) v = -negres[b.row + i];
      else if (MODE == CAM_NORMAL) v = jd[b.row + i] - negres[b.row + i];
      else v = 0;
      const TS* col = values + b.start + i;
      for (int c = 0; c < cw; ++c) {
        double j = (double)col[(int64_t)c * b.rows];
        acc[c] += MODE == CAM_SQUARES ? j * j : j * v;
      }
    }
  }
  for (int c = 0; c < cw; ++c) acc[c] = warp_allsum(acc[c]);
  if (lane < cw) {
    double a = acc[0];
    for (int c = 1; c < cw; ++c)
      if (c == lane) a = acc[c];
    out[cam * cw + lane] = MODE == CAM_SQUARES ? sqrt(a) : a;
  }
}

// Normalized Gram blocks of retained variables (block_factors.rs:87-99),
// lower triangle column major, one warp per variable.
template <int CW, class TS>
__global__ void k_cam_gram(Layout L, const int64_t* var_off, const int64_t* var_blk, const DBlockMeta* blocks,
                           const TS* values, const double* scales, TS* gram) {
  const int cw = CW ? CW : L.cw;
  constexpr int CM = CW ? CW : MAXW;
  constexpr int NL = CM * (CM + 1) / 2;
  int lane = threadIdx.x & 31;
  int64_t cam = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (cam >= L.nC) return;
  double acc[NL];
  const int nl = cw * (cw + 1) / 2;
  for (int k = 0; k < nl; ++k) acc[k] = 0;
  double inv[CM];
  for (int c = 0; c < cw; ++c) inv[c] = 1.0 / scales[cam * cw + c];
  for (int64_t k = var_off[cam] + lane; k < var_off[cam + 1]; k += 32) {
    DBlockMeta b = blocks[var_blk[k]];
    for (int i = 0; i < b.rows; ++i) {
      double jv[CM];
      for (int c = 0; c < cw; ++c) jv[c] = (double)values[b.start + (int64_t)c * b.rows + i] * inv[c];
      int idx = 0;
      for (int c = 0; c < cw; ++c)
        for (int r = c; r < cw; ++r) acc[idx++] += jv[c] * jv[r];
    }
  }
  int idx = 0;
  TS* g = gram + L.gram_offset(cam);
  for (int c = 0; c < cw; ++c)
    for (int r = c; r < cw; ++r) {
      double v = warp_allsum(acc[idx]);
      if (lane == (idx & 31)) g[c * cw + r] = (TS)v;
      ++idx;
    }
}

// Exact diagonal blocks of the reduced system for the Schur-diagonal
// preconditioner: S_cc = lambda I + B_c - sum_{e in c} E_e C_p^-1 E_e^T,
// factored in place; falls back to the (B + lambda I) factor when S_cc does
// not factor. One warp per retained variable.
template <int CW, int PW, class TS>
__global__ void k_cam_schur_diag(Layout L, const int64_t* cam_edge_off, const int64_t* cam_edge,
                                 const DEdgeMeta* edges, const TS* cross, const uint8_t* observed, const TS* gram,
                                 const TS* factors, TS* precond, double lambda) {
  const int cw = CW ? CW : L.cw, pw = PW ? PW : L.pw;
  constexpr int CM = CW ? CW : MAXW;
  constexpr int PM = PW ? PW : MAXW;
  constexpr int NL = CM * (CM + 1) / 2;
  int lane = threadIdx.x & 31;
  int64_t cam = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (cam >= L.nC) return;
  int64_t go = L.gram_offset(cam);
  if (!observed[cam]) return;
  double acc[NL];
  const int nl = cw * (cw + 1) / 2;
  for (int k = 0; k < nl; ++k) acc[k] = 0;
  for (int64_t k = cam_edge_off[cam] + lane; k < cam_edge_off[cam + 1]; k += 32) {
    int64_t e = cam_edge[k];
    int pt = edges[e].pt;
    const TS* E = cross + e * (int64_t)cw * pw;
    bool obs = observed[L.nC + pt];
    const TS* lc = factors + L.gram_offset(L.nC + pt);
    double y[CM * PM];
    for (int c = 0; c < cw; ++c) {
      double b[PM];
      for (int p = 0; p < pw; ++p) b[p] = (double)E[p * cw + c];
      if (obs) llt_solve<PW, TS, double>(lc, b, pw);
      else if (lambda != 0) for (int p = 0; p < pw; ++p) b[p] /= lambda;
      for (int p = 0; p < pw; ++p) y[c * pw + p] = b[p];
    }
    int idx = 0;
    for (int c = 0; c < cw; ++c)
      for (int r = c; r < cw; ++r) {
        double s = 0;
        for (int p = 0; p < pw; ++p) s += (double)E[p * cw + r] * y[c * pw + p];
        acc[idx++] += s;
      }
  }
  for (int k = 0; k < nl; ++k) acc[k] = warp_allsum(acc[k]);
  if (lane != 0) return;
  double s[CM * CM];
  int idx = 0;
  for (int c = 0; c < cw; ++c)
    for (int r = 0; r < cw; ++r) s[c * cw + r] = 0;
  for (int c = 0; c < cw; ++c)
    for (int r = c; r < cw; ++r) {
      s[c * cw + r] = (double)gram[go + c * cw + r] + (r == c ? lambda : 0.0) - acc[idx];
      ++idx;
    }
  bool ok = chol_inplace<CW>(s, cw);
  for (int c = 0; c < cw; ++c)
    for (int r = 0; r < cw; ++r)
      precond[go + c * cw + r] = ok ? (TS)(r >= c ? s[c * cw + r] : 0.0) : factors[go + c * cw + r];
}

}  // namespace fg
