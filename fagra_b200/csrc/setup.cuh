// Per-linearization setup kernels: column scales with their floor, normalized
// Gram blocks, J^T v reductions and the cross-block edge records, fused so each
// pass reads the Jacobian once. Nonfinite values raise a device flag that the
// host reads once per prepare_damping (src/linear_model.rs:225 and
// src/schur.rs:520 reject them with InvalidEvaluation).
#pragma once
#include "kernels.cuh"
#include "fastpath.cuh"

namespace fg {

template <int N>
__device__ __forceinline__ void block_allsums(double (&v)[N], double* sh /* >= 32*N */) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < N; ++k) sh[warp * N + k] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double s = 0;
    for (int w = 0; w < nw; ++w) s += sh[w * N + k];
    v[k] = s;
  }
  __syncthreads();
}

// One block per retained variable: raw column norms (hypot chain of
// src/linear_model.rs:217-224), floored scales, and the normalized Gram block
// (block_factors.rs:87-99), all from the variable's blocks in ONE pass: the raw
// Gram sum_i J_i^T J_i is accumulated and normalized afterwards,
// G_rc = raw_rc / (d_r d_c), its diagonal giving the squared column norms.
// Each thread walks four of the variable's blocks at a time so four
// index -> block -> value load chains are in flight.
template <int CW, class TS>
__global__ void k_cam_scales_gram(Layout L, const int64_t* var_off, const int64_t* var_blk, const DBlockMeta* blocks,
                                  const TS* values, double floor, double* scales, TS* gram, int* bad) {
  constexpr int CM = CW ? CW : MAXW;
  constexpr int NL = CM * (CM + 1) / 2;
  constexpr int U = 4;
  const int cw = CW ? CW : L.cw;
  __shared__ double sh[32 * NL];
  const int64_t cam = blockIdx.x;
  if (cam >= L.nC) return;
  const int64_t b0 = var_off[cam], b1 = var_off[cam + 1];
  double acc[NL];
#pragma unroll
  for (int k = 0; k < NL; ++k) acc[k] = 0;
  for (int64_t k0 = b0 + threadIdx.x; k0 < b1; k0 += U * (int64_t)blockDim.x) {
    DBlockMeta bm[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t k = k0 + u * (int64_t)blockDim.x;
      if (k < b1) bm[u] = blocks[var_blk[k]];
      else bm[u].rows = 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      for (int i = 0; i < bm[u].rows; ++i) {
        double jv[CM];
#pragma unroll
        for (int c = 0; c < CM; ++c)
          jv[c] = c < cw ? (double)values[bm[u].start + (int64_t)c * bm[u].rows + i] : 0.0;
        int idx = 0;
#pragma unroll
        for (int c = 0; c < CM; ++c)
#pragma unroll
          for (int r = c; r < CM; ++r) acc[idx++] += jv[c] * jv[r];
      }
    }
  }
  block_allsums<NL>(acc, sh);
  double d[CM];
  int idx = 0;
#pragma unroll
  for (int c = 0; c < CM; ++c) {
    if (c < cw) {
      const double raw = sqrt(acc[idx]);  // diagonal entry (c, c)
      if (!isfinite(raw) && threadIdx.x == 0) atomicOr(bad, 1);
      d[c] = fmax(raw, floor);
      if (threadIdx.x == 0) scales[cam * cw + c] = d[c];
    } else {
      d[c] = 1.0;
    }
    idx += CM - c;
  }
  TS* g = gram + L.gram_offset(cam);
  idx = 0;
#pragma unroll
  for (int c = 0; c < CM; ++c)
#pragma unroll
    for (int r = c; r < CM; ++r) {
      if (c < cw && r < cw && threadIdx.x == (idx & (blockDim.x - 1))) g[c * cw + r] = (TS)(acc[idx] / (d[c] * d[r]));
      ++idx;
    }
}

// One thread per eliminated variable: floored scales and normalized Gram block.
template <int PW, class TS>
__global__ void k_point_scales_gram(Layout L, const int64_t* var_off, const int64_t* var_blk,
                                    const DBlockMeta* blocks, const TS* values, double floor, double* scales,
                                    TS* gram, int* bad) {
  constexpr int PM = PW ? PW : MAXW;
  const int pw = PW ? PW : L.pw;
  const int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (pt >= L.nP) return;
  const int64_t v = L.nC + pt;
  // one pass: the raw Gram, normalized afterwards (its diagonal gives the
  // squared column norms), as k_cam_scales_gram
  double acc[PM * PM];
  for (int k = 0; k < pw * pw; ++k) acc[k] = 0;
  for (int64_t k = var_off[v]; k < var_off[v + 1]; ++k) {
    DBlockMeta b = blocks[var_blk[k]];
    for (int i = 0; i < b.rows; ++i) {
      double jv[PM];
      for (int p = 0; p < pw; ++p) jv[p] = (double)values[b.start + (int64_t)p * b.rows + i];
      for (int c = 0; c < pw; ++c)
        for (int r = c; r < pw; ++r) acc[c * pw + r] += jv[c] * jv[r];
    }
  }
  double d[PM];
  const int64_t base = L.retained + pt * pw;
  for (int p = 0; p < pw; ++p) {
    double raw = sqrt(acc[p * pw + p]);
    if (!isfinite(raw)) atomicOr(bad, 1);
    d[p] = fmax(raw, floor);
    scales[base + p] = d[p];
  }
  TS* g = gram + L.gram_offset(v);
  for (int c = 0; c < pw; ++c)
    for (int r = 0; r < pw; ++r) g[c * pw + r] = (TS)(r >= c ? acc[c * pw + r] / (d[c] * d[r]) : 0.0);
}

// ---- Device BAL layout (one emission per observation k: rows 2k and 2k+1;
// values [24k, 24k+18) the camera block, [24k+18, 24k+24) the point block, each
// 2 rows column-major, so element (row i, column c) sits at 2c + i). A camera's
// emissions are contiguous; a point's are listed by pt_edge. These kernels
// replace the block-metadata walks of the generic kernels above with direct
// 16-byte (8-byte for point blocks) loads.
template <class TS>
__device__ __forceinline__ void bal_cam_block(const TS* values, int64_t k, double (&v)[18]) {
  if (sizeof(TS) == 4) {
    const float4* q = reinterpret_cast<const float4*>(values + 24 * k);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float4 a = q[i];
      v[4 * i] = a.x; v[4 * i + 1] = a.y; v[4 * i + 2] = a.z; v[4 * i + 3] = a.w;
    }
    const float2 b = *reinterpret_cast<const float2*>(values + 24 * k + 16);
    v[16] = b.x;
    v[17] = b.y;
  } else {
    const double2* q = reinterpret_cast<const double2*>(values + 24 * k);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const double2 a = q[i];
      v[2 * i] = a.x; v[2 * i + 1] = a.y;
    }
  }
}
template <class TS>
__device__ __forceinline__ void bal_pt_block(const TS* values, int64_t k, double (&v)[6]) {
  if (sizeof(TS) == 4) {
    const float2* q = reinterpret_cast<const float2*>(values + 24 * k + 18);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float2 a = q[i];
      v[2 * i] = a.x; v[2 * i + 1] = a.y;
    }
  } else {
    const double2* q = reinterpret_cast<const double2*>(values + 24 * k + 18);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double2 a = q[i];
      v[2 * i] = a.x; v[2 * i + 1] = a.y;
    }
  }
}

// A camera block's 18 values in the storage type (16-byte loads).
template <class TS>
__device__ __forceinline__ void bal_cam_raw(const TS* values, int64_t k, TS (&v)[18]) {
  if (sizeof(TS) == 4) {
    const float4* q = reinterpret_cast<const float4*>(values + 24 * k);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float4 a = q[i];
      v[4 * i] = (TS)a.x; v[4 * i + 1] = (TS)a.y; v[4 * i + 2] = (TS)a.z; v[4 * i + 3] = (TS)a.w;
    }
    const float2 b = *reinterpret_cast<const float2*>(values + 24 * k + 16);
    v[16] = (TS)b.x;
    v[17] = (TS)b.y;
  } else {
    const double2* q = reinterpret_cast<const double2*>(values + 24 * k);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const double2 a = q[i];
      v[2 * i] = (TS)a.x; v[2 * i + 1] = (TS)a.y;
    }
  }
}

// One block of 64 threads per camera over its contiguous emissions, each
// thread loading its next emission while it accumulates the current one.
// MOMENTS: the gradient J^T r (g) and the raw Gram J^T J (raw: 45 entries,
// columns c <= r in column-major lower order) in one pass; NORMAL:
// J^T (jd - negres) (out).
constexpr int BAL_MOMENTS = 0, BAL_NORMAL = 1;
constexpr int BAL_CAM_THREADS = 64;
template <class TS, int MODE>
__global__ void __launch_bounds__(BAL_CAM_THREADS) k_bal_cam_pass(int64_t ncam, const int64_t* cam_off,
                                                                  const TS* values, const double* negres,
                                                                  const double* jd, double* out, double* raw) {
  constexpr int NA = MODE == BAL_MOMENTS ? 54 : 9;
  __shared__ double sh[32 * NA];
  const int64_t cam = blockIdx.x;
  if (cam >= ncam) return;
  double acc[NA];
#pragma unroll
  for (int k = 0; k < NA; ++k) acc[k] = 0;
  const int64_t k1 = cam_off[cam + 1];
  int64_t k = cam_off[cam] + threadIdx.x;
  TS v[18];
  double2 nr = make_double2(0, 0), jj = make_double2(0, 0);
  if (k < k1) {
    bal_cam_raw<TS>(values, k, v);
    nr = *reinterpret_cast<const double2*>(negres + 2 * k);
    if (MODE == BAL_NORMAL) jj = *reinterpret_cast<const double2*>(jd + 2 * k);
  }
  while (k < k1) {
    const int64_t kn = k + BAL_CAM_THREADS;
    TS vn[18];
    double2 nrn = make_double2(0, 0), jjn = make_double2(0, 0);
    if (kn < k1) {  // the next emission's loads are in flight during this one's arithmetic
      bal_cam_raw<TS>(values, kn, vn);
      nrn = *reinterpret_cast<const double2*>(negres + 2 * kn);
      if (MODE == BAL_NORMAL) jjn = *reinterpret_cast<const double2*>(jd + 2 * kn);
    }
    double w0 = -nr.x, w1 = -nr.y;
    if (MODE == BAL_NORMAL) {
      w0 = jj.x - nr.x;
      w1 = jj.y - nr.y;
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) acc[NA - 9 + c] += (double)v[2 * c] * w0 + (double)v[2 * c + 1] * w1;
    if (MODE == BAL_MOMENTS) {
      int idx = 0;
#pragma unroll
      for (int c = 0; c < 9; ++c)
#pragma unroll
        for (int r = c; r < 9; ++r)
          acc[idx++] += (double)v[2 * c] * (double)v[2 * r] + (double)v[2 * c + 1] * (double)v[2 * r + 1];
    }
    if (kn < k1) {
#pragma unroll
      for (int i = 0; i < 18; ++i) v[i] = vn[i];
      nr = nrn;
      jj = jjn;
    }
    k = kn;
  }
  block_allsums<NA>(acc, sh);
  if (threadIdx.x == 0) {  // static indices keep acc in registers
#pragma unroll
    for (int q = 0; q < NA; ++q) {
      if (q >= NA - 9) out[cam * 9 + (q - (NA - 9))] = acc[q];
      else raw[cam * 45 + q] = acc[q];
    }
  }
}

// One thread per point over its emissions (pt_edge): gradient J^T r into
// g[retained + 3p + c] and the raw Gram (6 entries: 00, 10, 20, 11, 21, 22).
template <class TS>
__global__ void k_bal_point_moments(int64_t npt, int64_t retained, const int64_t* pt_off, const int64_t* pt_edge,
                                    const TS* values, const double* negres, double* g, double* raw) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= npt) return;
  double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t k = pt_off[p]; k < pt_off[p + 1]; ++k) {
    const int64_t e = pt_edge[k];
    double v[6];
    bal_pt_block<TS>(values, e, v);
    const double2 nr = *reinterpret_cast<const double2*>(negres + 2 * e);
#pragma unroll
    for (int c = 0; c < 3; ++c) a[6 + c] -= v[2 * c] * nr.x + v[2 * c + 1] * nr.y;
    int idx = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = c; r < 3; ++r) a[idx++] += v[2 * c] * v[2 * r] + v[2 * c + 1] * v[2 * r + 1];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) g[retained + 3 * p + c] = a[6 + c];
#pragma unroll
  for (int k = 0; k < 6; ++k) raw[6 * p + k] = a[k];
}

// Floored column scales and the normalized Gram blocks from the raw moments
// (src/linear_model.rs:211-224, block_factors.rs:87-99): one thread per
// variable, cameras then points; the blocks are written whole (column-major,
// lower triangle, zeros above).
template <int W, class TS>
__device__ __forceinline__ void bal_scale_block(const double* r, double floor, double* scales, double* inv_scales,
                                                TS* gb, int* bad) {
  double d[W], id[W];
  int idx = 0;
#pragma unroll
  for (int c = 0; c < W; ++c) {  // diagonal entries: the squared column norms
    const double n = sqrt(r[idx]);
    if (!isfinite(n)) atomicOr(bad, 1);
    d[c] = fmax(n, floor);
    id[c] = 1.0 / d[c];
    scales[c] = d[c];
    inv_scales[c] = id[c];
    idx += W - c;
  }
  idx = 0;
#pragma unroll
  for (int c = 0; c < W; ++c)
#pragma unroll
    for (int rr = 0; rr < W; ++rr) {
      if (rr < c) {
        gb[c * W + rr] = (TS)0;
      } else {
        gb[c * W + rr] = (TS)(r[idx] * id[c] * id[rr]);
        ++idx;
      }
    }
}
template <class TS>
__global__ void k_bal_scales_gram(int64_t ncam, int64_t npt, const double* raw_cam, const double* raw_pt,
                                  double floor, double* scales, double* inv_scales, TS* gram, int* bad) {
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v < ncam) {
    bal_scale_block<9, TS>(raw_cam + 45 * v, floor, scales + 9 * v, inv_scales + 9 * v, gram + 81 * v, bad);
  } else if (v < ncam + npt) {
    const int64_t p = v - ncam;
    bal_scale_block<3, TS>(raw_pt + 6 * p, floor, scales + 9 * ncam + 3 * p, inv_scales + 9 * ncam + 3 * p,
                           gram + 81 * ncam + 9 * p, bad);
  }
}

// One block per retained variable: out[cam*cw + c] = sum over its blocks of
// GRADIENT: sum_i J[i,c] r[row+i]; NORMAL: sum_i J[i,c] (jd - negres)[row+i].
template <int CW, class TS, int MODE>
__global__ void k_cam_jt_block(Layout L, const int64_t* var_off, const int64_t* var_blk, const DBlockMeta* blocks,
                               const TS* values, const double* negres, const double* jd, double* out) {
  constexpr int CM = CW ? CW : MAXW;
  const int cw = CW ? CW : L.cw;
  __shared__ double sh[32 * CM];
  const int64_t cam = blockIdx.x;
  if (cam >= L.nC) return;
  double acc[CM];
  for (int c = 0; c < CM; ++c) acc[c] = 0;
  for (int64_t k = var_off[cam] + threadIdx.x; k < var_off[cam + 1]; k += blockDim.x) {
    DBlockMeta b = blocks[var_blk[k]];
    for (int i = 0; i < b.rows; ++i) {
      double v = MODE == CAM_NORMAL ? jd[b.row + i] - negres[b.row + i] : -negres[b.row + i];
      for (int c = 0; c < cw; ++c) acc[c] += (double)values[b.start + (int64_t)c * b.rows + i] * v;
    }
  }
  block_allsums<CM>(acc, sh);
  if (threadIdx.x == 0)
    for (int c = 0; c < cw; ++c) out[cam * cw + c] = acc[c];
}

// Cross blocks E_e[p,c] = sum_rows (J_cam[:,c]/D)(J_pt[:,p]/D) (src/schur.rs:504-519),
// one thread per (point-major edge, word): word < cw*pw writes the edge
// record and the reference-layout cross array; the last word packs the
// camera and tile-local point indices. Coalesced record writes.
template <class TS>
__global__ void k_edge_records_fused(int64_t nedges, int cw, int pw, const int64_t* pt_edge, const DEdgeMeta* edges,
                                     const DBlockMeta* blocks, const TS* values, const double* scales,
                                     const uint32_t* local_point, TS* rec, TS* cross, int* bad) {
  const int W = cw * pw + 1;
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nedges * W) return;
  int64_t k = t / W;
  int w = (int)(t % W);
  int64_t e = pt_edge[k];
  DEdgeMeta ed = edges[e];
  if (w < cw * pw) {
    int p = w / cw, c = w % cw;
    DBlockMeta l = blocks[ed.lblk], r = blocks[ed.rblk];
    const TS* lc = values + l.start + (int64_t)c * l.rows;
    const TS* rp = values + r.start + (int64_t)p * r.rows;
    double dl = scales[l.col + c], dr = scales[r.col + p];
    double s = 0;
    for (int i = 0; i < l.rows; ++i) s += ((double)lc[i] / dl) * ((double)rp[i] / dr);
    if (!isfinite(s)) atomicOr(bad, 1);
    rec[t] = (TS)s;
    cross[e * (int64_t)(cw * pw) + w] = (TS)s;
  } else {
    using Wd = RecWord<TS>;
    typename Wd::U word = Wd::pack((uint32_t)ed.cam, local_point[k]);
    memcpy(&rec[t], &word, sizeof(word));
  }
}

// Edge records for the single-pass operator (BAL 9/3 shape), one thread per
// point-major edge: E_e[p,c] = sum_rows (J_cam[:,c]/D)(J_pt[:,p]/D) computed
// from the Jacobian blocks once, staged in shared memory and stored to the
// contiguous record range with coalesced writes. cross (optional) receives the
// reference layout (e*3+p)*9+c for the generic kernels that still read it.
constexpr int REC_T = 128;
template <class TS>
__global__ void __launch_bounds__(REC_T) k_edge_records2(int64_t nedges, const int64_t* pt_edge,
                                                         const DEdgeMeta* edges, const DBlockMeta* blocks,
                                                         const TS* values, const double* scales,
                                                         const uint32_t* local_point, TS* rec, TS* cross, int* bad) {
  __shared__ TS tile[REC_T * 29];
  const int64_t k0 = (int64_t)blockIdx.x * REC_T, k = k0 + threadIdx.x;
  const int nk = (int)min((int64_t)REC_T, nedges - k0);
  if (k < nedges) {
    const int64_t e = pt_edge[k];
    const DEdgeMeta ed = edges[e];
    const DBlockMeta l = blocks[ed.lblk], r = blocks[ed.rblk];
    double ic[9], ip[3];
#pragma unroll
    for (int c = 0; c < 9; ++c) ic[c] = 1.0 / scales[l.col + c];
#pragma unroll
    for (int p = 0; p < 3; ++p) ip[p] = 1.0 / scales[r.col + p];
    double E[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) E[i] = 0;
    if (l.rows == 2 && r.rows == 2 && r.start == l.start + 18 && (l.start & 3) == 0) {
      // the BAL emission layout: 24 contiguous values, 16-byte aligned
      TS v[24];
      if (sizeof(TS) == 4) {
        const float4* q = reinterpret_cast<const float4*>(values + l.start);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          const float4 a = q[i];
          v[4 * i] = (TS)a.x; v[4 * i + 1] = (TS)a.y; v[4 * i + 2] = (TS)a.z; v[4 * i + 3] = (TS)a.w;
        }
      } else {
        const double2* q = reinterpret_cast<const double2*>(values + l.start);
#pragma unroll
        for (int i = 0; i < 12; ++i) {
          const double2 a = q[i];
          v[2 * i] = (TS)a.x; v[2 * i + 1] = (TS)a.y;
        }
      }
#pragma unroll
      for (int row = 0; row < 2; ++row) {
        double jc[9], jp[3];
#pragma unroll
        for (int c = 0; c < 9; ++c) jc[c] = (double)v[2 * c + row] * ic[c];
#pragma unroll
        for (int p = 0; p < 3; ++p) jp[p] = (double)v[18 + 2 * p + row] * ip[p];
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
          for (int c = 0; c < 9; ++c) E[p * 9 + c] += jc[c] * jp[p];
      }
    } else {
      for (int row = 0; row < l.rows; ++row) {
        double jc[9], jp[3];
#pragma unroll
        for (int c = 0; c < 9; ++c) jc[c] = (double)values[l.start + (int64_t)c * l.rows + row] * ic[c];
#pragma unroll
        for (int p = 0; p < 3; ++p) jp[p] = (double)values[r.start + (int64_t)p * r.rows + row] * ip[p];
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
          for (int c = 0; c < 9; ++c) E[p * 9 + c] += jc[c] * jp[p];
      }
    }
    bool ok = true;
    TS* t = tile + threadIdx.x * 29;
#pragma unroll
    for (int i = 0; i < 27; ++i) {
      ok = ok && isfinite(E[i]);
      t[i] = (TS)E[i];
    }
    typename RecWord<TS>::U word = RecWord<TS>::pack((uint32_t)ed.cam, local_point[k]);
    memcpy(&t[27], &word, sizeof(word));
    if (!ok) atomicOr(bad, 1);
    if (cross)
      for (int i = 0; i < 27; ++i) cross[e * 27 + i] = t[i];
  }
  __syncthreads();
  TS* out = rec + k0 * 28;
  for (int i = threadIdx.x; i < nk * 28; i += REC_T) out[i] = tile[(i / 28) * 29 + (i % 28)];
}

// Edge records of the device BAL layout (as k_edge_records2, whose record
// format and arithmetic they share): the emission's 24 values with six 16-byte
// loads, its camera and point from the edge list, and the inverse column
// scales k_bal_scales_gram wrote, without the block metadata.
template <class TS>
__global__ void __launch_bounds__(REC_T) k_edge_records_bal(int64_t nedges, int64_t retained, const int64_t* pt_edge,
                                                            const DEdgeMeta* edges, const TS* values,
                                                            const double* inv_scales, const uint32_t* local_point,
                                                            TS* rec, TS* cross, int* bad) {
  __shared__ TS tile[REC_T * 29];
  const int64_t k0 = (int64_t)blockIdx.x * REC_T, k = k0 + threadIdx.x;
  const int nk = (int)min((int64_t)REC_T, nedges - k0);
  if (k < nedges) {
    const int64_t e = pt_edge[k];
    const int2 cp = *reinterpret_cast<const int2*>(edges + e);  // (camera, point)
    const double* icp = inv_scales + 9 * (int64_t)cp.x;
    const double* ipp = inv_scales + retained + 3 * (int64_t)cp.y;
    double ic[9], ip[3];
#pragma unroll
    for (int c = 0; c < 9; ++c) ic[c] = icp[c];
#pragma unroll
    for (int q = 0; q < 3; ++q) ip[q] = ipp[q];
    double v[18], w[6];
    bal_cam_block<TS>(values, e, v);
    bal_pt_block<TS>(values, e, w);
    double E[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) E[i] = 0;
#pragma unroll
    for (int row = 0; row < 2; ++row) {
      double jc[9], jp[3];
#pragma unroll
      for (int c = 0; c < 9; ++c) jc[c] = v[2 * c + row] * ic[c];
#pragma unroll
      for (int q = 0; q < 3; ++q) jp[q] = w[2 * q + row] * ip[q];
#pragma unroll
      for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int c = 0; c < 9; ++c) E[q * 9 + c] += jc[c] * jp[q];
    }
    bool ok = true;
    TS* t = tile + threadIdx.x * 29;
#pragma unroll
    for (int i = 0; i < 27; ++i) {
      ok = ok && isfinite(E[i]);
      t[i] = (TS)E[i];
    }
    typename RecWord<TS>::U word = RecWord<TS>::pack((uint32_t)cp.x, local_point[k]);
    memcpy(&t[27], &word, sizeof(word));
    if (!ok) atomicOr(bad, 1);
    if (cross)
      for (int i = 0; i < 27; ++i) cross[e * 27 + i] = t[i];
  }
  __syncthreads();
  TS* out = rec + k0 * 28;
  for (int i = threadIdx.x; i < nk * 28; i += REC_T) out[i] = tile[(i / 28) * 29 + (i % 28)];
}

// Index maps of a BAL linearization (emission k: rows 2k, 2k+1; block 2k =
// camera ocam[k] (2x9 at 24k), block 2k+1 = point opt[k] (2x3 at 24k+18)),
// written on the device from the emission arrays and their two stable orders
// (by camera and by point, from the device radix orders).
__global__ void k_bal_structure(int64_t obs, int64_t ncam, const uint32_t* ocam, const uint32_t* opt,
                                const uint32_t* cam_order, const uint32_t* pt_order, DBlockMeta* blocks,
                                DEdgeMeta* edges, int64_t* var_blk, int64_t* cam_edge, int64_t* pt_edge,
                                int64_t* emi_off) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k > obs) return;
  if (k == obs) {
    emi_off[obs] = 2 * obs;
    return;
  }
  const int64_t c = ocam[k], p = opt[k];
  blocks[2 * k] = DBlockMeta{2 * k, 24 * k, 9 * c, 2, 9};
  blocks[2 * k + 1] = DBlockMeta{2 * k, 24 * k + 18, 9 * ncam + 3 * p, 2, 3};
  edges[k] = DEdgeMeta{(int32_t)c, (int32_t)p, 2 * k, 2 * k + 1};
  emi_off[k] = 2 * k;
  const int64_t ec = cam_order[k], ep = pt_order[k];
  var_blk[k] = 2 * ec;            // camera variables first, each in emission order
  var_blk[obs + k] = 2 * ep + 1;  // then the points
  cam_edge[k] = ec;
  pt_edge[k] = ep;
}

// Device batches of bipartite emissions (fg_schur_accumulate_pairs_device):
// emission e = e0 + k of a batch of `count` emissions with `rows` rows each
// has one retained block (variable cam[k], width cw) and one eliminated block
// (variable pt[k], width pw). Inputs are SoA so that consecutive threads read
// consecutive words: residual[i * count + k], retained Jacobian element (i, j)
// at jr[(j * rows + i) * count + k], eliminated at je[(j * rows + i) * count + k].
// The pass packs the reference's layout (src/linear_model.rs:180-210: -r per
// row, each block column-major, retained block first) and checks what
// CheckedSink checks (src/optimization.rs:541-612): a variable outside the
// layout is an invalid emission (flags[0]), a nonfinite value an invalid
// evaluation (flags[1]).
template <class TS>
__global__ void k_pairs_pack(int64_t count, int rows, int cw, int pw, int64_t ncam, int64_t npt, const uint32_t* cam,
                             const uint32_t* pt, const double* r, const double* jr, const double* je, int64_t e0,
                             int64_t row0, int64_t v0, uint32_t* em_cam, uint32_t* em_pt, int64_t* em_row,
                             int64_t* em_val, int32_t* em_rows, double* negres, TS* values, int* flags) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint32_t c = cam[k], p = pt[k];
  if ((int64_t)c >= ncam || (int64_t)p >= npt) atomicExch(&flags[0], 1);
  const int64_t row = row0 + k * rows, v = v0 + k * (int64_t)rows * (cw + pw);
  bool bad = false;
  for (int i = 0; i < rows; ++i) {
    const double x = r[(int64_t)i * count + k];
    bad |= !isfinite(x);
    negres[row + i] = -x;
  }
  for (int j = 0; j < cw; ++j)
    for (int i = 0; i < rows; ++i) {
      const double x = jr[((int64_t)j * rows + i) * count + k];
      bad |= !isfinite(x);
      values[v + (int64_t)j * rows + i] = (TS)x;
    }
  const int64_t vp = v + (int64_t)rows * cw;
  for (int j = 0; j < pw; ++j)
    for (int i = 0; i < rows; ++i) {
      const double x = je[((int64_t)j * rows + i) * count + k];
      bad |= !isfinite(x);
      values[vp + (int64_t)j * rows + i] = (TS)x;
    }
  if (bad) atomicExch(&flags[1], 1);
  em_cam[e0 + k] = c;
  em_pt[e0 + k] = p;
  em_row[e0 + k] = row;
  em_val[e0 + k] = v;
  em_rows[e0 + k] = rows;
}

// Index maps of the device pair emissions (as k_bal_structure, any widths and
// rows): block 2e = retained, 2e + 1 = eliminated, edge e, variables listing
// their blocks in emission order (from the stable orders by camera and point).
__global__ void k_pairs_structure(int64_t obs, int64_t retained, int cw, int pw, const uint32_t* ocam,
                                  const uint32_t* opt, const int64_t* em_row, const int64_t* em_val,
                                  const int32_t* em_rows, const uint32_t* cam_order, const uint32_t* pt_order,
                                  DBlockMeta* blocks, DEdgeMeta* edges, int64_t* var_blk, int64_t* cam_edge,
                                  int64_t* pt_edge, int64_t* emi_off) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k > obs) return;
  if (k == obs) {
    emi_off[obs] = 2 * obs;
    return;
  }
  const int64_t c = ocam[k], p = opt[k], row = em_row[k], v = em_val[k];
  const int32_t rows = em_rows[k];
  blocks[2 * k] = DBlockMeta{row, v, cw * c, rows, cw};
  blocks[2 * k + 1] = DBlockMeta{row, v + (int64_t)rows * cw, retained + pw * p, rows, pw};
  edges[k] = DEdgeMeta{(int32_t)c, (int32_t)p, 2 * k, 2 * k + 1};
  emi_off[k] = 2 * k;
  const int64_t ec = cam_order[k], ep = pt_order[k];
  var_blk[k] = 2 * ec;
  var_blk[obs + k] = 2 * ep + 1;
  cam_edge[k] = ec;
  pt_edge[k] = ep;
}

// flag = 1 if the emissions' cameras, points or rows differ from `prev`
// (cameras | points | rows, each n long).
__global__ void k_pairs_differ(int64_t n, const uint32_t* cam, const uint32_t* pt, const uint32_t* rows,
                               const uint32_t* prev, int* flag) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (cam[k] != prev[k] || pt[k] != prev[n + k] || rows[k] != prev[2 * n + k]) *flag = 1;
}

// Variable offsets of the BAL structure (cameras, then points; every variable
// lists its emissions) and which variables any emission touches.
__global__ void k_bal_var_offsets(int64_t ncam, int64_t npt, int64_t obs, const int64_t* cam_off,
                                  const int64_t* pt_off, int64_t* var_off, uint8_t* observed) {
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v > ncam + npt) return;
  auto at = [&](int64_t u) { return u <= ncam ? cam_off[u] : obs + pt_off[u - ncam]; };
  const int64_t o = at(v);
  var_off[v] = o;
  if (v < ncam + npt) observed[v] = at(v + 1) > o;
}

}  // namespace fg
