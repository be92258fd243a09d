// Learned block preconditioner: a message-passing network over the camera
// covisibility graph of the reduced camera system, with BF16 tensor-core GEMMs
// (tcgen05.mma, FP32 accumulation in tensor memory) for inference and training, Adam on
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
#include "umma.cuh"
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
// B(k,n) = TRB ? B[n*ldb+k] : B[k*ldb+n], on the fifth-generation tensor cores:
// operands rounded to bf16 into 128-byte-swizzled K-major shared-memory tiles
// (two stages of 128 x 64 A and 64 x 64 B), tcgen05.mma M=128 N=64 K=16 issued
// by one thread with the FP32 accumulator in tensor memory (64 columns), each
// stage released by a tcgen05.commit on its mbarrier, the accumulator read back
// with tcgen05.ld (thread = row) for the fused epilogue. Split-K over gridDim.z
// (EPI_STORE only, atomic accumulation into C).
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

constexpr int UM = 128, UN = 64, UK = 64;
constexpr int UTILE_A = UM * UK * 2, UTILE_B = UN * UK * 2;  // bytes of one stage's tiles
constexpr size_t UMMA_SMEM = 2 * (UTILE_A + UTILE_B) + 1024;  // two stages + alignment slack
constexpr uint32_t UIDESC = umma_idesc_bf16_f32(UM, UN);

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}
// 8 consecutive elements of a row (contiguous in memory) as bf16; vec when the
// 8 are inside the chunk and 16-byte loads are aligned, else guarded scalars.
template <class T>
__device__ __forceinline__ uint4 load8(const T* p, int valid, bool vec);
template <>
__device__ __forceinline__ uint4 load8<float>(const float* p, int valid, bool vec) {
  float v[8];
  if (vec && valid >= 8) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p)), b = __ldg(reinterpret_cast<const float4*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = i < valid ? p[i] : 0.f;
  }
  return make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
}
template <>
__device__ __forceinline__ uint4 load8<__nv_bfloat16>(const __nv_bfloat16* p, int valid, bool vec) {
  if (vec && valid >= 8) return __ldg(reinterpret_cast<const uint4*>(p));
  uint16_t h[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) h[i] = i < valid ? *reinterpret_cast<const uint16_t*>(p + i) : (uint16_t)0;
  return make_uint4(h[0] | ((uint32_t)h[1] << 16), h[2] | ((uint32_t)h[3] << 16), h[4] | ((uint32_t)h[5] << 16),
                    h[6] | ((uint32_t)h[7] << 16));
}

// One operand tile of R rows x UK columns of K into swizzled shared memory:
// element (row, k) = src(r0 + row, k0 + k); KCONTIG: src(r, k) = src[r*ld + k]
// (16-byte chunks along K), else src[k*ld + r] (8 rows per thread, scattered
// 2-byte stores). Rows >= rows and k >= kend are zero. All of a thread's loads
// are issued before its shared-memory stores (fetch, then place), so they
// overlap instead of waiting on stores the compiler cannot disambiguate.
template <int R>
struct TileRegs {
  static constexpr int N = R * UK / 8 / 128;
  uint4 v[N];
};
template <int R, bool KCONTIG, class T>
__device__ __forceinline__ void fetch_tile(TileRegs<R>& t, const T* src, int ld, int r0, int rows, int k0, int kend,
                                           bool vec) {
#pragma unroll
  for (int j = 0; j < TileRegs<R>::N; ++j) {
    const int q = threadIdx.x + 128 * j;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (KCONTIG) {
      const int gr = r0 + (q >> 3), gk = k0 + (q & 7) * 8;
      if (gr < rows && gk < kend) v = load8<T>(src + (size_t)gr * ld + gk, kend - gk, vec);
    } else {
      const int gr = r0 + (q % (R / 8)) * 8, gk = k0 + q / (R / 8);
      if (gk < kend && gr < rows) v = load8<T>(src + (size_t)gk * ld + gr, rows - gr, vec);
    }
    t.v[j] = v;
  }
}
template <int R, bool KCONTIG>
__device__ __forceinline__ void place_tile(uint8_t* tile, const TileRegs<R>& t) {
#pragma unroll
  for (int j = 0; j < TileRegs<R>::N; ++j) {
    const int q = threadIdx.x + 128 * j;
    if (KCONTIG) {
      *reinterpret_cast<uint4*>(tile + umma_sw128_offset(q >> 3, (q & 7) * 8)) = t.v[j];
    } else {
      const int rq = (q % (R / 8)) * 8, k = q / (R / 8);
      const uint16_t* h = reinterpret_cast<const uint16_t*>(&t.v[j]);
#pragma unroll
      for (int i = 0; i < 8; ++i) *reinterpret_cast<uint16_t*>(tile + umma_sw128_offset(rq + i, k)) = h[i];
    }
  }
}

template <class TA, class TB, bool TRA, bool TRB, int EPI>
__global__ void __launch_bounds__(128, 1) k_gemm(int M, int N, int K, const TA* __restrict__ A, int lda,
                                                 const TB* __restrict__ B, int ldb, float* __restrict__ Cm, int ldc,
                                                 Epi ep, int kchunk, int vec_a, int vec_b, int vec2, int* err) {
  extern __shared__ uint8_t gemm_smem[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  uint8_t* base = reinterpret_cast<uint8_t*>(((uintptr_t)gemm_smem + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * UM, n0 = blockIdx.y * UN;
  const int kb = blockIdx.z * kchunk;
  const int ke = min(K, kb + kchunk);
  const int nchunks = ke > kb ? (ke - kb + UK - 1) / UK : 0;
  const uint32_t bar0 = umma_smem_addr(&mbar[0]), bar1 = umma_smem_addr(&mbar[1]);
  if (warp == 0) {
    tmem_alloc(umma_smem_addr(&tmem_base), UN);
    tmem_relinquish();
  }
  if (tid == 0) {
    umma_mbar_init(bar0, 1);
    umma_mbar_init(bar1, 1);
    umma_mbar_init_fence();
  }
  tcgen05_before_sync();
  __syncthreads();
  tcgen05_after_sync();
  const uint32_t tmem = tmem_base;
  bool ok = true;
  int issued = 0;
  // chunk c + 1 is fetched into registers while chunk c is placed and issued
  TileRegs<UM> ta;
  TileRegs<UN> tb;
  if (nchunks > 0) {
    fetch_tile<UM, !TRA>(ta, A, lda, m0, M, kb, ke, vec_a != 0);
    fetch_tile<UN, TRB>(tb, B, ldb, n0, N, kb, ke, vec_b != 0);
  }
  for (int c = 0; c < nchunks; ++c) {
    const int s = c & 1;
    if (c >= 2) ok = umma_wait(s ? bar1 : bar0, ((c - 2) >> 1) & 1, err);
    if (!__syncthreads_and(ok)) break;  // stage s is free again (or the wait gave up everywhere)
    uint8_t* sa = base + s * UTILE_A;
    uint8_t* sb = base + 2 * UTILE_A + s * UTILE_B;
    place_tile<UM, !TRA>(sa, ta);
    place_tile<UN, TRB>(sb, tb);
    if (c + 1 < nchunks) {
      const int k1 = kb + (c + 1) * UK;
      fetch_tile<UM, !TRA>(ta, A, lda, m0, M, k1, ke, vec_a != 0);
      fetch_tile<UN, TRB>(tb, B, ldb, n0, N, k1, ke, vec_b != 0);
    }
    umma_fence_smem();
    __syncthreads();
    if (tid == 0) {
      tcgen05_after_sync();
      const uint32_t a0 = umma_smem_addr(sa), b0 = umma_smem_addr(sb);
#pragma unroll
      for (int kk = 0; kk < UK / 16; ++kk)
        umma_bf16(tmem, umma_desc_sw128(a0 + 32 * kk), umma_desc_sw128(b0 + 32 * kk), UIDESC, (c | kk) != 0);
      umma_commit(s ? bar1 : bar0);
    }
    issued = c + 1;
  }
  // every issued MMA has completed once the last commits of both stages arrived
  bool done = true;
  if (issued >= 1) done = umma_wait(((issued - 1) & 1) ? bar1 : bar0, ((issued - 1) >> 1) & 1, err) && done;
  if (issued >= 2) done = umma_wait(((issued - 2) & 1) ? bar1 : bar0, ((issued - 2) >> 1) & 1, err) && done;
  done = __syncthreads_and(done && issued == nchunks);
  tcgen05_after_sync();
  // accumulator rows (thread = row) into shared memory over the finished
  // operand tiles, 65-float row pitch (conflict-free both ways)
  float* stage = reinterpret_cast<float*>(base);
  if (done && nchunks > 0) {
    uint32_t r[32];
    const uint32_t row_addr = tmem + ((uint32_t)(warp * 32) << 16);
    float* srow = stage + (warp * 32 + lane) * 65;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      tmem_ld32(row_addr + 32 * h, r);
      tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 32; ++j) srow[32 * h + j] = __uint_as_float(r[j]);
    }
  } else {
    float* srow = stage + (warp * 32 + lane) * 65;
#pragma unroll
    for (int j = 0; j < 64; ++j) srow[j] = 0.f;
  }
  tcgen05_before_sync();
  __syncthreads();
  if (warp == 0) {
    tcgen05_after_sync();
    tmem_dealloc(tmem, UN);
  }
  if (!done) return;  // the error flag is set; nothing is written
  // epilogue, warp per row: lane owns columns 2 lane, 2 lane + 1 (float2
  // accesses when every stride and base allows them)
  const bool split = gridDim.z > 1;
  const int nloc = min(UN, N - n0);
  for (int rr = warp; rr < UM; rr += 4) {
    const int m = m0 + rr;
    if (m >= M) break;
    const float* srow = stage + rr * 65;
    const int j = 2 * lane;
    const int n = n0 + j;
    if (j >= nloc) continue;
    const bool pair = vec2 && j + 1 < nloc;
    float v0 = srow[j], v1 = pair ? srow[j + 1] : 0.f;
    auto ld2 = [&](const float* p, float& a, float& b) {
      if (pair) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        a = t.x;
        b = t.y;
      } else {
        a = *p;
      }
    };
    auto st2 = [&](float* p, float a, float b) {
      if (pair) *reinterpret_cast<float2*>(p) = make_float2(a, b);
      else *p = a;
    };
    if (EPI == EPI_STORE) {
      float* c = Cm + (size_t)m * ldc + n;
      if (split) {
        if (pair) atomicAdd(reinterpret_cast<float2*>(c), make_float2(v0, v1));
        else atomicAdd(c, v0);
      } else {
        if (ep.accumulate) {
          float a0 = 0.f, a1 = 0.f;
          ld2(c, a0, a1);
          v0 += a0;
          v1 += a1;
        }
        st2(c, v0, v1);
      }
    } else if (EPI == EPI_BIAS_RELU) {
      const float z0 = v0 + __ldg(ep.bias + n), z1 = pair ? v1 + __ldg(ep.bias + n + 1) : 0.f;
      float r0 = 0.f, r1 = 0.f;
      if (ep.r) ld2(ep.r + (size_t)m * ep.ldr + n, r0, r1);
      st2(ep.z + (size_t)m * ep.ldz + n, z0, z1);
      st2(ep.h + (size_t)m * ep.ldh + n, r0 + fmaxf(z0, 0.f), r1 + fmaxf(z1, 0.f));
    } else if (EPI == EPI_BIAS) {
      st2(Cm + (size_t)m * ldc + n, v0 + __ldg(ep.bias + n), pair ? v1 + __ldg(ep.bias + n + 1) : 0.f);
    } else if (EPI == EPI_SPLIT) {
      // split_at is even, so a pair never straddles it
      if (n < ep.split_at) {
        float r0 = 0.f, r1 = 0.f;
        ld2(ep.r + (size_t)m * ep.ldr + n, r0, r1);
        st2(Cm + (size_t)m * ldc + n, v0 + r0, v1 + r1);
      } else {
        st2(ep.h + (size_t)m * ep.ldh + (n - ep.split_at), v0, v1);
      }
    } else if (EPI == EPI_STORE_MASK) {
      float q0 = 0.f, q1 = 0.f;
      ld2(ep.zmask + (size_t)m * ep.ldzm + n, q0, q1);
      st2(Cm + (size_t)m * ldc + n, v0, v1);
      st2(ep.d2 + (size_t)m * ep.ldd2 + n, q0 > 0.f ? v0 : 0.f, q1 > 0.f ? v1 : 0.f);
    }
    if (!pair && j + 1 < nloc) {  // the second column alone
      const int n1 = n + 1;
      const float w = srow[j + 1];
      if (EPI == EPI_STORE) {
        float* c = Cm + (size_t)m * ldc + n1;
        if (split) atomicAdd(c, w);
        else *c = ep.accumulate ? *c + w : w;
      } else if (EPI == EPI_BIAS_RELU) {
        const float z = w + __ldg(ep.bias + n1);
        const float res = ep.r ? ep.r[(size_t)m * ep.ldr + n1] : 0.f;
        ep.z[(size_t)m * ep.ldz + n1] = z;
        ep.h[(size_t)m * ep.ldh + n1] = res + fmaxf(z, 0.f);
      } else if (EPI == EPI_BIAS) {
        Cm[(size_t)m * ldc + n1] = w + __ldg(ep.bias + n1);
      } else if (EPI == EPI_SPLIT) {
        if (n1 < ep.split_at) Cm[(size_t)m * ldc + n1] = w + ep.r[(size_t)m * ep.ldr + n1];
        else ep.h[(size_t)m * ep.ldh + (n1 - ep.split_at)] = w;
      } else if (EPI == EPI_STORE_MASK) {
        Cm[(size_t)m * ldc + n1] = w;
        ep.d2[(size_t)m * ep.ldd2 + n1] = ep.zmask[(size_t)m * ep.ldzm + n1] > 0.f ? w : 0.f;
      }
    }
  }
}

template <class T>
bool vec16(const T* p, int ld) {
  constexpr int per = 16 / (int)sizeof(T);
  return ((uintptr_t)p % 16) == 0 && ld % per == 0;
}

template <class TA, class TB, bool TRA, bool TRB, int EPI>
fg_status gemm(cudaStream_t st, int nsm, int M, int N, int K, const TA* A, int lda, const TB* B, int ldb, float* Cm,
               int ldc, const Epi& ep, bool allow_split, int* err) {
  if (M <= 0 || N <= 0) return FG_OK;
  const unsigned gx = (unsigned)((M + UM - 1) / UM), gy = (unsigned)((N + UN - 1) / UN);
  int splits = 1;
  if (allow_split && EPI == EPI_STORE && K > 2 * UK) {
    // up to four CTAs per SM (50 KB of shared memory each): the K chunks of a
    // CTA run one after another, so the memory parallelism is in the CTA count
    const int want = std::max(1, (4 * nsm) / (int)(gx * gy));
    splits = std::min(want, (K + UK - 1) / UK);
  }
  int kchunk = (K + splits - 1) / splits;
  kchunk = std::max(UK, (kchunk + UK - 1) / UK * UK);
  splits = std::max(1, (K + kchunk - 1) / kchunk);
  if (K <= 0) {  // empty reduction: the product is zero
    splits = 1;
    kchunk = UK;
  }
  if (EPI == EPI_STORE && splits > 1 && !ep.accumulate)
    FG_CUDA(cudaMemset2DAsync(Cm, (size_t)ldc * sizeof(float), 0, (size_t)N * sizeof(float), (size_t)M, st));
  auto kern = k_gemm<TA, TB, TRA, TRB, EPI>;
  FG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UMMA_SMEM));
  // 16-byte loads need aligned rows: along K for K-contiguous operands, along M / N otherwise
  const int va = vec16(A, lda) ? 1 : 0, vb = vec16(B, ldb) ? 1 : 0;
  // float2 epilogue accesses: every output / input row stride even and base 8-byte aligned
  auto ok2 = [](const float* p, int ld) { return !p || (((uintptr_t)p % 8) == 0 && ld % 2 == 0); };
  const int v2 = ok2(Cm, ldc) && ok2(ep.z, ep.ldz) && ok2(ep.h, ep.ldh) && ok2(ep.r, ep.ldr) &&
                         ok2(ep.zmask, ep.ldzm) && ok2(ep.d2, ep.ldd2) && ep.split_at % 2 == 0
                     ? 1
                     : 0;
  dim3 grid(gx, gy, (unsigned)splits);
  FG_LAUNCH(kern, grid, 128, UMMA_SMEM, st, M, N, K, A, lda, B, ldb, Cm, ldc, ep, kchunk, va, vb, v2, err);
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

// Pair weights are summed in 64-bit fixed point (2^-36 units), so the
// covisibility matrix does not depend on the order of the atomic additions.
// Each weight is a trace of a product of two PSD matrices whose eigenvalues
// are at most 1 in the whitened coordinates (E (C + lambda)^-1 E^T <= B), so
// a pair adds at most pw <= 4; weights are clamped to [0, 64] before the
// conversion, which keeps 2^27 pairs per camera pair away from overflow.
constexpr double PAIR_SCALE = 68719476736.0;  // 2^36
__device__ __forceinline__ unsigned long long pair_fixed(double w) {
  return (unsigned long long)__double2ll_rn(fmin(fmax(w, 0.0), 64.0) * PAIR_SCALE);
}

// Pair weights w_ij += <K_e, K_f> over the edge pairs of each point (warp per point).
__global__ void k_pairs(int64_t nP, int64_t nC, const int64_t* pt_edge_off, const int64_t* pt_edge,
                        const DEdgeMeta* edges, const float* Kin, int pw, unsigned long long* adj) {
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
      const unsigned long long q = pair_fixed((double)w);
      atomicAdd(adj + (int64_t)ci * nC + cj, q);
      atomicAdd(adj + (int64_t)cj * nC + ci, q);
    }
  }
}

// Row-normalized sqrt weights in bf16 (row stride lda, zero past column nC),
// plus features 45 (log1p degree / 4) and 46 (log1p coupling) of observed
// cameras; the fixed-point row is cleared for the next system. Block of 256
// per row, sums in a fixed order.
__global__ void k_normalize(int64_t nC, int64_t lda, unsigned long long* adj, const uint8_t* mask, float* X0,
                            __nv_bfloat16* Abf) {
  const int64_t i = blockIdx.x;
  unsigned long long* row = adj + i * nC;
  double s = 0;
  int cnt = 0;
  for (int64_t j = threadIdx.x; j < nC; j += blockDim.x) {
    const unsigned long long v = row[j];
    if (v) {
      s += sqrt((double)v / PAIR_SCALE);
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
  for (int64_t j = threadIdx.x; j < lda; j += blockDim.x) {
    float a = 0.f;
    if (j < nC) {
      const unsigned long long v = row[j];
      if (v) a = (float)(sqrt((double)v / PAIR_SCALE) * inv);
      row[j] = 0;
    }
    Abf[i * lda + j] = __float2bfloat16_rn(a);
  }
  if (threadIdx.x == 0 && mask[i]) {
    X0[i * NF + 45] = (float)(log1p((double)sc[0]) / 4.0);
    X0[i * NF + 46] = (float)log1p(tot);
  }
}

// ---- the 9/3 (BAL) feature pass, the same quantities in two kernels that
// read every edge once (after the positions). V_e = E_e L_p^-T (so V_e V_e^T = E_e C_p^-1 E_e^T) and
// G_e = L_c^-1 V_e (so K_e = G_e^T G_e); unobserved variables use
// L = sqrt(lambda) I as above.

// The point-sorted position of every edge: pos[pt_edge[k]] = k (for a view
// without the backend's camera-major (position, point) array).
__global__ void k_gnn_pos(int64_t nedges, const int64_t* pt_edge, int32_t* pos) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < nedges) pos[pt_edge[k]] = (int32_t)k;
}

// Block of 128 per camera (L_c in shared memory), the camera's edges in
// chunks of 128: each thread first reads its edge's position, point index and
// point factor entries, then the block copies the chunk's records (E_e from
// the fast path's point-sorted records, 28 storage words each, as 16-byte
// vectors spread over all threads; the reference-layout cross array, 27 words
// per edge, thread per edge) into shared memory. Then, thread per edge:
// U = sum_e V_e V_e^T in FP64 and K_e = G_e^T G_e with G_e = L_c^-1 V_e,
// written at the edge's point-sorted position (K lower, 6 floats, camera
// index in slot 6); then P = L_c^-1 U L_c^-T and the node-feature row as
// k_node_features writes it.
constexpr int CAMS93_NT = 128;
template <class TS>
__global__ void __launch_bounds__(CAMS93_NT, sizeof(TS) == 4 ? 4 : 2)
    k_gnn_cams93(Layout L, const int64_t* cam_edge_off, const int64_t* cam_edge, const int2* meta, const int32_t* pos,
                 const TS* src, int by_edge, const DEdgeMeta* edges, const uint8_t* observed, const TS* factors,
                 double lambda, float* X0, uint8_t* mask, float* Kout) {
  using T = TS;
  constexpr int VPR = 28 * (int)sizeof(TS) / 16;  // 16-byte vectors per record
  const int64_t cam = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float* row = X0 + cam * NF;
  const int64_t e0 = cam_edge_off[cam], e1 = cam_edge_off[cam + 1];
  if (!observed[cam]) {
    if (tid == 0) mask[cam] = 0;
    if (tid < NF) row[tid] = tid == 49 ? 1.f : 0.f;
    for (int64_t k = e0 + tid; k < e1; k += CAMS93_NT) {
      float4* ko = reinterpret_cast<float4*>(Kout + (int64_t)(meta ? meta[k].x : pos[cam_edge[k]]) * 8);
      ko[0] = make_float4(0.f, 0.f, 0.f, 0.f);
      ko[1] = make_float4(0.f, 0.f, __int_as_float((int)cam), 0.f);
    }
    return;
  }
  __shared__ __align__(16) T srec[CAMS93_NT * 28];
  __shared__ int32_t spos[CAMS93_NT];
  __shared__ T sl[81], srd[9];
  __shared__ double red[4][45];
  __shared__ double U[81], W[81];
  const TS* lc = factors + L.gram_offset(cam);
  if (tid < 81) sl[tid] = lc[tid];
  if (tid < 9) srd[tid] = (T)1 / lc[tid * 9 + tid];
  // per-thread partial sums in the storage precision (a thread sees about
  // 1/128 of the camera's edges), combined in FP64 below
  T acc[45];
#pragma unroll
  for (int i = 0; i < 45; ++i) acc[i] = 0;
  const T isl = (T)(1.0 / sqrt(lambda));
  // an edge's source index (cross array only), point-sorted position and
  // point: one coalesced int2 from the camera-major array, else gathered
  auto fetch = [&](int64_t k, int64_t& e, int32_t& pc, int32_t& py) {
    if (meta) {
      const int2 m = meta[k];
      pc = m.x;
      py = m.y;
      e = by_edge ? cam_edge[k] : 0;
    } else {
      e = cam_edge[k];
      pc = pos[e];
      py = edges[e].pt;
    }
  };
  // the first chunk's edge metadata; a later chunk's is fetched while the
  // chunk before it is computed
  int64_t ne = 0;
  int32_t npc = 0, npy = 0;
  if (e0 + tid < e1) fetch(e0 + tid, ne, npc, npy);
  for (int64_t base = e0; base < e1; base += CAMS93_NT) {
    const int nv = (int)(e1 - base < CAMS93_NT ? e1 - base : CAMS93_NT);
    const bool have = base + tid < e1;
    const int64_t e = ne, pc = npc;
    const int py = npy;
    T r0 = isl, r1 = isl, r2 = isl, p10 = 0, p20 = 0, p21 = 0;
    if (have) {
      spos[tid] = (int32_t)pc;
      // the factor entries are read whether or not the point is observed
      // (every variable has its block), so the two loads go out together
      const TS* lp = factors + L.gram_offset(L.nC + py);
      const T f0 = lp[0], f1 = lp[1], f2 = lp[2], f4 = lp[4], f5 = lp[5], f8 = lp[8];
      if (observed[L.nC + py]) {
        r0 = (T)1 / f0; r1 = (T)1 / f4; r2 = (T)1 / f8;
        p10 = f1; p20 = f2; p21 = f5;
      }
      if (by_edge) {
        const TS* E = src + e * 27;
#pragma unroll
        for (int i = 0; i < 27; ++i) srec[tid * 28 + i] = E[i];
      }
    }
    __syncthreads();
    if (!by_edge) {
      // all of a thread's vector loads are issued before its shared stores
      const uint4* s4 = reinterpret_cast<const uint4*>(src);
      uint4* d4 = reinterpret_cast<uint4*>(srec);
      uint4 t[VPR];
#pragma unroll
      for (int j = 0; j < VPR; ++j) {
        const int i = tid + j * CAMS93_NT;
        if (i < nv * VPR) {
          const int r = i / VPR;
          t[j] = s4[(int64_t)spos[r] * VPR + (i - r * VPR)];
        }
      }
#pragma unroll
      for (int j = 0; j < VPR; ++j) {
        const int i = tid + j * CAMS93_NT;
        if (i < nv * VPR) d4[i] = t[j];
      }
    }
    if (base + CAMS93_NT + tid < e1) fetch(base + CAMS93_NT + tid, ne, npc, npy);
    if (!by_edge) __syncthreads();
    if (have) {
      // V = E L_p^-T: row c solves L_p y = E(c, :)^T
      T v[27];
      {
        T E[28];
        if constexpr (sizeof(TS) == 4) {
          const float4* r4 = reinterpret_cast<const float4*>(srec + tid * 28);
#pragma unroll
          for (int q = 0; q < 7; ++q) {
            const float4 t = r4[q];
            E[4 * q] = t.x; E[4 * q + 1] = t.y; E[4 * q + 2] = t.z; E[4 * q + 3] = t.w;
          }
        } else {
          const double2* r2v = reinterpret_cast<const double2*>(srec + tid * 28);
#pragma unroll
          for (int q = 0; q < 14; ++q) {
            const double2 t = r2v[q];
            E[2 * q] = t.x; E[2 * q + 1] = t.y;
          }
        }
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          const T y0 = E[c] * r0;
          const T y1 = (E[9 + c] - p10 * y0) * r1;
          const T y2 = (E[18 + c] - p20 * y0 - p21 * y1) * r2;
          v[c] = y0; v[9 + c] = y1; v[18 + c] = y2;
        }
      }
      int idx = 0;
#pragma unroll
      for (int c = 0; c < 9; ++c)
#pragma unroll
        for (int r = c; r < 9; ++r) acc[idx++] += v[r] * v[c] + v[9 + r] * v[9 + c] + v[18 + r] * v[18 + c];
#pragma unroll
      for (int i = 0; i < 9; ++i) {  // G = L_c^-1 V, the three columns together
        T s0 = v[i], s1 = v[9 + i], s2 = v[18 + i];
#pragma unroll
        for (int j = 0; j < i; ++j) {
          const T l = sl[j * 9 + i];
          s0 -= l * v[j];
          s1 -= l * v[9 + j];
          s2 -= l * v[18 + j];
        }
        v[i] = s0 * srd[i];
        v[9 + i] = s1 * srd[i];
        v[18 + i] = s2 * srd[i];
      }
      T K[6];  // K00, K10, K20, K11, K21, K22
      int kx = 0;
#pragma unroll
      for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int r = q; r < 3; ++r) {
          T sk = 0;
#pragma unroll
          for (int c = 0; c < 9; ++c) sk += v[9 * r + c] * v[9 * q + c];
          K[kx++] = sk;
        }
      float4* ko = reinterpret_cast<float4*>(Kout + pc * 8);
      ko[0] = make_float4((float)K[0], (float)K[1], (float)K[2], (float)K[3]);
      ko[1] = make_float4((float)K[4], (float)K[5], __int_as_float((int)cam), 0.f);
    }
    __syncthreads();  // the next chunk overwrites srec and spos
  }
#pragma unroll
  for (int i = 0; i < 45; ++i) {
    const double sum = lane_allsum((double)acc[i]);
    if (lane == 0) red[warp][i] = sum;
  }
  __syncthreads();
  if (tid < 45) {
    const double sum = (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]);
    int c = 0, r = tid;  // lower entry tid (column-major) -> (r, c)
    while (r >= 9 - c) {
      r -= 9 - c;
      ++c;
    }
    r += c;
    U[c * 9 + r] = sum;
    U[r * 9 + c] = sum;
  }
  __syncthreads();
  if (tid < 9) {  // W = L^-1 U, column tid
    double x[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) x[i] = U[tid * 9 + i];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      double t = x[i];
#pragma unroll
      for (int j = 0; j < i; ++j) t -= (double)lc[j * 9 + i] * x[j];
      x[i] = t / (double)lc[i * 9 + i];
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) W[tid * 9 + i] = x[i];
  }
  __syncthreads();
  if (tid < 9) {  // P = L^-1 W^T, column tid (row tid of W)
    double x[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) x[i] = W[i * 9 + tid];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      double t = x[i];
#pragma unroll
      for (int j = 0; j < i; ++j) t -= (double)lc[j * 9 + i] * x[j];
      x[i] = t / (double)lc[i * 9 + i];
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) U[tid * 9 + i] = x[i];  // U now holds P (column-major)
  }
  __syncthreads();
  if (tid < NF) {
    float f = 0.f;
    if (tid < 45) {
      int c = 0, r = tid;
      while (r >= 9 - c) {
        r -= 9 - c;
        ++c;
      }
      r += c;
      f = (float)(0.5 * (U[c * 9 + r] + U[r * 9 + c]));
    } else if (tid == 47) {
      f = (float)(log10(fmax(lambda, 1e-12)) / 12.0);
    } else if (tid == 48) {
      double tr = 0;
      for (int c = 0; c < 9; ++c) tr += U[c * 9 + c];
      f = (float)(tr / 9);
    } else if (tid == 49) {
      f = 1.f;
    }
    if (tid != 45 && tid != 46) row[tid] = f;  // 45 and 46 are k_normalize's
  }
  if (tid == 0) mask[cam] = 1;
}

// Warp per point: the pairs (a, b) of its edges spread over the lanes;
// w = <K_a, K_b>_F into the fixed-point covisibility of both orders.
__global__ void __launch_bounds__(128) k_gnn_pairs93(int64_t nP, int64_t nC, const int64_t* pt_edge_off,
                                                     const float* Kin, unsigned long long* adj) {
  const int lane = threadIdx.x & 31;
  const int64_t pt = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (pt >= nP) return;
  const int64_t o = pt_edge_off[pt];
  const int64_t t = pt_edge_off[pt + 1] - o;
  const int64_t np = t * (t - 1) / 2;
  for (int64_t q = lane; q < np; q += 32) {
    int64_t a = 0, r = q;
    while (r >= t - 1 - a) {
      r -= t - 1 - a;
      ++a;
    }
    const int64_t b = a + 1 + r;
    const float4* ka = reinterpret_cast<const float4*>(Kin + (o + a) * 8);
    const float4* kb = reinterpret_cast<const float4*>(Kin + (o + b) * 8);
    const float4 a0 = ka[0], a1 = ka[1], b0 = kb[0], b1 = kb[1];
    const int ci = __float_as_int(a1.z), cj = __float_as_int(b1.z);
    if (ci == cj) continue;
    const double w = (double)a0.x * b0.x + (double)a0.w * b0.w + (double)a1.y * b1.y +
                     2.0 * ((double)a0.y * b0.y + (double)a0.z * b0.z + (double)a1.x * b1.x);
    const unsigned long long fx = pair_fixed(w);
    if (fx) {
      atomicAdd(adj + (int64_t)ci * nC + cj, fx);
      atomicAdd(adj + (int64_t)cj * nC + ci, fx);
    }
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

// The 9-wide head as k_head_minv below, warp per camera with the 9 x 9
// products spread over the lanes (shared memory per warp).
template <class TS>
__global__ void __launch_bounds__(128) k_head_minv93(Layout L, const float* O, const uint8_t* mask,
                                                     const TS* factors, TS* minv, unsigned* nonfinite) {
  __shared__ double sh[4][4][81];  // per warp: A (row-major), Li (row-major), Mh, T
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t cam = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (cam >= L.nC || !mask[cam]) return;  // uniform across the warp
  double* A = sh[warp][0];
  double* Li = sh[warp][1];
  double* Mh = sh[warp][2];
  double* T = sh[warp][3];
  const float* o = O + cam * NH;
  for (int k = lane; k < 81; k += 32) A[k] = 0;
  __syncwarp();
  if (lane < 45) {
    int c = 0, r = lane;
    while (r >= 9 - c) {
      r -= 9 - c;
      ++c;
    }
    r += c;
    A[r * 9 + c] = (double)OUT_SCALE * (double)o[lane];
  }
  __syncwarp();
  if (lane < 9) A[lane * 9 + lane] += 1.0;
  const TS* l = factors + L.gram_offset(cam);
  if (lane < 9) {  // column lane of L^-1
    double x[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      double s = i == lane ? 1.0 : 0.0;
#pragma unroll
      for (int j = 0; j < i; ++j) s -= (double)l[j * 9 + i] * x[j];
      x[i] = s / (double)l[i * 9 + i];
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) Li[i * 9 + lane] = x[i];
  }
  __syncwarp();
  for (int e = lane; e < 81; e += 32) {  // Mh = A A^T + eps I
    const int i = e / 9, j = e % 9;
    double s = 0;
#pragma unroll
    for (int k = 0; k < 9; ++k) s += A[i * 9 + k] * A[j * 9 + k];
    Mh[e] = s + (i == j ? (double)EPSILON : 0.0);
  }
  __syncwarp();
  for (int e = lane; e < 81; e += 32) {  // T = Mh L^-1
    const int a = e / 9, j = e % 9;
    double t = 0;
#pragma unroll
    for (int b = 0; b < 9; ++b) t += Mh[a * 9 + b] * Li[b * 9 + j];
    T[e] = t;
  }
  __syncwarp();
  double out[2];
  int pi[2], pj[2];
  bool ok = true;
#pragma unroll
  for (int u = 0; u < 2; ++u) {  // upper pairs (i <= j) lane and lane + 32
    const int p = lane + 32 * u;
    pi[u] = -1;
    if (p >= 45) continue;
    int i = 0, r = p;
    while (r >= 9 - i) {
      r -= 9 - i;
      ++i;
    }
    const int j = i + r;
    double s = 0;
#pragma unroll
    for (int a = 0; a < 9; ++a) s += Li[a * 9 + i] * T[a * 9 + j];
    ok = ok && isfinite(s);
    out[u] = s;
    pi[u] = i;
    pj[u] = j;
  }
  if (__any_sync(0xffffffffu, !ok)) {
    if (lane == 0) atomicAdd(nonfinite, 1u);
    return;
  }
  TS* dst = minv + cam * 81;
#pragma unroll
  for (int u = 0; u < 2; ++u)
    if (pi[u] >= 0) {
      dst[pi[u] * 9 + pj[u]] = (TS)out[u];
      dst[pj[u] * 9 + pi[u]] = (TS)out[u];
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
  int64_t ldA = 0;  // row stride of A: C rounded up to 64, zero padded
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
  DBuf<float> Z[NLAYER + 1], HA[NLAYER], H3, O, dO, dHa, dHb, dA, dZ, edgeK;
  DBuf<unsigned long long> adj;  // fixed-point covisibility, C x C, left cleared by k_normalize
  int64_t adj_cap = -1;          // entries of adj known to be zero
  DBuf<int32_t> edgePos;         // point-sorted position of every edge (views without cam_meta)
  DBuf<double> dloss;
  DBuf<unsigned> dcount;
  DBuf<int> gemm_err;  // set by a GEMM whose tensor-core wait ran out
  HBuf<double> hloss;
  HBuf<unsigned> hcount;
  HBuf<int> herr;
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
    FG_TRY(gemm_err.resize(1));
    FG_CUDA(cudaMemsetAsync(gemm_err.get(), 0, sizeof(int), st));
    FG_TRY(herr.resize(1));
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

  // The previous precondition call's read-back, when it has landed: the
  // nonfinite count goes to *nonfinite, a set GEMM flag becomes
  // FG_DEVICE_TIMEOUT (and is cleared).
  cudaEvent_t status_ev = nullptr;
  bool status_pending = false;
  fg_status take_async_status(unsigned* nonfinite) {
    if (!status_ev) FG_CUDA(cudaEventCreateWithFlags(&status_ev, cudaEventDisableTiming));
    if (!status_pending || cudaEventQuery(status_ev) != cudaSuccess) return FG_OK;
    status_pending = false;
    *nonfinite = hcount.get()[0];
    if (herr.get()[0]) {
      herr.get()[0] = 0;
      FG_CUDA(cudaMemsetAsync(gemm_err.get(), 0, sizeof(int), st));
      set_error("a tensor-core GEMM of the learned preconditioner timed out");
      return FG_DEVICE_TIMEOUT;
    }
    return FG_OK;
  }
  ~Gnn() {
    if (status_ev) cudaEventDestroy(status_ev);
  }

  // FG_DEVICE_TIMEOUT (and the flag cleared) when a GEMM gave up waiting on
  // its tensor-core commits since the last check; call after a stream sync.
  fg_status check_gemm() {
    if (status_pending) {  // this sync lands the pending read-back too
      FG_CUDA(cudaStreamSynchronize(st));
      unsigned ignored = 0;
      FG_TRY(take_async_status(&ignored));
    }
    FG_CUDA(cudaMemcpyAsync(herr.get(), gemm_err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    if (herr.get()[0]) {
      FG_CUDA(cudaMemsetAsync(gemm_err.get(), 0, sizeof(int), st));
      set_error("a tensor-core GEMM of the learned preconditioner timed out");
      return FG_DEVICE_TIMEOUT;
    }
    return FG_OK;
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
    s.ldA = std::max<int64_t>((C + 63) / 64 * 64, 64);
    FG_TRY(s.X0.resize(C * NF));
    FG_TRY(s.A.resize(std::max<int64_t>(C * s.ldA, 1)));
    FG_TRY(s.mask.resize(std::max<int64_t>(C, 1)));
    if (adj_cap < C * C) {
      FG_TRY(adj.resize(std::max<int64_t>(C * C, 1)));
      FG_CUDA(cudaMemsetAsync(adj.get(), 0, (size_t)std::max<int64_t>(C * C, 1) * sizeof(unsigned long long), st));
    }
    adj_cap = -1;  // dirty until k_normalize has cleared the rows again
    const TS* fac = (const TS*)v.factors;
    if (L.cw == 9 && L.pw == 3) {
      FG_TRY(edgeK.resize(std::max<int64_t>(v.nedges * 8, 1)));
      const TS* src = v.rec ? (const TS*)v.rec : (const TS*)v.cross;
      if (!v.cam_meta) {  // positions gathered through pos
        FG_TRY(edgePos.resize(std::max<int64_t>(v.nedges, 1)));
        if (v.nedges)
          FG_LAUNCH(k_gnn_pos, grid_for(v.nedges, 256), 256, 0, st, v.nedges, v.pt_edge, edgePos.get());
      }
      FG_LAUNCH(k_gnn_cams93<TS>, (unsigned)C, CAMS93_NT, 0, st, L, v.cam_edge_off, v.cam_edge, v.cam_meta,
                v.cam_meta ? (const int32_t*)nullptr : (const int32_t*)edgePos.get(), src, v.rec ? 0 : 1, v.edges,
                v.observed, fac, v.lambda, s.X0.get(), s.mask.get(), edgeK.get());
      if (v.nedges && L.nP)
        FG_LAUNCH(k_gnn_pairs93, grid_for((size_t)L.nP * 32, 128), 128, 0, st, (int64_t)L.nP, C, v.pt_edge_off,
                  edgeK.get(), adj.get());
    } else {
      FG_TRY(edgeK.resize(std::max<int64_t>(v.nedges * 16, 1)));
      const TS* cr = (const TS*)v.cross;
      FG_LAUNCH(k_node_features<TS>, grid_for((size_t)C * 32, 128), 128, 0, st, L, v.cam_edge_off, v.cam_edge,
                v.edges, cr, v.observed, fac, v.lambda, s.X0.get(), s.mask.get());
      if (v.nedges) {
        FG_LAUNCH(k_edge_k<TS>, grid_for(v.nedges, 128), 128, 0, st, L, v.nedges, v.edges, cr, v.observed, fac,
                  v.lambda, edgeK.get());
        if (L.nP)
          FG_LAUNCH(k_pairs, grid_for((size_t)L.nP * 32, 128), 128, 0, st, (int64_t)L.nP, C, v.pt_edge_off,
                    v.pt_edge, v.edges, edgeK.get(), L.pw, adj.get());
      }
    }
    FG_LAUNCH(k_normalize, (unsigned)C, 256, 0, st, C, s.ldA, adj.get(), s.mask.get(), s.X0.get(), s.A.get());
    adj_cap = C * C;
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
                                                                     nullptr, 0, e0, false, gemm_err.get())));
    for (int l = 0; l < NLAYER; ++l) {
      Epi ea;
      FG_TRY((gemm<__nv_bfloat16, float, false, false, EPI_STORE>(st, nsm, C, NH, C, s.A.get(), (int)s.ldA, HA[l].get(), 2 * NH,
                                                                   HA[l].get() + NH, 2 * NH, ea, true, gemm_err.get())));
      Epi ez;
      ez.bias = w.get() + P.b[l];
      ez.z = Z[l + 1].get();
      ez.ldz = NH;
      ez.h = l + 1 < NLAYER ? HA[l + 1].get() : H3.get();
      ez.ldh = l + 1 < NLAYER ? 2 * NH : NH;
      ez.r = HA[l].get();
      ez.ldr = 2 * NH;
      FG_TRY((gemm<float, __nv_bfloat16, false, false, EPI_BIAS_RELU>(st, nsm, C, NH, 2 * NH, HA[l].get(), 2 * NH,
                                                                       W + P.w[l], NH, nullptr, 0, ez, false, gemm_err.get())));
    }
    Epi eo;
    eo.bias = w.get() + P.b_out;
    FG_TRY((gemm<float, __nv_bfloat16, false, false, EPI_BIAS>(st, nsm, C, NH, NH, H3.get(), NH, W + P.w_out, NH,
                                                                O.get(), NH, eo, false, gemm_err.get())));
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
                                                        NH, none, true, gemm_err.get())));
    FG_LAUNCH(k_colsum, 1, 256, 0, st, C, dO.get(), NH, G + P.b_out);
    Epi em;
    em.zmask = Z[NLAYER].get();
    em.ldzm = NH;
    em.d2 = dZ.get();
    em.ldd2 = NH;
    FG_TRY((gemm<float, __nv_bfloat16, false, true, EPI_STORE_MASK>(st, nsm, C, NH, NH, dO.get(), NH, W + P.w_out, NH,
                                                                     dHa.get(), NH, em, false, gemm_err.get())));
    float* dh = dHa.get();
    float* dh2 = dHb.get();
    for (int l = NLAYER - 1; l >= 0; --l) {
      FG_TRY((gemm<float, float, true, false, EPI_STORE>(st, nsm, 2 * NH, NH, C, HA[l].get(), 2 * NH, dZ.get(), NH,
                                                          G + P.w[l], NH, none, true, gemm_err.get())));
      FG_LAUNCH(k_colsum, 1, 256, 0, st, C, dZ.get(), NH, G + P.b[l]);
      Epi es;
      es.split_at = NH;
      es.r = dh;
      es.ldr = NH;
      es.h = dA.get();
      es.ldh = NH;
      FG_TRY((gemm<float, __nv_bfloat16, false, true, EPI_SPLIT>(st, nsm, C, 2 * NH, NH, dZ.get(), NH, W + P.w[l], NH,
                                                                  dh2, NH, es, false, gemm_err.get())));
      Epi acc;
      acc.accumulate = 1;
      FG_TRY((gemm<__nv_bfloat16, float, true, false, EPI_STORE>(st, nsm, C, NH, C, s.A.get(), (int)s.ldA, dA.get(), NH, dh2,
                                                                  NH, acc, true, gemm_err.get())));
      FG_LAUNCH(k_relu_mask, grid_for((size_t)C * NH, 256), 256, 0, st, (int64_t)C * NH, dh2, Z[l].get(), dZ.get());
      std::swap(dh, dh2);
    }
    FG_TRY((gemm<float, float, true, false, EPI_STORE>(st, nsm, NF, NH, C, s.X0.get(), NF, dZ.get(), NH, G + P.w_in,
                                                        NH, none, true, gemm_err.get())));
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
    if (v.L.cw == 9)
      FG_LAUNCH(k_head_minv93<TS>, grid_for((size_t)live.C * 32, 128), 128, 0, st, v.L, O.get(), live.mask.get(),
                (const TS*)v.factors, (TS*)minv, dcount.get());
    else
      FG_LAUNCH(k_head_minv<TS>, grid_for(live.C, 64), 64, 0, st, v.L, O.get(), live.mask.get(), (const TS*)v.factors,
              (TS*)minv, dcount.get());
    // No host sync on the solve path: the count and the GEMM flag of this call
    // are read back asynchronously and reported by the next call once its copy
    // has landed (the PCG that follows polls the stream anyway).
    FG_TRY(take_async_status(nonfinite));
    FG_CUDA(cudaMemcpyAsync(hcount.get(), dcount.get(), sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaMemcpyAsync(herr.get(), gemm_err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaEventRecord(status_ev, st));
    status_pending = true;
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
    FG_TRY(check_gemm());
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
    FG_TRY(check_gemm());
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
    const size_t ld = (size_t)s.ldA;
    std::vector<__nv_bfloat16> tmp(C * ld);
    FG_CUDA(cudaMemcpyAsync(tmp.data(), s.A.get(), C * ld * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < C; ++i)
      for (size_t j = 0; j < C; ++j) adjacency[i * C + j] = __bfloat162float(tmp[i * ld + j]);
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
  s->ldA = std::max<int64_t>(((int64_t)C + 63) / 64 * 64, 64);
  const size_t ld = (size_t)s->ldA;
  FG_TRY(s->A.resize(std::max<size_t>(C * ld, 1)));
  FG_TRY(s->mask.resize(std::max<size_t>(C, 1)));
  FG_TRY(s->PX.resize(std::max<size_t>(n, 1)));
  FG_TRY(s->PY.resize(std::max<size_t>(n, 1)));
  std::vector<__nv_bfloat16> tmp(C * ld, __float2bfloat16_rn(0.f));
  for (size_t i = 0; i < C; ++i)
    for (size_t j = 0; j < C; ++j) tmp[i * ld + j] = __float2bfloat16_rn(adjacency[i * C + j]);
  if (C) {
    FG_CUDA(cudaMemcpyAsync(s->X0.get(), features, C * fg::NF * sizeof(float), cudaMemcpyHostToDevice, G.st));
    FG_CUDA(cudaMemcpyAsync(s->A.get(), tmp.data(), C * ld * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, G.st));
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
