// Single-pass reduced operator for BAL-shaped Schur systems (retained width 9,
// eliminated width 3): y = lambda x + B x - E C^-1 E^T x with every cross
// block read from HBM exactly once per application.
//
// Layout (rebuilt at prepare_damping): cross blocks in point-major order as
// 28-word edge records [E (27, row p*9+c) | camera index + warp-tile-local
// point index], point records of 8 words [C^-1 packed lower (6) | unused], and
// warp tiles = contiguous point ranges of at most 32 edges; a stage is WPS
// consecutive warp tiles.
//
// k_fast_apply: one CTA per SM; FAST_GROUPS groups of WPS warps each stream
// their stages through shared memory with cp.async.bulk (TMA, 1-D) into a
// two-stage mbarrier pipeline. Each warp owns one warp tile per stage:
//   lane per edge:    u_e = E_e^T x_cam            (x staged in shared memory)
//   segmented shuffle scan over the lanes of each point: sum_e u_e
//   last lane of each point: t_p = C_p^-1 sum u
//   lane per edge:    y_cam -= E_e t_p  (shared-memory atomics into a
//                                       CTA-private 9C accumulator)
// One group barrier per stage; the accumulator is flushed to a per-CTA
// partial vector. No global atomics.
// k_fast_reduce: q = lambda x + B x + sum_CTA partials, and the PCG step
// length alpha from p.q in the last block.
#pragma once
#include "kernels.cuh"
#include "sort.cuh"
#include <vector>

namespace fg {

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Non-blocking probe of the phase (mbarrier.test_wait).
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `limit` polls and reports failure.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned limit) {
  for (unsigned i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 64) __nanosleep(64);
  }
  return false;
}

template <class TS>
struct RecWord;  // integer type filling the 28th word of an edge record
template <>
struct RecWord<float> {
  using U = uint32_t;
  __host__ __device__ static U pack(uint32_t cam, uint32_t lp) { return (cam & 0xFFFFFFu) | (lp << 24); }
  __host__ __device__ static uint32_t cam(U w) { return w & 0xFFFFFFu; }
  __host__ __device__ static uint32_t lp(U w) { return w >> 24; }
};
template <>
struct RecWord<double> {
  using U = uint64_t;
  __host__ __device__ static U pack(uint32_t cam, uint32_t lp) { return (uint64_t)cam | ((uint64_t)lp << 32); }
  __host__ __device__ static uint32_t cam(U w) { return (uint32_t)w; }
  __host__ __device__ static uint32_t lp(U w) { return (uint32_t)(w >> 32); }
};

template <class TS>
struct FastShape;  // warps per stage (one warp tile of <= 32 edges per warp)
template <>
struct FastShape<float> {
  static constexpr int WPS = 8;
};
template <>
struct FastShape<double> {
  static constexpr int WPS = 4;
};
constexpr int FAST_GROUPS = 2;  // independent stage pipelines per CTA sharing one accumulator
constexpr int FAST_STAGES = 2;  // TMA stages per group

// Point records: packed lower C^-1 from the Cholesky factor L (C^-1 = L^-T L^-1),
// plus the tile-local edge range (written once per structure, kept here).
template <class TS>
__global__ void k_fast_point_records(Layout L, const TS* factors, const uint8_t* observed, double lambda, TS* prec) {
  int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (pt >= L.nP) return;
  int64_t var = L.nC + pt;
  double ci[6];
  if (observed[var]) {
    const TS* l = factors + L.gram_offset(var);  // column major 3x3 lower
    double l00 = l[0], l10 = l[1], l20 = l[2], l11 = l[4], l21 = l[5], l22 = l[8];
    // M = L^-1 (lower)
    double m00 = 1.0 / l00, m11 = 1.0 / l11, m22 = 1.0 / l22;
    double m10 = -l10 * m00 * m11;
    double m21 = -l21 * m11 * m22;
    double m20 = -(l20 * m00 + l21 * m10) * m22;
    // C^-1 = M^T M, packed lower (00, 10, 20, 11, 21, 22)
    ci[0] = m00 * m00 + m10 * m10 + m20 * m20;
    ci[1] = m10 * m11 + m20 * m21;
    ci[2] = m20 * m22;
    ci[3] = m11 * m11 + m21 * m21;
    ci[4] = m21 * m22;
    ci[5] = m22 * m22;
  } else {
    double v = lambda != 0 ? 1.0 / lambda : 1.0;
    ci[0] = v; ci[1] = 0; ci[2] = 0; ci[3] = v; ci[4] = 0; ci[5] = v;
  }
  TS* r = prec + pt * 8;
  for (int i = 0; i < 6; ++i) r[i] = (TS)ci[i];
  r[6] = 0;
  r[7] = 0;
}

template <class TS>
__device__ __forceinline__ uint32_t rec_u32(const TS* p) {
  if (sizeof(TS) == 4) {
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
  }
  uint64_t v;
  memcpy(&v, p, 8);
  return (uint32_t)v;
}

struct FastTiles {
  const int64_t* wt_e0;  // nwt + 1: first point-major edge of each warp tile
  const int64_t* wt_p0;  // nwt + 1: first point of each warp tile
  int64_t nwt, nstages;
};

template <class TS, class TV>
struct FastSmem {
  static constexpr int WPS = FastShape<TS>::WPS, SE = WPS * 32;
  // FP32 records: the operator's accumulator is 64-bit fixed point held as two
  // 32-bit words per coordinate (see k_fast_apply)
  static constexpr bool FIXED = std::is_same<TS, float>::value;
  // fractional bits below the largest |x| (FP32 vectors 40, FP64 vectors 44)
  static constexpr int FIXED_BITS = std::is_same<TV, float>::value ? 40 : 44;
  __host__ __device__ static constexpr size_t stage_bytes() { return (size_t)SE * 28 * sizeof(TS); }
  __host__ __device__ static constexpr size_t vec_bytes(int64_t ncam) {
    return ((size_t)ncam * 9 * sizeof(TV) + 127) & ~(size_t)127;
  }
  __host__ __device__ static constexpr size_t word_bytes(int64_t ncam) {
    return ((size_t)ncam * 9 * sizeof(uint32_t) + 127) & ~(size_t)127;
  }
  // the accumulator region: two 32-bit words per coordinate (FIXED) or one TV
  __host__ __device__ static constexpr size_t acc_bytes(int64_t ncam) {
    return FIXED ? (2 * word_bytes(ncam) > vec_bytes(ncam) ? 2 * word_bytes(ncam) : vec_bytes(ncam)) : vec_bytes(ncam);
  }
  __host__ __device__ static constexpr size_t bytes(int64_t ncam, bool stage_x) {
    return acc_bytes(ncam) + (stage_x ? vec_bytes(ncam) : 0) + 128 + FAST_GROUPS * FAST_STAGES * stage_bytes();
  }
};

__device__ __forceinline__ void group_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Loads the 27 cross values and the packed index word of one edge record with
// 16-byte shared-memory loads.
template <class TV>
__device__ __forceinline__ void load_record(const float* rec, TV (&E)[27], uint32_t& cam, uint32_t& lp) {
  const float4* v = reinterpret_cast<const float4*>(rec);
  float f[28];
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    float4 a = v[i];
    f[4 * i] = a.x; f[4 * i + 1] = a.y; f[4 * i + 2] = a.z; f[4 * i + 3] = a.w;
  }
#pragma unroll
  for (int i = 0; i < 27; ++i) E[i] = (TV)f[i];
  uint32_t w = __float_as_uint(f[27]);
  cam = RecWord<float>::cam(w);
  lp = RecWord<float>::lp(w);
}
template <class TV>
__device__ __forceinline__ void load_record(const double* rec, TV (&E)[27], uint32_t& cam, uint32_t& lp) {
  const double2* v = reinterpret_cast<const double2*>(rec);
  double f[28];
#pragma unroll
  for (int i = 0; i < 14; ++i) {
    double2 a = v[i];
    f[2 * i] = a.x; f[2 * i + 1] = a.y;
  }
#pragma unroll
  for (int i = 0; i < 27; ++i) E[i] = (TV)f[i];
  uint64_t w = (uint64_t)__double_as_longlong(f[27]);
  cam = RecWord<double>::cam(w);
  lp = RecWord<double>::lp(w);
}

// The packed lower C^-1 of a point record (the first 6 of its 8 words).
template <class TS, class TV>
__device__ __forceinline__ void load_point(const TS* r, TV& c0, TV& c1, TV& c2, TV& c3, TV& c4, TV& c5) {
  if (sizeof(TS) == 4) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(r));
    const float2 b = __ldg(reinterpret_cast<const float2*>(r) + 2);
    c0 = (TV)a.x; c1 = (TV)a.y; c2 = (TV)a.z; c3 = (TV)a.w; c4 = (TV)b.x; c5 = (TV)b.y;
  } else {
    const double2* q = reinterpret_cast<const double2*>(r);
    const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    c0 = (TV)a.x; c1 = (TV)a.y; c2 = (TV)b.x; c3 = (TV)b.y; c4 = (TV)c.x; c5 = (TV)c.y;
  }
}

// Adds 9 values to the 64-bit fixed-point accumulator held as low and high
// 32-bit words: all nine low-word atomics are issued first (their returned
// old values give the carries), then the nine high words as reductions
// without a return, so the round trips overlap instead of forming a chain.
// An FP32 value times a power of two converts exactly from FP32 (fmf != 0)
// or from FP64: the integer is the same.
template <class TV>
__device__ __forceinline__ void fixed_scatter(uint32_t* ylo, uint32_t* yhi, int64_t y0, const TV (&v)[9], double fm,
                                              float fmf) {
  uint32_t lo[9], hi[9], old[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const long long q = (std::is_same<TV, float>::value && fmf != 0.f) ? __float2ll_rn((float)v[c] * fmf)
                                                                       : __double2ll_rn((double)v[c] * fm);
    lo[c] = (uint32_t)q;
    hi[c] = (uint32_t)((unsigned long long)q >> 32);
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) old[c] = atomicAdd(&ylo[y0 + c], lo[c]);
#pragma unroll
  for (int c = 0; c < 9; ++c) atomicAdd(&yhi[y0 + c], hi[c] + ((uint32_t)(old[c] + lo[c]) < old[c] ? 1u : 0u));
}

// fx_mul in FP32 for fixed_scatter: nonzero only when it is exactly
// representable as a normal FP32 number (a power of two in [2^-120, 2^120]).
__device__ __forceinline__ float fixed_mulf(double fm) {
  return (fm >= 0x1p-120 && fm <= 0x1p120) ? (float)fm : 0.f;
}

// Inclusive segmented sum over the lanes of each run of equal keys, with an
// early exit once no lane has a run predecessor at the current distance
// (short tracks need 3 steps instead of 5).
template <class TV>
__device__ __forceinline__ void seg_scan3(TV& u0, TV& u1, TV& u2, uint32_t key, int lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t lo = __shfl_up_sync(0xffffffffu, key, off);
    const bool take = lane >= off && lo == key;
    if (!__any_sync(0xffffffffu, take)) break;
    const TV v0 = __shfl_up_sync(0xffffffffu, u0, off), v1 = __shfl_up_sync(0xffffffffu, u1, off);
    const TV v2 = __shfl_up_sync(0xffffffffu, u2, off);
    if (take) {
      u0 += v0;
      u1 += v1;
      u2 += v2;
    }
  }
}

// Modes of the edge-record pass (all read every record once):
//   FAST_APPLY:   partials <- -E C^-1 E^T x                 (x = z + beta p)
//   FAST_RHS:     partials <- -E w_p, w_p read per point     (src/schur.rs:230-242)
//   FAST_RECOVER: step_p = C^-1 (w_p - sum_e E_e^T z_c) / D_p (src/schur.rs:319-343)
enum FastMode { FAST_APPLY = 0, FAST_RHS = 1, FAST_RECOVER = 2 };
struct FastExtra {
  const double* wp;      // RHS: C^-1 (-g/D) per eliminated coordinate; RECOVER: g (index 3p+i)
  const double* scales;  // RECOVER: D for eliminated coordinates (index 3p+i)
  double* step;          // RECOVER: output, eliminated coordinates (index 3p+i)
};

// skip:  return at once when *skip != 0 (finished PCG)
// gate:  return at once when *gate == 0 (conditional residual replacement)
template <class TS, class TV, bool XS, int MODE = FAST_APPLY>
__global__ void __launch_bounds__(FAST_GROUPS * FastShape<TS>::WPS * 32, 1)
    k_fast_apply(int64_t ncam, FastTiles tiles, const TS* erec, const TS* prec, const TV* z, const TV* pv,
                 const double* beta, TV* partials, const int* skip, const int* gate, int* error, FastExtra ex) {
  constexpr int WPS = FastShape<TS>::WPS, GT = WPS * 32, NTHR = FAST_GROUPS * GT, SE = WPS * 32;
  if (skip && *skip) return;
  if (gate && !*gate) return;
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31;
  const int g = tid / GT, w = (tid % GT) >> 5, gtid = tid % GT;
  const int64_t ny = ncam * 9;
  const size_t vb = FastSmem<TS, TV>::vec_bytes(ncam);
  // the accumulator ys (every mode but FAST_RECOVER, which scatters nothing)
  // and, with XS, the staged x. FP32 operator (FIXED): the accumulator is 64-bit
  // fixed point in units of 2^-k (k from the largest |x|), held as low and high
  // 32-bit words; a contribution adds its low word with a 32-bit atomic whose
  // returned old value gives the carry, then high word + carry (two integer
  // shared-memory atomics cost less than one FP32 atomic here, and the sums are
  // exact, so the result does not depend on the order of the atomics).
  constexpr bool FIXED = FastSmem<TS, TV>::FIXED && MODE == FAST_APPLY;
  constexpr bool NEED_Y = MODE != FAST_RECOVER;
  const size_t acc = FastSmem<TS, TV>::acc_bytes(ncam);
  const size_t x0 = NEED_Y ? acc : 0, bar0 = x0 + (XS ? vb : 0);
  TV* ys = reinterpret_cast<TV*>(smem);
  uint32_t* ylo = reinterpret_cast<uint32_t*>(smem);
  uint32_t* yhi = reinterpret_cast<uint32_t*>(smem + FastSmem<TS, TV>::word_bytes(ncam));
  TV* xs = reinterpret_cast<TV*>(smem + x0);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + bar0);
  unsigned char* stage_base = smem + bar0 + 128;
  constexpr size_t sbytes = FastSmem<TS, TV>::stage_bytes();
  unsigned char* gstage = stage_base + (size_t)g * FAST_STAGES * sbytes;
  uint64_t* gbar = bars + FAST_STAGES * g;
  volatile int* fail = reinterpret_cast<volatile int*>(bars + FAST_GROUPS * FAST_STAGES);  // one flag per group

  const TV bv = pv ? (TV)*beta : (TV)0;
  double xmax = 0.0;
  for (int64_t i = tid; i < ny; i += NTHR) {
    if (NEED_Y) {
      if (FIXED) {
        ylo[i] = 0;
        yhi[i] = 0;
      } else {
        ys[i] = 0;
      }
    }
    const TV xi = pv ? z[i] + bv * pv[i] : z[i];
    if (XS) xs[i] = xi;
    if (FIXED) xmax = isfinite((double)xi) ? fmax(xmax, fabs((double)xi)) : (double)INFINITY;
  }
  // FIXED: every block sees the same x, so every block derives the same unit
  __shared__ double wmax[32];
  __shared__ double fx_mul_s, fx_unit_s;
  if (FIXED) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
    if (lane == 0) wmax[tid >> 5] = xmax;
  }
  if (tid == 0) {
    for (int i = 0; i < FAST_GROUPS * FAST_STAGES; ++i) mbar_init(&bars[i], 1);
    for (int i = 0; i < FAST_GROUPS; ++i) fail[i] = 0;
    mbar_fence_init();
  }
  __syncthreads();
  if (FIXED && tid == 0) {
    double m = 0.0;
    for (int w2 = 0; w2 < NTHR / 32; ++w2) m = fmax(m, wmax[w2]);
    // unit 2^-k with |x| < 2^(B-k), B = 40 (FP32 vectors) or 44: a contribution
    // (at most a few hundred |x|max) stays below 2^(B+9) units and a block's
    // partial sums far below 2^63
    constexpr int B = FastSmem<TS, TV>::FIXED_BITS;
    int e = 0;
    if (m > 0.0 && isfinite(m)) frexp(m, &e);
    fx_mul_s = isfinite(m) ? ldexp(1.0, B - e) : 0.0;
    fx_unit_s = isfinite(m) ? ldexp(1.0, e - B) : (double)NAN;
  }
  if (FIXED) __syncthreads();
  const double fx_mul = FIXED ? fx_mul_s : 0.0;
  const float fx_mulf = FIXED ? fixed_mulf(fx_mul_s) : 0.f;

  auto issue = [&](int64_t sidx, int b) {
    int64_t wt0 = sidx * WPS, wt1 = min(wt0 + WPS, tiles.nwt);
    int64_t e0 = tiles.wt_e0[wt0], e1 = tiles.wt_e0[wt1];
    unsigned eb = (unsigned)((e1 - e0) * 28 * sizeof(TS));
    unsigned char* dst = gstage + b * sbytes;
    mbar_expect_tx(&gbar[b], eb);
    if (eb) tma_load_1d(dst, erec + e0 * 28, eb, &gbar[b]);
  };

  const int64_t first = (int64_t)blockIdx.x * FAST_GROUPS + g, stride = (int64_t)gridDim.x * FAST_GROUPS;
  if (gtid == 0)
    for (int b = 0; b < FAST_STAGES; ++b)
      if (first + b * stride < tiles.nstages) issue(first + b * stride, b);
  bool failed = false;
  int k = 0;
  for (int64_t sidx = first; sidx < tiles.nstages; sidx += stride, ++k) {
    const int b = k % FAST_STAGES;
    const unsigned parity = (k / FAST_STAGES) & 1;
    // Bounded wait; a timeout is made uniform across the group through the
    // flag read after the stage barrier, so no thread is left at the barrier.
    // The warp tile's bounds come from global memory: load them before the
    // wait so their latency overlaps the stage's arrival.
    const int64_t wt = sidx * WPS + w;
    int64_t e_lo = 0, gp0 = 0;  // gp0: global index of the tile's first point
    int cnt = 0;
    if (wt < tiles.nwt) {
      const int64_t se0 = tiles.wt_e0[sidx * WPS];
      const int64_t ew = tiles.wt_e0[wt], ew1 = tiles.wt_e0[wt + 1];
      gp0 = tiles.wt_p0[wt];
      e_lo = ew - se0;
      cnt = (int)(ew1 - ew);
    }
    const bool ok = mbar_wait_bounded(&gbar[b], parity, 1u << 22);
    if (!ok) fail[g] = 1;
    if (ok && wt < tiles.nwt) {
      const TS* er = reinterpret_cast<const TS*>(gstage + b * sbytes);
      TV E[27];
      uint32_t cam = 0, lp = 0xFFFFu;
      TV u0 = 0, u1 = 0, u2 = 0;
      TV c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0;  // the point's C^-1 (packed lower)
      if (lane < cnt) {
        load_record<TV>(er + (size_t)(e_lo + lane) * 28, E, cam, lp);
        // every lane fetches its point's C^-1 now (L1 serves the point's other
        // lanes), so its latency overlaps the x gather and the scan
        if (MODE != FAST_RHS) load_point<TS, TV>(prec + (gp0 + lp) * 8, c0, c1, c2, c3, c4, c5);
      }
      if (MODE != FAST_RHS && lane < cnt) {
        TV xc[9];
        if (XS) {
#pragma unroll
          for (int c = 0; c < 9; ++c) xc[c] = xs[(int64_t)cam * 9 + c];
        } else {
#pragma unroll
          for (int c = 0; c < 9; ++c) {
            int64_t i = (int64_t)cam * 9 + c;
            xc[c] = pv ? z[i] + bv * pv[i] : z[i];
          }
        }
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          u0 += E[c] * xc[c];
          u1 += E[9 + c] * xc[c];
          u2 += E[18 + c] * xc[c];
        }
      }
      // segmented inclusive scan over the lanes of each point (inactive lanes
      // get keys of their own)
      seg_scan3<TV>(u0, u1, u2, lane < cnt ? lp : 0x10000u + lane, lane);
      uint32_t lpn = __shfl_down_sync(0xffffffffu, lp, 1);
      bool last = lane < cnt && (lane == cnt - 1 || lpn != lp);
      TV t0 = 0, t1 = 0, t2 = 0;
      if (MODE == FAST_RHS) {
        if (last) {
          const double* w3 = ex.wp + 3 * (gp0 + lp);
          t0 = (TV)w3[0];
          t1 = (TV)w3[1];
          t2 = (TV)w3[2];
        }
      } else if (last) {
        if (MODE == FAST_RECOVER) {
          const int64_t q = 3 * (gp0 + lp);
          TV a0 = (TV)(-ex.wp[q] / ex.scales[q]) - u0, a1 = (TV)(-ex.wp[q + 1] / ex.scales[q + 1]) - u1;
          TV a2 = (TV)(-ex.wp[q + 2] / ex.scales[q + 2]) - u2;
          ex.step[q] = (double)(c0 * a0 + c1 * a1 + c2 * a2) / ex.scales[q];
          ex.step[q + 1] = (double)(c1 * a0 + c3 * a1 + c4 * a2) / ex.scales[q + 1];
          ex.step[q + 2] = (double)(c2 * a0 + c4 * a1 + c5 * a2) / ex.scales[q + 2];
        } else {
          t0 = c0 * u0 + c1 * u1 + c2 * u2;
          t1 = c1 * u0 + c3 * u1 + c4 * u2;
          t2 = c2 * u0 + c4 * u1 + c5 * u2;
        }
      }
      if (MODE != FAST_RECOVER) {
        // each lane takes its point's t from the point's last lane: the first
        // flagged lane at or after this one
        const unsigned ends = __ballot_sync(0xffffffffu, last) & ~((1u << lane) - 1u);
        const int src = ends ? __ffs(ends) - 1 : lane;
        t0 = __shfl_sync(0xffffffffu, t0, src);
        t1 = __shfl_sync(0xffffffffu, t1, src);
        t2 = __shfl_sync(0xffffffffu, t2, src);
      }
      if (MODE != FAST_RECOVER && lane < cnt) {
        if (FIXED) {
          TV v[9];
#pragma unroll
          for (int c = 0; c < 9; ++c) v[c] = -(E[c] * t0 + E[9 + c] * t1 + E[18 + c] * t2);
          fixed_scatter(ylo, yhi, (int64_t)cam * 9, v, fx_mul, fx_mulf);
        } else {
          TV* y = ys + (int64_t)cam * 9;
#pragma unroll
          for (int c = 0; c < 9; ++c) atomicAdd(&y[c], -(E[c] * t0 + E[9 + c] * t1 + E[18 + c] * t2));
        }
      }
    }
    group_sync(1 + g, GT);  // every warp of the group is done with stage b
    if (fail[g]) {
      failed = true;
      break;
    }
    if (gtid == 0 && sidx + FAST_STAGES * stride < tiles.nstages) issue(sidx + FAST_STAGES * stride, b);
  }
  if (failed) {
    if (gtid == 0) atomicExch(error, 1);
    for (int b = 0; b < FAST_STAGES; ++b) mbar_wait_bounded(&gbar[b], ((k + b) / FAST_STAGES) & 1, 1u << 16);
  }
  __syncthreads();
  if (MODE == FAST_RECOVER) return;
  TV* out = partials + (int64_t)blockIdx.x * ny;
  if (FIXED) {
    const double unit = fx_unit_s;
    for (int64_t i = tid; i < ny; i += NTHR) {
      const long long q = (long long)(((unsigned long long)yhi[i] << 32) | (unsigned long long)ylo[i]);
      out[i] = (TV)((double)q * unit);
    }
  } else {
    for (int64_t i = tid; i < ny; i += NTHR) out[i] = ys[i];
  }
}

// Direct variant of the FAST_APPLY pass: no shared-memory staging of records.
// Each warp grid-strides over warp tiles; a lane loads its 112/224-byte record
// with 16-byte global loads (a tile's records are contiguous, so a warp's
// loads coalesce), reduces its point with the same segmented shuffle scan and
// re-reads E from L1 for the scatter, which keeps registers low enough for
// 1,024 threads per SM. No stage barriers; x staged in shared memory.
constexpr int DIRECT_THREADS = 1024;
template <class TS>
__device__ __forceinline__ void load_cross_global(const TS* rec, float (&E)[27], uint32_t& cam, uint32_t& lp);
template <>
__device__ __forceinline__ void load_cross_global<float>(const float* rec, float (&E)[27], uint32_t& cam,
                                                          uint32_t& lp) {
  const float4* v = reinterpret_cast<const float4*>(rec);
  float f[28];
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    float4 a = __ldg(v + i);
    f[4 * i] = a.x; f[4 * i + 1] = a.y; f[4 * i + 2] = a.z; f[4 * i + 3] = a.w;
  }
#pragma unroll
  for (int i = 0; i < 27; ++i) E[i] = f[i];
  uint32_t w = __float_as_uint(f[27]);
  cam = RecWord<float>::cam(w);
  lp = RecWord<float>::lp(w);
}

template <bool XS>
__global__ void __launch_bounds__(DIRECT_THREADS, 1)
    k_fast_apply_direct(int64_t ncam, FastTiles tiles, const float* erec, const float* prec, const float* z,
                        const float* pv, const double* beta, float* partials, const int* skip, const int* gate) {
  if (skip && *skip) return;
  if (gate && !*gate) return;
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  constexpr int NW = DIRECT_THREADS / 32;
  const int64_t ny = ncam * 9;
  const size_t vb = FastSmem<float, float>::vec_bytes(ncam);
  float* ys = reinterpret_cast<float*>(smem);
  float* xs = reinterpret_cast<float*>(smem + vb);
  float* tpw = reinterpret_cast<float*>(smem + vb * (XS ? 2 : 1)) + w * 96;
  const float bv = pv ? (float)*beta : 0.f;
  for (int64_t i = tid; i < ny; i += DIRECT_THREADS) {
    ys[i] = 0;
    if (XS) xs[i] = pv ? z[i] + bv * pv[i] : z[i];
  }
  __syncthreads();
  for (int64_t wt = (int64_t)blockIdx.x * NW + w; wt < tiles.nwt; wt += (int64_t)gridDim.x * NW) {
    const int64_t e0 = tiles.wt_e0[wt];
    const int cnt = (int)(tiles.wt_e0[wt + 1] - e0);
    const int64_t p0 = tiles.wt_p0[wt];
    const float* rec = erec + (e0 + lane) * 28;
    uint32_t cam = 0, lp = 0xFFFFu;
    float u0 = 0, u1 = 0, u2 = 0;
    if (lane < cnt) {
      float E[27];
      load_cross_global<float>(rec, E, cam, lp);
      float xc[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        int64_t i = (int64_t)cam * 9 + c;
        xc[c] = XS ? xs[i] : (pv ? z[i] + bv * pv[i] : z[i]);
      }
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        u0 += E[c] * xc[c];
        u1 += E[9 + c] * xc[c];
        u2 += E[18 + c] * xc[c];
      }
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      float v0 = __shfl_up_sync(0xffffffffu, u0, off), v1 = __shfl_up_sync(0xffffffffu, u1, off);
      float v2 = __shfl_up_sync(0xffffffffu, u2, off);
      uint32_t lo = __shfl_up_sync(0xffffffffu, lp, off);
      if (lane >= off && lo == lp) {
        u0 += v0;
        u1 += v1;
        u2 += v2;
      }
    }
    uint32_t lpn = __shfl_down_sync(0xffffffffu, lp, 1);
    if (lane < cnt && (lane == cnt - 1 || lpn != lp)) {
      const float4* r = reinterpret_cast<const float4*>(prec + (p0 + lp) * 8);
      float4 ca = __ldg(r), cb = __ldg(r + 1);
      tpw[lp * 3] = ca.x * u0 + ca.y * u1 + ca.z * u2;
      tpw[lp * 3 + 1] = ca.y * u0 + ca.w * u1 + cb.x * u2;
      tpw[lp * 3 + 2] = ca.z * u0 + cb.x * u1 + cb.y * u2;
    }
    __syncwarp();
    if (lane < cnt) {
      float E[27];
      uint32_t c2, l2;
      load_cross_global<float>(rec, E, c2, l2);  // L1 hit: same lines as above
      float t0 = tpw[lp * 3], t1 = tpw[lp * 3 + 1], t2 = tpw[lp * 3 + 2];
      float* y = ys + (int64_t)cam * 9;
#pragma unroll
      for (int c = 0; c < 9; ++c) atomicAdd(&y[c], -(E[c] * t0 + E[9 + c] * t1 + E[18 + c] * t2));
    }
    __syncwarp();
  }
  __syncthreads();
  float* out = partials + (int64_t)blockIdx.x * ny;
  for (int64_t i = tid; i < ny; i += DIRECT_THREADS) out[i] = ys[i];
}

// Prefetching variant of the direct pass: 512 threads per SM, and each warp
// issues the 16-byte loads of its NEXT warp tile (records and tile bounds)
// into registers before it works on the current one, so the HBM latency of
// one tile overlaps the shuffle scan, the point solve and the shared-memory
// scatter of the previous tile. E stays in registers for the scatter (no
// L1 re-read).
constexpr int PF_THREADS = 512;
template <bool XS>
__global__ void __launch_bounds__(PF_THREADS, 1)
    k_fast_apply_pf(int64_t ncam, FastTiles tiles, const float* erec, const float* prec, const float* z,
                    const float* pv, const double* beta, float* partials, const int* skip, const int* gate) {
  if (skip && *skip) return;
  if (gate && !*gate) return;
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  constexpr int NW = PF_THREADS / 32;
  const int64_t ny = ncam * 9;
  const size_t vb = FastSmem<float, float>::vec_bytes(ncam);
  float* ys = reinterpret_cast<float*>(smem);
  float* xs = reinterpret_cast<float*>(smem + vb);
  float* tpw = reinterpret_cast<float*>(smem + vb * (XS ? 2 : 1)) + w * 96;
  const float bv = pv ? (float)*beta : 0.f;
  for (int64_t i = tid; i < ny; i += PF_THREADS) {
    ys[i] = 0;
    if (XS) xs[i] = pv ? z[i] + bv * pv[i] : z[i];
  }
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * NW;
  int64_t wt = (int64_t)blockIdx.x * NW + w;
  float4 nb[7];
  int ncnt = 0;
  int64_t np0 = 0;
  if (wt < tiles.nwt) {
    const int64_t e0 = tiles.wt_e0[wt];
    ncnt = (int)(tiles.wt_e0[wt + 1] - e0);
    np0 = tiles.wt_p0[wt];
    if (lane < ncnt) {
      const float4* v = reinterpret_cast<const float4*>(erec + (e0 + lane) * 28);
#pragma unroll
      for (int i = 0; i < 7; ++i) nb[i] = __ldg(v + i);
    }
  }
  for (; wt < tiles.nwt; wt += stride) {
    // take the prefetched tile
    const int cnt = ncnt;
    const int64_t p0 = np0;
    float E[27];
    uint32_t cam = 0, lp = 0xFFFFu;
    if (lane < cnt) {
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        E[4 * i] = nb[i].x;
        E[4 * i + 1] = nb[i].y;
        E[4 * i + 2] = nb[i].z;
        E[4 * i + 3] = nb[i].w;
      }
      E[24] = nb[6].x;
      E[25] = nb[6].y;
      E[26] = nb[6].z;
      const uint32_t wd = __float_as_uint(nb[6].w);
      cam = RecWord<float>::cam(wd);
      lp = RecWord<float>::lp(wd);
    }
    // issue the next tile's loads
    const int64_t wn = wt + stride;
    ncnt = 0;
    if (wn < tiles.nwt) {
      const int64_t e0 = tiles.wt_e0[wn];
      ncnt = (int)(tiles.wt_e0[wn + 1] - e0);
      np0 = tiles.wt_p0[wn];
      if (lane < ncnt) {
        const float4* v = reinterpret_cast<const float4*>(erec + (e0 + lane) * 28);
#pragma unroll
        for (int i = 0; i < 7; ++i) nb[i] = __ldg(v + i);
      }
    }
    float u0 = 0, u1 = 0, u2 = 0;
    if (lane < cnt) {
      float xc[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        const int64_t i = (int64_t)cam * 9 + c;
        xc[c] = XS ? xs[i] : (pv ? z[i] + bv * pv[i] : z[i]);
      }
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        u0 += E[c] * xc[c];
        u1 += E[9 + c] * xc[c];
        u2 += E[18 + c] * xc[c];
      }
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      float v0 = __shfl_up_sync(0xffffffffu, u0, off), v1 = __shfl_up_sync(0xffffffffu, u1, off);
      float v2 = __shfl_up_sync(0xffffffffu, u2, off);
      uint32_t lo = __shfl_up_sync(0xffffffffu, lp, off);
      if (lane >= off && lo == lp) {
        u0 += v0;
        u1 += v1;
        u2 += v2;
      }
    }
    const uint32_t lpn = __shfl_down_sync(0xffffffffu, lp, 1);
    if (lane < cnt && (lane == cnt - 1 || lpn != lp)) {
      const float4* r = reinterpret_cast<const float4*>(prec + (p0 + lp) * 8);
      float4 ca = __ldg(r), cb = __ldg(r + 1);
      tpw[lp * 3] = ca.x * u0 + ca.y * u1 + ca.z * u2;
      tpw[lp * 3 + 1] = ca.y * u0 + ca.w * u1 + cb.x * u2;
      tpw[lp * 3 + 2] = ca.z * u0 + cb.x * u1 + cb.y * u2;
    }
    __syncwarp();
    if (lane < cnt) {
      const float t0 = tpw[lp * 3], t1 = tpw[lp * 3 + 1], t2 = tpw[lp * 3 + 2];
      float* y = ys + (int64_t)cam * 9;
#pragma unroll
      for (int c = 0; c < 9; ++c) atomicAdd(&y[c], -(E[c] * t0 + E[9 + c] * t1 + E[18 + c] * t2));
    }
    __syncwarp();
  }
  __syncthreads();
  float* out = partials + (int64_t)blockIdx.x * ny;
  for (int64_t i = tid; i < ny; i += PF_THREADS) out[i] = ys[i];
}

// q = lambda x + B x + sum_b partials[b] with x = z (+ beta p); 32 coordinates
// x 32 rows of partial vectors per block, so each thread sums only a handful
// of partials (one or two rounds of independent loads: the pass is latency-
// bound, 5 MB). Optional p.q -> alpha in the last block.
constexpr int FR_ROWS = 32;
template <class TS, class TV>
__global__ void __launch_bounds__(FR_ROWS * 32) k_fast_reduce(int64_t ncam, int nparts, const TV* partials, const TS* gram,
                                                      const uint8_t* observed, const TV* z, const TV* pv,
                                                      const double* beta, double lambda, const double* lam_dev,
                                                      int use_gram, TV* q, double* dparts,
                                                      PcgState* st, const int* gate) {
  pdl_wait();
  pdl_trigger();
  if (st && st->done) return;
  if (gate && !*gate) return;
  __shared__ TV acc_s[FR_ROWS][33];
  const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
  const int64_t ny = ncam * 9;
  const int64_t i = (int64_t)blockIdx.x * 32 + lx;
  TV acc = 0;
  if (i < ny) {
    int b = ly;
    for (; b + 3 * FR_ROWS < nparts; b += 4 * FR_ROWS) {
      TV a0 = partials[(int64_t)b * ny + i], a1 = partials[(int64_t)(b + FR_ROWS) * ny + i];
      TV a2 = partials[(int64_t)(b + 2 * FR_ROWS) * ny + i], a3 = partials[(int64_t)(b + 3 * FR_ROWS) * ny + i];
      acc += (a0 + a1) + (a2 + a3);
    }
    for (; b < nparts; b += FR_ROWS) acc += partials[(int64_t)b * ny + i];
  }
  acc_s[ly][lx] = acc;
  __syncthreads();
  double dot = 0;
  if (ly == 0 && i < ny) {
    TV sum = 0;
#pragma unroll
    for (int k = 0; k < FR_ROWS; ++k) sum += acc_s[k][lx];
    const TV bv = pv ? (TV)*beta : (TV)0;
    int64_t cam = i / 9;
    int r = (int)(i % 9);
    TV xi = pv ? z[i] + bv * pv[i] : z[i];
    const double lam = lam_dev ? *lam_dev : lambda;
    TV v = (TV)lam * xi;
    if (use_gram && observed[cam]) {
      const TS* g = gram + cam * 81;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        int64_t k = cam * 9 + j;
        TV xj = pv ? z[k] + bv * pv[k] : z[k];
        TS gv = j >= r ? g[r * 9 + j] : g[j * 9 + r];
        v += (TV)gv * xj;
      }
    }
    v += sum;
    q[i] = v;
    dot = (double)xi * (double)v;
  }
  if (!st) return;
  double s[1] = {dot};
  block_sums<1>(s);
  if (threadIdx.x == 0) dparts[blockIdx.x] = s[0];
  if (arrive_last(&st->counter0)) {
    double tot[1];
    finish_sums<1>(dparts, tot);
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

// Coarse Galerkin matrix of the two-level PCG in one pass over the edge
// records: E(lambda) = W^T S W with S = lambda I + B - E C^-1 E^T, computed as
//   lambda W^T W + sum_cam W_cam^T B_cam W_cam           (k_coarse_cams)
//   - sum_p u_p^T C_p^-1 u_p, u_p = sum_{e in p} E_e^T W_cam(e)   (k_coarse_tiles)
// instead of nk operator applications. k_coarse_tiles walks the operator's
// warp tiles (lane per edge, 16-byte record loads), sums u over each point's
// lanes with the same segmented shuffle scan, and the point's last lane adds
// u^T C^-1 u. W is staged camera-major, coordinate-major, vector-minor with 8
// slots: wc[cam * 72 + c * 8 + a]. out: nk x nk (nk = 7), accumulated with
// atomics (zeroed by the caller).
constexpr int COARSE_WARPS = 8;
template <class TS>
__device__ __forceinline__ void coarse_record(const TS* rec, float (&E)[28], typename RecWord<TS>::U& word);
template <>
__device__ __forceinline__ void coarse_record<float>(const float* rec, float (&E)[28], uint32_t& word) {
  const float4* v = reinterpret_cast<const float4*>(rec);
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    const float4 a = __ldg(v + i);
    E[4 * i] = a.x; E[4 * i + 1] = a.y; E[4 * i + 2] = a.z; E[4 * i + 3] = a.w;
  }
  word = __float_as_uint(E[27]);
}
template <>
__device__ __forceinline__ void coarse_record<double>(const double* rec, float (&E)[28], uint64_t& word) {
  const double2* v = reinterpret_cast<const double2*>(rec);
#pragma unroll
  for (int i = 0; i < 14; ++i) {
    const double2 a = __ldg(v + i);
    E[2 * i] = (float)a.x; E[2 * i + 1] = (float)a.y;
    if (i == 13) word = (uint64_t)__double_as_longlong(a.y);
  }
}
// u[a] += E_e^T W_a(cam) for one edge record (the gauge's block structure, as
// in k_coarse_tiles).
template <class TS>
__device__ __forceinline__ void coarse_edge(const TS* rec, const float* wc, float (&u)[7][3]) {
  float E[28];
  typename RecWord<TS>::U word;
  coarse_record<TS>(rec, E, word);
  const float4* wv = reinterpret_cast<const float4*>(wc + (int64_t)RecWord<TS>::cam(word) * 72);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float4 lo = __ldg(wv + 2 * c);
    const float x[3] = {lo.x, lo.y, lo.z};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int p = 0; p < 3; ++p) u[a][p] += E[p * 9 + c] * x[a];
  }
#pragma unroll
  for (int c = 3; c < 6; ++c) {
    const float4 lo = __ldg(wv + 2 * c), hi = __ldg(wv + 2 * c + 1);
    const float x[4] = {lo.w, hi.x, hi.y, hi.z};
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int p = 0; p < 3; ++p) u[3 + a][p] += E[p * 9 + c] * x[a];
  }
}
// acc (packed lower 7x7) += u^T C^-1 u for one point record.
template <class TS>
__device__ __forceinline__ void coarse_point(const TS* r, const float (&u)[7][3], double (&acc)[28]) {
  const double c00 = r[0], c10 = r[1], c20 = r[2], c11 = r[3], c21 = r[4], c22 = r[5];
  int idx = 0;
#pragma unroll
  for (int a = 0; a < 7; ++a) {
    const double t0 = c00 * u[a][0] + c10 * u[a][1] + c20 * u[a][2];
    const double t1 = c10 * u[a][0] + c11 * u[a][1] + c21 * u[a][2];
    const double t2 = c20 * u[a][0] + c21 * u[a][1] + c22 * u[a][2];
#pragma unroll
    for (int b = 0; b <= a; ++b) acc[idx++] += (double)u[b][0] * t0 + (double)u[b][1] * t1 + (double)u[b][2] * t2;
  }
}

// 16-byte asynchronous global -> shared copies (cp.async, no registers held
// while in flight); wait_all makes the thread's own copies visible to it.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// A warp takes its tiles first, first + G, ... (G warps in the grid, sized to
// one resident wave): lane l holds the bounds of the warp's tile 32 c + l of
// batch c (one coalesced load per 32 tiles, read by shuffle). FP32 records:
// the next tile's records are copied into the lane's shared-memory slot
// (cp.async) while the current tile's sums and point terms are computed; FP64
// records (224 bytes) are loaded when their tile is processed.
template <class TS>
__global__ void __launch_bounds__(COARSE_WARPS * 32, 2)
    k_coarse_tiles(FastTiles tiles, const TS* erec, const TS* prec, const float* wc, double* out) {
  constexpr int NK = 7, NL = NK * (NK + 1) / 2;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double acc[NL];
#pragma unroll
  for (int k = 0; k < NL; ++k) acc[k] = 0;
  const int64_t G = (int64_t)gridDim.x * COARSE_WARPS;
  const int64_t first = (int64_t)blockIdx.x * COARSE_WARPS + w;
  const int64_t nmine = first < tiles.nwt ? (tiles.nwt - 1 - first) / G + 1 : 0;
  __shared__ int64_t sb_e0[COARSE_WARPS][32], sb_p0[COARSE_WARPS][32];
  __shared__ int sb_cnt[COARSE_WARPS][32];
  auto load_batch = [&](int64_t c) {
    const int64_t t = first + (c * 32 + lane) * G;
    __syncwarp();  // every lane has read the batch it replaces
    if (t < tiles.nwt) {
      const int64_t a = tiles.wt_e0[t];
      sb_e0[w][lane] = a;
      sb_cnt[w][lane] = (int)(tiles.wt_e0[t + 1] - a);
      sb_p0[w][lane] = tiles.wt_p0[t];
    }
    __syncwarp();
  };
  constexpr bool ASYNC = sizeof(TS) == 4;
  __shared__ __align__(16) float srec[ASYNC ? COARSE_WARPS * 32 * 28 : 4];
  float* slot = srec + (ASYNC ? (w * 32 + lane) * 28 : 0);
  // for a shallow FP32 tile k (warp-uniform, k < nmine), the copy of this
  // lane's record into its slot (the batch holding tile k is loaded first)
  auto fetch = [&](int64_t k) {
    if (k > 0 && (k & 31) == 0) load_batch(k >> 5);
    if constexpr (ASYNC) {
      const int src = (int)(k & 31);
      const int64_t e0 = sb_e0[w][src];
      const int cnt = sb_cnt[w][src];
      if (cnt <= 32 && lane < cnt) {
        const float* g = reinterpret_cast<const float*>(erec + (e0 + lane) * 28);
#pragma unroll
        for (int q = 0; q < 7; ++q) cp_async16(slot + 4 * q, g + 4 * q);
      }
      cp_async_commit();
    }
  };
  if (nmine) {
    load_batch(0);
    fetch(0);
  }
  for (int64_t k = 0; k < nmine; ++k) {
    // this tile's bounds, read before fetch(k + 1) may replace the batch
    const int64_t e0 = sb_e0[w][k & 31], p0 = sb_p0[w][k & 31];
    const int cnt = sb_cnt[w][k & 31];
    float u[NK][3];
#pragma unroll
    for (int a = 0; a < NK; ++a) u[a][0] = u[a][1] = u[a][2] = 0.f;
    if (cnt > 32) {
      // a point with more than 32 observations: chunks of 32 edges, one sum
      for (int c0 = lane; c0 < cnt; c0 += 32) coarse_edge<TS>(erec + (e0 + c0) * 28, wc, u);
      if (k + 1 < nmine) fetch(k + 1);
#pragma unroll
      for (int a = 0; a < NK; ++a)
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) u[a][p] += __shfl_xor_sync(0xffffffffu, u[a][p], o);
      if (lane == 0) coarse_point(prec + p0 * 8, u, acc);
      continue;
    }
    uint32_t lp = 0xFFFFu;
    if (lane < cnt) {
      float E[28];
      typename RecWord<TS>::U word;
      if constexpr (ASYNC) {
        cp_async_wait_all();
        const float4* v = reinterpret_cast<const float4*>(slot);
#pragma unroll
        for (int q = 0; q < 7; ++q) {
          const float4 t = v[q];
          E[4 * q] = t.x; E[4 * q + 1] = t.y; E[4 * q + 2] = t.z; E[4 * q + 3] = t.w;
        }
        word = (typename RecWord<TS>::U)__float_as_uint(E[27]);
      } else {
        coarse_record<TS>(erec + (e0 + lane) * 28, E, word);
      }
      lp = RecWord<TS>::lp(word);
      // W is the similarity gauge of k_bal_gauge: the rotation directions
      // (a < 3) move only the angle-axis coordinates 0..2, the translation
      // and scale directions (a >= 3) only the translation 3..5, and none the
      // intrinsics, so E^T W needs 6 of the 9 camera columns and 63 products.
      const float4* wv = reinterpret_cast<const float4*>(wc + (int64_t)RecWord<TS>::cam(word) * 72);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float4 lo = __ldg(wv + 2 * c);
        const float x[3] = {lo.x, lo.y, lo.z};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int p = 0; p < 3; ++p) u[a][p] += E[p * 9 + c] * x[a];
      }
#pragma unroll
      for (int c = 3; c < 6; ++c) {
        const float4 lo = __ldg(wv + 2 * c), hi = __ldg(wv + 2 * c + 1);
        const float x[4] = {lo.w, hi.x, hi.y, hi.z};
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int p = 0; p < 3; ++p) u[3 + a][p] += E[p * 9 + c] * x[a];
      }
    }
    // this tile's records are in u: the next tile's copies go out now
    if (k + 1 < nmine) fetch(k + 1);
    // segmented sums over each point's lanes; inactive lanes get keys of
    // their own, and the scan stops once no run is longer than the offset
    const uint32_t key = lane < cnt ? lp : 0x10000u + lane;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t lo = __shfl_up_sync(0xffffffffu, key, off);
      const bool take = lane >= off && lo == key;
      if (!__any_sync(0xffffffffu, take)) break;
#pragma unroll
      for (int a = 0; a < NK; ++a)
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const float v = __shfl_up_sync(0xffffffffu, u[a][p], off);
          if (take) u[a][p] += v;
        }
    }
    const uint32_t lpn = __shfl_down_sync(0xffffffffu, lp, 1);
    if (lane < cnt && (lane == cnt - 1 || lpn != lp)) coarse_point(prec + (p0 + lp) * 8, u, acc);
  }
  __shared__ double sh[COARSE_WARPS][NL];
#pragma unroll
  for (int k = 0; k < NL; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[w][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < NL) {
    double v = 0;
    for (int q = 0; q < COARSE_WARPS; ++q) v += sh[q][threadIdx.x];
    int a = 0, k = threadIdx.x;
    while (k > a) k -= ++a;  // packed lower index -> (a, b = k)
    atomicAdd(out + a * NK + k, -v);
    if (a != k) atomicAdd(out + k * NK + a, -v);
  }
}

// Camera part of the coarse matrix and the camera-major copy of W used by
// k_coarse_tiles. Each block runs four groups of 64 threads, a group per
// camera: thread (a, c) stages w_a[c], computes (B w_a + lambda w_a)[c], and
// threads 0..27 accumulate the 28 products w_b . (B + lambda) w_a (b <= a)
// over the group's cameras; a block adds its sums to out with atomics.
// B_cam: the normalized Gram block (lower, column major), wd: W row-major
// (NK x n), NK = 7.
template <class TS>
__global__ void __launch_bounds__(256) k_coarse_cams(int64_t ncam, const double* wd, const TS* gram,
                                                     const uint8_t* observed, double lambda, float* wc, int ws,
                                                     double* out) {
  constexpr int NK = 7, NL = NK * (NK + 1) / 2;
  __shared__ double w_s[4][NK][9], bw_s[4][NK][9], sum_s[4][NL];
  const int g = threadIdx.x >> 6, t = threadIdx.x & 63;
  const int64_t n = ncam * 9;
  int pa = 0, pb = 0;  // thread t < NL owns the pair (pa, pb), pb <= pa
  if (t < NL) {
    while ((pa + 1) * (pa + 2) / 2 <= t) ++pa;
    pb = t - pa * (pa + 1) / 2;
  }
  double acc = 0;
  // uniform trip count across the block (the barriers), a group idles past ncam
  for (int64_t base = (int64_t)blockIdx.x * 4; base < ncam; base += (int64_t)gridDim.x * 4) {
    const int64_t cam = base + g;
    const bool live = cam < ncam;
    const int a = t / 9, c = t % 9;
    if (live && t < NK * 9) {
      const double v = wd[a * n + cam * 9 + c];
      w_s[g][a][c] = v;
      wc[cam * ws + c * 8 + a] = (float)v;
    }
    __syncthreads();
    if (live && t < NK * 9) {  // row c of (B + lambda) w_a
      const TS* gb = gram + cam * 81;
      double v = lambda * w_s[g][a][c];
      if (observed[cam])
#pragma unroll
        for (int k = 0; k < 9; ++k) v += (double)(c >= k ? gb[k * 9 + c] : gb[c * 9 + k]) * w_s[g][a][k];
      bw_s[g][a][c] = v;
    }
    __syncthreads();
    if (live && t < NL) {
      double v = 0;
#pragma unroll
      for (int r = 0; r < 9; ++r) v += w_s[g][pb][r] * bw_s[g][pa][r];
      acc += v;
    }
    __syncthreads();
  }
  if (t < NL) sum_s[g][t] = acc;
  __syncthreads();
  if (threadIdx.x < NL) {
    const double v = sum_s[0][t] + sum_s[1][t] + sum_s[2][t] + sum_s[3][t];
    atomicAdd(out + pa * NK + pb, v);
    if (pa != pb) atomicAdd(out + pb * NK + pa, v);
  }
}

// Warp tiles over point-major edges, built on the device: each segment of
// TILE_SEG points is tiled greedily (contiguous point ranges of at most 32
// edges and 32 points, the first tile starting at the segment's first point),
// one single-warp CTA per segment. The warp stages the segment's point offsets
// in shared memory with coalesced loads; lane 0 walks them there (four points
// per step, loads ahead of the greedy decisions) and records each point's
// tile start, so the sequential greedy costs neither a memory round trip nor
// a shuffle per point. Pass 0 counts each segment's tiles and flags a point
// with more than 32 edges; after an exclusive scan of the counts, pass 1
// writes each tile's first edge and point and, lane per point, every edge's
// tile-local point index.
constexpr int TILE_SEG = 1024;
__global__ void __launch_bounds__(32) k_fast_tiles(int pass, int64_t npt, const int64_t* pt_off, uint32_t* seg,
                                                   uint32_t* total, uint32_t* too_deep, int64_t* e0, int64_t* p0,
                                                   uint32_t* lp) {
  __shared__ int64_t soff[TILE_SEG + 1];
  __shared__ int32_t stp[TILE_SEG];
  const int64_t s = blockIdx.x;
  const int lane = threadIdx.x;
  if (s >= (npt + TILE_SEG - 1) / TILE_SEG) return;  // no points: nothing to tile
  const int64_t pa = s * TILE_SEG, pb = min(pa + TILE_SEG, npt);
  const int np = (int)(pb - pa);
  bool deep = false;
  for (int i = lane; i <= np; i += 32) soff[i] = pt_off[pa + i];
  __syncwarp();
  for (int i = lane; i < np; i += 32) deep |= soff[i + 1] - soff[i] > 32;
  if (lane == 0) {
    int64_t te = soff[0];
    int tp = 0;  // segment-local first point of the current tile
    uint32_t t = pass ? seg[s] : 0u, count = 1;
    if (pass) {
      e0[t] = te;
      p0[t] = pa;
    }
    stp[0] = 0;
    for (int q0 = 1; q0 < np; q0 += 4) {
      int64_t ka[4], kb[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        ka[j] = soff[min(q0 + j, np)];
        kb[j] = soff[min(q0 + j + 1, np)];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int q = q0 + j;
        if (q < np) {
          if (kb[j] - te > 32 || q + 1 - tp > 32) {
            te = ka[j];
            tp = q;
            ++count;
            if (pass) {
              ++t;
              e0[t] = te;
              p0[t] = pa + q;
            }
          }
          stp[q] = tp;
        }
      }
    }
    if (!pass) seg[s] = count;
    if (pass && s == (npt + TILE_SEG - 1) / TILE_SEG - 1) {
      e0[*total] = pt_off[npt];
      p0[*total] = npt;
    }
  }
  if (!pass && __any_sync(0xffffffffu, deep) && lane == 0) *too_deep = 1u;
  if (pass) {
    __syncwarp();
    for (int q = lane; q < np; q += 32) {
      const uint32_t v = (uint32_t)(q - stp[q]);
      for (int64_t k = soff[q]; k < soff[q + 1]; ++k) lp[k] = v;
    }
  }
}

}  // namespace fg

#include "ring.cuh"

namespace fg {

template <class TS>
struct FastPath {
  bool on = false;          // records are current and the shape qualifies
  bool structure = false;   // tiles and local indices built for the current structure
  bool disabled = false;    // force the generic operator (tests)
  bool has_deep = false;    // some point has more than 32 observations (a tile of its own)
  bool global_acc = false;  // FP32 records: the camera sums do not fit one SM (ring kernel, global accumulator)
  int64_t nwt = 0, nstages = 0;
  int grid = 0;
  DBuf<unsigned char> d_gacc;  // global accumulator of the ring kernel (cleared by its reduction)
  unsigned poll_limit = RING_POLL_LIMIT;  // consumer-wait polls of the ring kernel
  DBuf<int64_t> d_pbeg, d_ebeg;
  DBuf<uint32_t> d_lp;
  DBuf<TS> d_erec, d_prec;
  DBuf<float> d_parts_f;
  DBuf<double> d_parts_d;
  DBuf<int> d_error;

  bool enabled() const { return on && !disabled; }
  bool tuned = false;  // operator variant chosen for the current structure
  void invalidate() {
    on = false;
    structure = false;
    tuned = false;
  }

  // Tiles for the current structure from the device point offsets; a point
  // with more than 32 observations becomes a tile of its own, which only the
  // FP32 ring kernel and the coarse pass handle (the FP64 records then keep
  // the generic operator).
  DBuf<uint32_t> d_tile_aux;  // per-segment tile counts | total | too-deep flag
  HBuf<uint32_t> h_tile_aux;
  template <class Impl>
  fg_status build(Impl& s) {
    const int64_t nP = (int64_t)s.nP, nseg = (nP + TILE_SEG - 1) / TILE_SEG;
    cudaStream_t st = s.st;
    FG_TRY(d_tile_aux.resize((size_t)nseg + 2));
    FG_TRY(h_tile_aux.resize(2));
    FG_TRY(d_pbeg.resize((size_t)nP + 1));
    FG_TRY(d_ebeg.resize((size_t)nP + 1));
    FG_TRY(d_lp.resize(std::max<size_t>(s.nedges, 1)));
    uint32_t* aux = d_tile_aux.get();
    FG_CUDA(cudaMemsetAsync(aux, 0, ((size_t)nseg + 2) * sizeof(uint32_t), st));
    const int64_t* off = s.d_pt_edge_off.get();
    FG_LAUNCH(k_fast_tiles, (unsigned)std::max<int64_t>(nseg, 1), 32, 0, st, 0, nP, off, aux, aux + nseg, aux + nseg + 1,
              d_ebeg.get(), d_pbeg.get(), d_lp.get());
    FG_LAUNCH(k_scan_exclusive_u32, 1, 1024, 0, st, aux, nseg, aux + nseg);
    FG_LAUNCH(k_fast_tiles, (unsigned)std::max<int64_t>(nseg, 1), 32, 0, st, 1, nP, off, aux, aux + nseg, aux + nseg + 1,
              d_ebeg.get(), d_pbeg.get(), d_lp.get());
    FG_CUDA(cudaMemcpyAsync(h_tile_aux.get(), aux + nseg, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    has_deep = h_tile_aux.get()[1] != 0;
    if (has_deep && !std::is_same<TS, float>::value) return FG_OK;
    nwt = (int64_t)h_tile_aux.get()[0];
    nstages = (nwt + FastShape<TS>::WPS - 1) / FastShape<TS>::WPS;
    FG_TRY(d_erec.resize(std::max<size_t>(s.nedges * 28, 1)));
    FG_TRY(d_prec.resize(std::max<size_t>(s.nP * 8, 1)));
    FG_TRY(d_error.resize(1));
    FG_CUDA(cudaMemsetAsync(d_error.get(), 0, sizeof(int), st));
    structure = true;
    return FG_OK;
  }

  // Whether the BAL single-pass operator applies to this system; builds the
  // tiles once per structure. The caller then writes the edge records.
  template <class Impl>
  bool ready_for(Impl& s) {
    if (disabled || s.cw != 9 || s.pw != 3 || s.nC == 0 || s.nP == 0 || s.nedges == 0) return false;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s.dev);
    const int64_t nc = (int64_t)s.nC;
    if (std::is_same<TS, float>::value) {
      // the ring kernel takes any camera count: shared accumulator when the
      // operator's and the right-hand side's fit next to the rings, else global
      const size_t need = std::max(
          std::max(RingSmem<float, FAST_APPLY, RACC_SHARED>::bytes(nc, false, ring_warps_shared<float>(),
                                                                   RING_SLOTS_SHARED),
                   RingSmem<double, FAST_APPLY, RACC_SHARED>::bytes(nc, false, ring_warps_shared<double>(),
                                                                    RING_SLOTS_SHARED)),
          RingSmem<double, FAST_RHS, RACC_SHARED>::bytes(nc, false, ring_warps_shared<double>(), RING_SLOTS_SHARED));
      global_acc = need > (size_t)optin;
    } else {
      size_t need = std::max(FastSmem<TS, double>::bytes(nc, false), FastSmem<TS, TS>::bytes(nc, false));
      if (need > (size_t)optin) return false;  // accumulator does not fit one SM's shared memory
    }
    if (!structure) {
      if (build(s) != FG_OK || !structure) return false;
      attr_set[0][0] = attr_set[0][1] = attr_set[1][0] = attr_set[1][1] = 0;
    }
    grid = sm_count(s.dev);
    if (global_acc) {
      const size_t gb = std::max((size_t)GACC_COPIES * s.nC * GACC_STRIDE * sizeof(float), s.nC * 9 * sizeof(double));
      if (d_gacc.size() < gb) {
        if (d_gacc.resize(gb) != FG_OK) return false;
        if (cudaMemsetAsync(d_gacc.get(), 0, gb, s.st) != cudaSuccess) return false;
      }
      return true;
    }
    if (d_parts_f.resize((size_t)grid * s.nC * 9) != FG_OK) return false;
    if (d_parts_d.resize((size_t)grid * s.nC * 9) != FG_OK) return false;
    return true;
  }

  // Whether operator variant v can run on this structure (the direct and
  // stage-group kernels need the shared accumulator and tiles of <= 32 edges).
  bool variant_ok(int v) const {
    if (!std::is_same<TS, float>::value) return true;
    return v == 1 || (!global_acc && !has_deep);
  }

  // The ring kernel in mode MODE on vectors TV; `reduce` as in apply.
  template <class TV, int MODE, class Impl>
  fg_status launch_ring(Impl& s, const TV* z, const TV* pv, const double* beta, TV* parts, const int* skip,
                        const int* gate, FastExtra ex) {
    if (!optin) cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s.dev);
    FastTiles tl{d_ebeg.get(), d_pbeg.get(), nwt, nstages};
    const int64_t nc = (int64_t)s.nC;
    const float* er = reinterpret_cast<const float*>(d_erec.get());
    const float* pr = reinterpret_cast<const float*>(d_prec.get());
    if (!global_acc) {
      constexpr int NW = ring_warps_shared<TV>(), R = RING_SLOTS_SHARED;
      const bool xs = RingSmem<TV, MODE, RACC_SHARED>::bytes(nc, true, NW, R) <= (size_t)optin;
      const size_t sm = RingSmem<TV, MODE, RACC_SHARED>::bytes(nc, xs, NW, R);
      auto kern = xs ? k_ring<TV, MODE, RACC_SHARED, true, NW, R> : k_ring<TV, MODE, RACC_SHARED, false, NW, R>;
      FG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      FG_LAUNCH_PDL(kern, grid, NW * 32, sm, s.st, nc, tl, er, pr, z, pv, beta, parts, (void*)nullptr, skip, gate,
                    d_error.get(), ex, poll_limit);
    } else {
      constexpr int NW = RING_WARPS_GLOBAL, R = RING_SLOTS_GLOBAL;
      const size_t sm = RingSmem<TV, MODE, RACC_GLOBAL>::bytes(nc, false, NW, R);
      auto kern = k_ring<TV, MODE, RACC_GLOBAL, false, NW, R>;
      FG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      FG_LAUNCH(kern, grid, NW * 32, sm, s.st, nc, tl, er, pr, z, pv, beta, (TV*)nullptr, (void*)d_gacc.get(), skip,
                gate, d_error.get(), ex, poll_limit);
    }
    return FG_OK;
  }

  // The reduction after a ring pass with the global accumulator.
  template <class TV, class Impl>
  fg_status launch_gacc_reduce(Impl& s, const TV* z, const TV* pv, const double* beta, double lambda,
                               const double* lam_dev, int use_gram, TV* out, double* dparts, PcgState* pst,
                               const int* gate, bool fp64) {
    const int64_t ny = (int64_t)s.nC * 9;
    FG_LAUNCH((k_gacc_reduce<TV>), grid_for(ny, 256), 256, 0, s.st, (int64_t)s.nC, (void*)d_gacc.get(), (int)fp64,
              reinterpret_cast<const float*>(s.d_gram.get()), s.d_observed.get(), z, pv, beta, lambda, lam_dev,
              use_gram, out, dparts, pst, gate);
    return FG_OK;
  }

  // The coarse Galerkin matrix W^T S(lambda) W in two passes (cameras, then
  // edges), nk <= 8 coarse vectors; out (device, nk x nk) is overwritten.
  DBuf<float> d_wc;
  // Only the 7-vector similarity gauge of BAL takes this path.
  template <class Impl>
  fg_status coarse_gram(Impl& s, double lambda, const double* wd, int nk, double* out) {
    if (nk != 7) return FG_UNSUPPORTED_STRUCTURE;
    constexpr int WS = 72;
    FG_TRY(d_wc.resize((size_t)s.nC * WS));
    FG_CUDA(cudaMemsetAsync(d_wc.get(), 0, (size_t)s.nC * WS * sizeof(float), s.st));
    FG_CUDA(cudaMemsetAsync(out, 0, (size_t)nk * nk * sizeof(double), s.st));
    FG_LAUNCH(k_coarse_cams<TS>, std::max(1u, std::min<unsigned>(grid_for(s.nC, 4), (unsigned)grid)), 256, 0, s.st,
              (int64_t)s.nC, wd, s.d_gram.get(), s.d_observed.get(), lambda, d_wc.get(), WS, out);
    FastTiles tl{d_ebeg.get(), d_pbeg.get(), nwt, nstages};
    // one resident wave (two CTAs per SM); the warps walk their tiles with the
    // next tile's loads in flight
    const unsigned blocks = (unsigned)std::min<int64_t>((nwt + COARSE_WARPS - 1) / COARSE_WARPS, 2 * (int64_t)grid);
    FG_LAUNCH(k_coarse_tiles<TS>, std::max(blocks, 1u), COARSE_WARPS * 32, 0, s.st, tl, (const TS*)d_erec.get(),
              (const TS*)d_prec.get(), (const float*)d_wc.get(), out);
    return FG_OK;
  }

  // After each block factorization: refresh C^-1 in the point records.
  template <class Impl>
  fg_status refresh_points(Impl& s, double lambda) {
    if (!on) return FG_OK;
    FG_LAUNCH(k_fast_point_records<TS>, grid_for(s.nP, 256), 256, 0, s.st, s.layout(), s.d_factors.get(),
              s.d_observed.get(), lambda, d_prec.get());
    return FG_OK;
  }

  // After passes launched without their reduction (timing): clear the global
  // accumulator they left behind.
  template <class Impl>
  fg_status settle(Impl& s) {
    if (global_acc && d_gacc.size()) FG_CUDA(cudaMemsetAsync(d_gacc.get(), 0, d_gacc.size(), s.st));
    return FG_OK;
  }

  // A bounded TMA wait that gave up leaves 1 in d_error.
  template <class Impl>
  fg_status check(Impl& s) {
    if (!on) return FG_OK;
    int h = 0;
    FG_CUDA(cudaMemcpyAsync(&h, d_error.get(), sizeof(int), cudaMemcpyDeviceToHost, s.st));
    FG_CUDA(cudaStreamSynchronize(s.st));
    if (h) {
      // reported once: the next solve starts with a clear flag
      FG_CUDA(cudaMemsetAsync(d_error.get(), 0, sizeof(int), s.st));
      set_error("reduced operator: a bounded shared-memory pipeline wait timed out");
      return FG_DEVICE_TIMEOUT;
    }
    return FG_OK;
  }

  // out = lambda x + B x - E C^-1 E^T x. pst != nullptr: PCG step (skips when
  // finished, computes alpha). gate != nullptr: runs only while *gate != 0.
  int optin = 0;
  size_t attr_set[2][2] = {{0, 0}, {0, 0}};  // [TV is double][stage x] -> smem size already granted

  int variant = 1;  // FP32 operator: 1 = TMA-staged stages, 2 = direct global loads, 3 = prefetching direct

  // reduce = false: the pass alone, leaving the per-CTA partial vectors (timing)
  template <class Impl, class TV>
  fg_status apply(Impl& s, PView<TV> x, double lambda, TV* out, double* dparts, PcgState* pst,
                  const int* gate = nullptr, const double* lam_dev = nullptr, bool reduce = true) {
    TV* parts = std::is_same<TV, float>::value ? (TV*)d_parts_f.get() : (TV*)d_parts_d.get();
    if constexpr (std::is_same<TS, float>::value) {
      if (variant == 1 || !variant_ok(variant)) {
        FG_TRY((launch_ring<TV, FAST_APPLY>(s, x.z, x.pprev, x.beta, parts, pst ? &pst->done : nullptr, gate,
                                            FastExtra{})));
        if (!reduce) return FG_OK;
        if (global_acc)
          return launch_gacc_reduce<TV>(s, x.z, x.pprev, x.beta, lambda, lam_dev, 1, out, dparts, pst, gate,
                                        !std::is_same<TV, float>::value);
        FG_LAUNCH_PDL((k_fast_reduce<TS, TV>), grid_for(s.nC * 9, 32), FR_ROWS * 32, 0, s.st, (int64_t)s.nC, grid,
                      (const TV*)parts, s.d_gram.get(), s.d_observed.get(), x.z, x.pprev, x.beta, lambda, lam_dev, 1,
                      out, dparts, pst, gate);
        return FG_OK;
      }
    }
    if (std::is_same<TS, float>::value && std::is_same<TV, float>::value && (variant == 2 || variant == 3)) {
      FG_TRY(apply_direct(s, (const float*)x.z, (const float*)x.pprev, x.beta, (float*)parts,
                          pst ? &pst->done : nullptr, gate, variant == 3));
      if (!reduce) return FG_OK;
      FG_LAUNCH((k_fast_reduce<TS, TV>), grid_for(s.nC * 9, 32), FR_ROWS * 32, 0, s.st, (int64_t)s.nC, grid,
                (const TV*)parts, s.d_gram.get(), s.d_observed.get(), x.z, x.pprev, x.beta, lambda, lam_dev, 1, out,
                dparts, pst, gate);
      return FG_OK;
    }
    if (!optin) cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s.dev);
    bool xs = FastSmem<TS, TV>::bytes((int64_t)s.nC, true) <= (size_t)optin;
    size_t sm = FastSmem<TS, TV>::bytes((int64_t)s.nC, xs);
    size_t& granted = attr_set[std::is_same<TV, double>::value ? 1 : 0][xs ? 1 : 0];
    FastTiles tl{d_ebeg.get(), d_pbeg.get(), nwt, nstages};
    const int* skip = pst ? &pst->done : nullptr;
    constexpr int NTHR = FAST_GROUPS * FastShape<TS>::WPS * 32;
    if (xs) {
      auto kern = k_fast_apply<TS, TV, true>;
      if (granted < sm) {
        FG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        granted = sm;
      }
      FG_LAUNCH(kern, grid, NTHR, sm, s.st, (int64_t)s.nC, tl, d_erec.get(), d_prec.get(), x.z, x.pprev, x.beta,
                parts, skip, gate, d_error.get(), FastExtra{});
    } else {
      auto kern = k_fast_apply<TS, TV, false>;
      if (granted < sm) {
        FG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        granted = sm;
      }
      FG_LAUNCH(kern, grid, NTHR, sm, s.st, (int64_t)s.nC, tl, d_erec.get(), d_prec.get(), x.z, x.pprev, x.beta,
                parts, skip, gate, d_error.get(), FastExtra{});
    }
    if (!reduce) return FG_OK;
    FG_LAUNCH((k_fast_reduce<TS, TV>), grid_for(s.nC * 9, 32), FR_ROWS * 32, 0, s.st, (int64_t)s.nC, grid,
              (const TV*)parts, s.d_gram.get(), s.d_observed.get(), x.z, x.pprev, x.beta, lambda, lam_dev, 1, out,
              dparts, pst, gate);
    return FG_OK;
  }

  size_t direct_granted = 0, pf_granted = 0;
  template <class Impl>
  fg_status apply_direct(Impl& s, const float* z, const float* pv, const double* beta, float* parts, const int* skip,
                         const int* gate, bool prefetch) {
    if (!optin) cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s.dev);
    size_t vb = FastSmem<float, float>::vec_bytes((int64_t)s.nC);
    size_t tpw = (size_t)((prefetch ? PF_THREADS : DIRECT_THREADS) / 32) * 96 * sizeof(float);
    bool xs = 2 * vb + tpw <= (size_t)optin;
    size_t sm = vb * (xs ? 2 : 1) + tpw;
    FastTiles tl{d_ebeg.get(), d_pbeg.get(), nwt, nstages};
    if (prefetch) {
      auto kern = xs ? k_fast_apply_pf<true> : k_fast_apply_pf<false>;
      if (pf_granted < sm) {
        FG_CUDA(cudaFuncSetAttribute(k_fast_apply_pf<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        FG_CUDA(cudaFuncSetAttribute(k_fast_apply_pf<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        pf_granted = sm;
      }
      FG_LAUNCH(kern, grid, PF_THREADS, sm, s.st, (int64_t)s.nC, tl, (const float*)d_erec.get(),
                (const float*)d_prec.get(), z, pv, beta, parts, skip, gate);
      return FG_OK;
    }
    if (xs) {
      if (direct_granted < sm) {
        FG_CUDA(cudaFuncSetAttribute(k_fast_apply_direct<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        direct_granted = sm;
      }
      FG_LAUNCH(k_fast_apply_direct<true>, grid, DIRECT_THREADS, sm, s.st, (int64_t)s.nC, tl,
                (const float*)d_erec.get(), (const float*)d_prec.get(), z, pv, beta, parts, skip, gate);
    } else {
      if (direct_granted < sm) {
        FG_CUDA(cudaFuncSetAttribute(k_fast_apply_direct<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        direct_granted = sm;
      }
      FG_LAUNCH(k_fast_apply_direct<false>, grid, DIRECT_THREADS, sm, s.st, (int64_t)s.nC, tl,
                (const float*)d_erec.get(), (const float*)d_prec.get(), z, pv, beta, parts, skip, gate);
    }
    return FG_OK;
  }

  // rhs_c = w_c - sum_{e in c} E_e w_p (src/schur.rs:216-242) from the edge
  // records; w is the scaled-gradient work vector with C^-1 already applied
  // to its eliminated part.
  template <class Impl>
  fg_status rhs(Impl& s, const double* w, double* rhs_out) {
    if constexpr (std::is_same<TS, float>::value) {
      FG_TRY((launch_ring<double, FAST_RHS>(s, w, (const double*)nullptr, (const double*)nullptr, d_parts_d.get(),
                                            (const int*)nullptr, (const int*)nullptr,
                                            FastExtra{w + s.retained, nullptr, nullptr})));
      if (global_acc)
        return launch_gacc_reduce<double>(s, w, (const double*)nullptr, (const double*)nullptr, 1.0,
                                          (const double*)nullptr, 0, rhs_out, (double*)nullptr, (PcgState*)nullptr,
                                          (const int*)nullptr, true);
      FG_LAUNCH((k_fast_reduce<TS, double>), grid_for(s.nC * 9, 32), FR_ROWS * 32, 0, s.st, (int64_t)s.nC, grid,
                (const double*)d_parts_d.get(), s.d_gram.get(), s.d_observed.get(), w, (const double*)nullptr,
                (const double*)nullptr, 1.0, (const double*)nullptr, 0, rhs_out, (double*)nullptr, (PcgState*)nullptr,
                (const int*)nullptr);
      return FG_OK;
    }
    if (!optin) cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s.dev);
    size_t sm = FastSmem<TS, double>::bytes((int64_t)s.nC, false);
    auto kern = k_fast_apply<TS, double, false, FAST_RHS>;
    FG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    FastTiles tl{d_ebeg.get(), d_pbeg.get(), nwt, nstages};
    FastExtra ex{w + s.retained, nullptr, nullptr};
    FG_LAUNCH(kern, grid, FAST_GROUPS * FastShape<TS>::WPS * 32, sm, s.st, (int64_t)s.nC, tl, d_erec.get(),
              d_prec.get(), w, (const double*)nullptr, (const double*)nullptr, d_parts_d.get(), (const int*)nullptr,
              (const int*)nullptr, d_error.get(), ex);
    FG_LAUNCH((k_fast_reduce<TS, double>), grid_for(s.nC * 9, 32), FR_ROWS * 32, 0, s.st, (int64_t)s.nC, grid,
              (const double*)d_parts_d.get(), s.d_gram.get(), s.d_observed.get(), w, (const double*)nullptr,
              (const double*)nullptr, 1.0, (const double*)nullptr, 0, rhs_out, (double*)nullptr, (PcgState*)nullptr,
              (const int*)nullptr);
    return FG_OK;
  }

  // step_p = C^-1 (-g_p/D_p - sum_{e in p} E_e^T z_c) / D_p for every point
  // with observations (src/schur.rs:312-344); g is the gradient.
  template <class Impl>
  fg_status recover(Impl& s, const double* zred, const double* g, const double* scales, double* step) {
    if constexpr (std::is_same<TS, float>::value) {
      return launch_ring<double, FAST_RECOVER>(s, zred, (const double*)nullptr, (const double*)nullptr,
                                               (double*)nullptr, (const int*)nullptr, (const int*)nullptr,
                                               FastExtra{g + s.retained, scales + s.retained, step + s.retained});
    }
    if (!optin) cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s.dev);
    // x staged in the space the other modes give their accumulator
    size_t sm = FastSmem<TS, double>::bytes((int64_t)s.nC, false);
    auto kern = k_fast_apply<TS, double, true, FAST_RECOVER>;
    FG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    FastTiles tl{d_ebeg.get(), d_pbeg.get(), nwt, nstages};
    FastExtra ex{g + s.retained, scales + s.retained, step + s.retained};
    FG_LAUNCH(kern, grid, FAST_GROUPS * FastShape<TS>::WPS * 32, sm, s.st, (int64_t)s.nC, tl, d_erec.get(),
              d_prec.get(), zred, (const double*)nullptr, (const double*)nullptr, d_parts_d.get(), (const int*)nullptr,
              (const int*)nullptr, d_error.get(), ex);
    return FG_OK;
  }
};

}  // namespace fg
