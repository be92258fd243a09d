// Per-warp TMA rings for the single-pass BAL reduced operator (FP32 edge
// records). Every warp streams its own warp tiles (tile first + k G) through
// a private ring of R shared-memory slots, so no barrier couples the warps of
// a CTA inside the main loop and a slow tile stalls only its own warp.
//
// A slot holds one warp tile: its edge records (<= 32 x 112 bytes) and the
// point records of the tile's points (<= 32 x 32 bytes), both fetched by
// lane 0 with 1-D bulk copies (cp.async.bulk) onto the slot's mbarrier, so
// neither the cross blocks nor C^-1 is a dependent global load of the
// consumer. Two things keep enough bytes in flight with few slots:
//  * a slot is handed to the next tile as soon as its lanes hold the tile's
//    records and C^-1 in registers, before the tile's arithmetic, so the
//    copy of tile k + R overlaps the work on tile k;
//  * the bounds of the warp's tiles are loaded 32 tiles at a time (lane l
//    holds tile 32 c + l) one batch ahead, so no refill waits on a global
//    load of its bounds.
//
// Camera accumulation, chosen by the number of cameras:
//  * shared (RACC_SHARED): the CTA-private 9C accumulator of k_fast_apply
//    (64-bit fixed point in two 32-bit words for the operator, FP64 for the
//    right-hand side), flushed to one partial row per CTA;
//  * global (RACC_GLOBAL, when 9C does not fit one SM): vector reductions
//    red.global.add.v4.f32 into GACC_COPIES copies of a camera-padded
//    accumulator (12 floats per camera), the copy chosen by CTA, summed in
//    FP64 by the reduction kernel, which also clears them; FP64 vectors use
//    red.global.add.f64 into one copy of 9 doubles per camera.
//
// A point with more than 32 observations is a tile of its own ("deep"); its
// records are read from global memory in chunks of 32 by the warp, which
// reduces the point's sum across the chunks.
//
// Included by fastpath.cuh after the shared helpers (PTX wrappers, record
// loaders, FastTiles, FastExtra) and before FastPath, which launches it.
#pragma once

namespace fg {

constexpr int RING_EDGE_BYTES = 32 * 28 * 4;                 // edge records of one warp tile
constexpr int RING_SLOT_BYTES = RING_EDGE_BYTES + 32 * 8 * 4;  // + its point records
// Shared accumulator: one slot per warp; 20 warps for FP32 vectors (96
// registers a thread), 16 for FP64 vectors, which need more registers.
template <class TV>
constexpr int ring_warps_shared() {
  return std::is_same<TV, float>::value ? 20 : 16;
}
constexpr int RING_SLOTS_SHARED = 1;
constexpr int RING_WARPS_GLOBAL = 16;  // with two slots per warp (global accumulator)
constexpr int RING_SLOTS_GLOBAL = 2;
constexpr int GACC_COPIES = 8;   // FP32 global accumulator copies
constexpr int GACC_STRIDE = 12;  // floats per camera in an FP32 copy (three 16-byte vectors)
constexpr unsigned RING_POLL_LIMIT = 1u << 22;
enum RingAcc { RACC_SHARED = 0, RACC_GLOBAL = 1 };

template <class TV, int MODE, int ACC>
struct RingSmem {
  // FP32 records: the operator (FAST_APPLY) accumulates 64-bit fixed point
  static constexpr bool FIXED = MODE == FAST_APPLY && ACC == RACC_SHARED;
  static constexpr int FIXED_BITS = std::is_same<TV, float>::value ? 40 : 44;
  __host__ __device__ static size_t acc_bytes(int64_t ncam) {
    if (ACC != RACC_SHARED || MODE == FAST_RECOVER) return 0;
    if (FIXED) return 2 * FastSmem<float, float>::word_bytes(ncam);
    return FastSmem<float, double>::vec_bytes(ncam);  // FAST_RHS: FP64
  }
  __host__ __device__ static size_t xs_bytes(int64_t ncam, bool xs) {
    return xs && MODE != FAST_RHS ? FastSmem<float, TV>::vec_bytes(ncam) : 0;
  }
  __host__ __device__ static size_t bytes(int64_t ncam, bool xs, int nw, int slots) {
    const size_t bars = ((size_t)nw * slots * 8 + 127) & ~(size_t)127;
    return acc_bytes(ncam) + xs_bytes(ncam, xs) + bars + (size_t)nw * slots * RING_SLOT_BYTES;
  }
};

// All lanes poll; the result is uniform across the warp. The first poll does
// not block (test_wait), the later ones may suspend for a while (try_wait), so
// a limit of one poll gives up at once unless the copies have landed.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, unsigned parity, unsigned limit) {
  for (unsigned i = 0; i < limit; ++i) {
    const bool ok = i == 0 ? mbar_test_wait(bar, parity) : mbar_try_wait(bar, parity);
    if (__all_sync(0xffffffffu, ok)) return true;
    if (i > 64) __nanosleep(64);
  }
  return false;
}

// One tile's bounds.
struct RingTile {
  int64_t e0, p0;
  int cnt, np;
};
// Bounds of the warp's tiles kb + lane (tile index first + (kb + lane) G),
// zero past the warp's last tile.
__device__ __forceinline__ RingTile ring_batch(const FastTiles& t, int64_t first, int64_t G, int64_t nmine, int64_t kb,
                                               int lane) {
  RingTile r{0, 0, 0, 0};
  if (kb + lane < nmine) {
    const int64_t wt = first + (kb + lane) * G;
    r.e0 = t.wt_e0[wt];
    r.cnt = (int)(t.wt_e0[wt + 1] - r.e0);
    r.p0 = t.wt_p0[wt];
    r.np = (int)(t.wt_p0[wt + 1] - r.p0);
  }
  return r;
}
// The bounds lane l holds in batch a (cur) or b, for every lane.
__device__ __forceinline__ RingTile ring_pick(const RingTile& a, const RingTile& b, bool cur, int l) {
  RingTile o;
  o.e0 = __shfl_sync(0xffffffffu, cur ? a.e0 : b.e0, l);
  o.p0 = __shfl_sync(0xffffffffu, cur ? a.p0 : b.p0, l);
  o.cnt = __shfl_sync(0xffffffffu, cur ? a.cnt : b.cnt, l);
  o.np = __shfl_sync(0xffffffffu, cur ? a.np : b.np, l);
  return o;
}

// The camera scatter of one edge's y -= E t (9 values) into the accumulator.
template <class TV, int MODE, int ACC>
struct RingScatter {
  uint32_t* ylo;
  uint32_t* yhi;
  double* yd;   // shared FP64 (RHS) or global FP64 copy
  float* gf;    // global FP32 copy of this CTA
  double fx_mul;
  float fx_mulf;  // fx_mul in FP32 when it is a normal FP32 number, else 0
  __device__ __forceinline__ void add(uint32_t cam, const TV (&v)[9]) const {
    if (ACC == RACC_SHARED) {
      if (RingSmem<TV, MODE, ACC>::FIXED) {
        fixed_scatter(ylo, yhi, (int64_t)cam * 9, v, fx_mul, fx_mulf);
      } else {
        double* y = yd + (int64_t)cam * 9;
#pragma unroll
        for (int c = 0; c < 9; ++c) atomicAdd(&y[c], (double)v[c]);
      }
    } else if (std::is_same<TV, float>::value && MODE == FAST_APPLY) {
      float* p = gf + (int64_t)cam * GACC_STRIDE;
      asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"((float)v[0]), "f"((float)v[1]),
                   "f"((float)v[2]), "f"((float)v[3])
                   : "memory");
      asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p + 4), "f"((float)v[4]), "f"((float)v[5]),
                   "f"((float)v[6]), "f"((float)v[7])
                   : "memory");
      asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p + 8), "f"((float)v[8]) : "memory");
    } else {
      double* y = yd + (int64_t)cam * 9;
#pragma unroll
      for (int c = 0; c < 9; ++c) atomicAdd(&y[c], (double)v[c]);
    }
  }
};

// x for camera coordinates: staged copy, or z + beta p from global memory.
template <class TV, bool XS>
__device__ __forceinline__ void ring_x(uint32_t cam, const TV* xs, const TV* z, const TV* pv, TV bv, TV (&xc)[9]) {
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const int64_t i = (int64_t)cam * 9 + c;
    xc[c] = XS ? xs[i] : (pv ? __ldg(z + i) + bv * __ldg(pv + i) : __ldg(z + i));
  }
}

template <class TV, int MODE, int ACC, bool XS, int NW, int R>
__global__ void __launch_bounds__(NW * 32, 1)
    k_ring(int64_t ncam, FastTiles tiles, const float* erec, const float* prec, const TV* z, const TV* pv,
           const double* beta, TV* partials, void* gacc, const int* skip, const int* gate, int* error,
           FastExtra ex, unsigned poll_limit) {
  using SM = RingSmem<TV, MODE, ACC>;
  constexpr bool FIXED = SM::FIXED;
  constexpr bool NEED_X = MODE != FAST_RHS;
  constexpr bool SCATTER = MODE != FAST_RECOVER;
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  constexpr int NTHR = NW * 32;
  const int64_t ny = ncam * 9;
  const size_t acc = SM::acc_bytes(ncam);
  const size_t xsb = SM::xs_bytes(ncam, XS);
  uint32_t* ylo = reinterpret_cast<uint32_t*>(smem);
  uint32_t* yhi = reinterpret_cast<uint32_t*>(smem + FastSmem<float, float>::word_bytes(ncam));
  double* yds = reinterpret_cast<double*>(smem);
  TV* xs = reinterpret_cast<TV*>(smem + acc);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + acc + xsb);
  unsigned char* ring = smem + acc + xsb + (((size_t)NW * R * 8 + 127) & ~(size_t)127) + (size_t)w * R * RING_SLOT_BYTES;
  uint64_t* wbar = bars + w * R;

  // this CTA's own shared memory (the accumulator and the slot barriers) is
  // set up before the dependency wait, overlapping the previous kernel's tail;
  // every global access comes after it
  if (ACC == RACC_SHARED && SCATTER) {
    for (int64_t i = tid; i < ny; i += NTHR) {
      if (FIXED) {
        ylo[i] = 0;
        yhi[i] = 0;
      } else {
        yds[i] = 0;
      }
    }
  }
  if (lane == 0) {
    for (int b = 0; b < R; ++b) mbar_init(&wbar[b], 1);
    mbar_fence_init();
  }
  pdl_wait();
  pdl_trigger();
  if (skip && *skip) return;
  if (gate && !*gate) return;
  const TV bv = pv ? (TV)*beta : (TV)0;
  double xmax = 0.0;
  if (NEED_X && (XS || FIXED)) {
    for (int64_t i = tid; i < ny; i += NTHR) {
      const TV xi = pv ? z[i] + bv * pv[i] : z[i];
      if (XS) xs[i] = xi;
      if (FIXED) xmax = isfinite((double)xi) ? fmax(xmax, fabs((double)xi)) : (double)INFINITY;
    }
  }
  __shared__ double wmax[32];
  __shared__ double fx_mul_s, fx_unit_s;
  if (FIXED) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
    if (lane == 0) wmax[w] = xmax;
  }
  __syncthreads();
  if (FIXED && tid == 0) {
    double m = 0.0;
    for (int k = 0; k < NW; ++k) m = fmax(m, wmax[k]);
    // unit 2^-k with |x| < 2^(B-k): a contribution (at most a few hundred
    // |x|max, the per-point Gram bound E_p C_p^-1 E_p^T <= B_p) stays below
    // 2^(B+9) units and a CTA's partial sums far below 2^63
    int e = 0;
    if (m > 0.0 && isfinite(m)) frexp(m, &e);
    fx_mul_s = isfinite(m) ? ldexp(1.0, SM::FIXED_BITS - e) : 0.0;
    fx_unit_s = isfinite(m) ? ldexp(1.0, e - SM::FIXED_BITS) : (double)NAN;
  }
  if (FIXED) __syncthreads();

  RingScatter<TV, MODE, ACC> sc;
  sc.ylo = ylo;
  sc.yhi = yhi;
  sc.fx_mul = FIXED ? fx_mul_s : 0.0;
  sc.fx_mulf = FIXED ? fixed_mulf(fx_mul_s) : 0.f;
  sc.gf = ACC == RACC_GLOBAL ? reinterpret_cast<float*>(gacc) + (int64_t)(blockIdx.x % GACC_COPIES) * ncam * GACC_STRIDE
                             : nullptr;
  sc.yd = ACC == RACC_SHARED ? yds : reinterpret_cast<double*>(gacc);

  const int64_t G = (int64_t)gridDim.x * NW;
  const int64_t first = (int64_t)blockIdx.x * NW + w;
  const int64_t nmine = first < tiles.nwt ? (tiles.nwt - 1 - first) / G + 1 : 0;  // this warp's tiles
  // Lane l holds the bounds of this warp's tile 32 c + l for the current batch
  // c (ba) and the next (bb): one coalesced round of loads per 32 tiles, off
  // the critical path of the refills.
  RingTile ba = ring_batch(tiles, first, G, nmine, 0, lane), bb = ring_batch(tiles, first, G, nmine, 32, lane);
  int64_t cbatch = 0;
  auto bounds = [&](int64_t kk) { return ring_pick(ba, bb, (kk >> 5) == cbatch, (int)(kk & 31)); };
  // lane 0 issues the copies of a tile into slot b (a deep tile needs none:
  // an arrival without transaction bytes completes the slot's phase)
  auto issue = [&](const RingTile& t, int b) {
    if (lane != 0) return;
    const bool shallow = t.cnt <= 32;
    const unsigned eb = shallow ? (unsigned)t.cnt * 112u : 0u;
    const unsigned pb = shallow && MODE != FAST_RHS ? (unsigned)t.np * 32u : 0u;
    unsigned char* dst = ring + (size_t)b * RING_SLOT_BYTES;
    mbar_expect_tx(&wbar[b], eb + pb);
    if (eb) tma_load_1d(dst, erec + t.e0 * 28, eb, &wbar[b]);
    if (pb) tma_load_1d(dst + RING_EDGE_BYTES, prec + t.p0 * 8, pb, &wbar[b]);
  };
  // the slot's data is in registers: hand the slot to the tile R ahead
  auto refill = [&](int64_t k, int b) {
    __syncwarp();
    if (k + R < nmine) {
      const RingTile n = bounds(k + R);
      if (lane == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(n, b);
    }
  };
#pragma unroll
  for (int b = 0; b < R; ++b)
    if (b < nmine) issue(bounds(b), b);
  bool failed = false;
  int64_t k = 0;
  for (; k < nmine; ++k) {
    const int b = (int)(k % R);
    const unsigned parity = (unsigned)((k / R) & 1);
    const RingTile t = bounds(k);
    if (!warp_wait(&wbar[b], parity, poll_limit)) {
      failed = true;
      break;
    }
    const unsigned char* slot = ring + (size_t)b * RING_SLOT_BYTES;
    if (t.cnt <= 32) {
      // ---------------------------------------------------- shallow tile
      TV E[27];
      uint32_t cam = 0, lp = 0xFFFFu;
      TV c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0;  // the lane's point C^-1 (packed lower)
      if (lane < t.cnt) {
        load_record<TV>(reinterpret_cast<const float*>(slot) + lane * 28, E, cam, lp);
        if (MODE != FAST_RHS) {
          const float4* pr = reinterpret_cast<const float4*>(slot + RING_EDGE_BYTES + (size_t)lp * 32);
          const float4 ca = pr[0], cb = pr[1];
          c0 = ca.x; c1 = ca.y; c2 = ca.z; c3 = ca.w; c4 = cb.x; c5 = cb.y;
        }
      }
      refill(k, b);
      TV u0 = 0, u1 = 0, u2 = 0;
      if (NEED_X && lane < t.cnt) {
        TV xc[9];
        ring_x<TV, XS>(cam, xs, z, pv, bv, xc);
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          u0 += E[c] * xc[c];
          u1 += E[9 + c] * xc[c];
          u2 += E[18 + c] * xc[c];
        }
      }
      // inactive lanes get keys of their own so they never extend a run
      if (NEED_X) seg_scan3<TV>(u0, u1, u2, lane < t.cnt ? lp : 0x10000u + lane, lane);
      const uint32_t lpn = __shfl_down_sync(0xffffffffu, lp, 1);
      const bool last = lane < t.cnt && (lane == t.cnt - 1 || lpn != lp);
      TV t0 = 0, t1 = 0, t2 = 0;
      if (last) {
        if (MODE == FAST_RHS) {
          const double* w3 = ex.wp + 3 * (t.p0 + lp);
          t0 = (TV)w3[0];
          t1 = (TV)w3[1];
          t2 = (TV)w3[2];
        } else if (MODE == FAST_RECOVER) {
          const int64_t q = 3 * (t.p0 + lp);
          const TV a0 = (TV)(-ex.wp[q] / ex.scales[q]) - u0, a1 = (TV)(-ex.wp[q + 1] / ex.scales[q + 1]) - u1;
          const TV a2 = (TV)(-ex.wp[q + 2] / ex.scales[q + 2]) - u2;
          ex.step[q] = (double)(c0 * a0 + c1 * a1 + c2 * a2) / ex.scales[q];
          ex.step[q + 1] = (double)(c1 * a0 + c3 * a1 + c4 * a2) / ex.scales[q + 1];
          ex.step[q + 2] = (double)(c2 * a0 + c4 * a1 + c5 * a2) / ex.scales[q + 2];
        } else {
          t0 = c0 * u0 + c1 * u1 + c2 * u2;
          t1 = c1 * u0 + c3 * u1 + c4 * u2;
          t2 = c2 * u0 + c4 * u1 + c5 * u2;
        }
      }
      if (SCATTER) {
        // each lane takes its point's t from the point's last lane
        const unsigned ends = __ballot_sync(0xffffffffu, last) & ~((1u << lane) - 1u);
        const int src = ends ? __ffs(ends) - 1 : lane;
        t0 = __shfl_sync(0xffffffffu, t0, src);
        t1 = __shfl_sync(0xffffffffu, t1, src);
        t2 = __shfl_sync(0xffffffffu, t2, src);
        if (lane < t.cnt) {
          TV v[9];
#pragma unroll
          for (int c = 0; c < 9; ++c) v[c] = -(E[c] * t0 + E[9 + c] * t1 + E[18 + c] * t2);
          sc.add(cam, v);
        }
      }
    } else {
      // ---------------------------------------------------- deep tile: one point
      refill(k, b);  // its slot carries no data
      TV u0 = 0, u1 = 0, u2 = 0;
      if (NEED_X) {
        for (int c0 = 0; c0 < t.cnt; c0 += 32) {
          if (c0 + lane < t.cnt) {
            float Ef[27];
            uint32_t cam, lp;
            load_cross_global<float>(erec + (t.e0 + c0 + lane) * 28, Ef, cam, lp);
            TV E[27];
#pragma unroll
            for (int i = 0; i < 27; ++i) E[i] = (TV)Ef[i];
            TV xc[9];
            ring_x<TV, XS>(cam, xs, z, pv, bv, xc);
#pragma unroll
            for (int c = 0; c < 9; ++c) {
              u0 += E[c] * xc[c];
              u1 += E[9 + c] * xc[c];
              u2 += E[18 + c] * xc[c];
            }
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          u0 += __shfl_xor_sync(0xffffffffu, u0, o);
          u1 += __shfl_xor_sync(0xffffffffu, u1, o);
          u2 += __shfl_xor_sync(0xffffffffu, u2, o);
        }
      }
      TV t0 = 0, t1 = 0, t2 = 0;
      if (MODE == FAST_RHS) {
        const double* w3 = ex.wp + 3 * t.p0;
        t0 = (TV)w3[0];
        t1 = (TV)w3[1];
        t2 = (TV)w3[2];
      } else {
        const float* pr = prec + t.p0 * 8;
        const TV c0 = pr[0], c1 = pr[1], c2 = pr[2], c3 = pr[3], c4 = pr[4], c5 = pr[5];
        if (MODE == FAST_RECOVER) {
          if (lane == 0) {
            const int64_t q = 3 * t.p0;
            const TV a0 = (TV)(-ex.wp[q] / ex.scales[q]) - u0, a1 = (TV)(-ex.wp[q + 1] / ex.scales[q + 1]) - u1;
            const TV a2 = (TV)(-ex.wp[q + 2] / ex.scales[q + 2]) - u2;
            ex.step[q] = (double)(c0 * a0 + c1 * a1 + c2 * a2) / ex.scales[q];
            ex.step[q + 1] = (double)(c1 * a0 + c3 * a1 + c4 * a2) / ex.scales[q + 1];
            ex.step[q + 2] = (double)(c2 * a0 + c4 * a1 + c5 * a2) / ex.scales[q + 2];
          }
        } else {
          t0 = c0 * u0 + c1 * u1 + c2 * u2;
          t1 = c1 * u0 + c3 * u1 + c4 * u2;
          t2 = c2 * u0 + c4 * u1 + c5 * u2;
        }
      }
      if (SCATTER) {
        for (int c0 = 0; c0 < t.cnt; c0 += 32) {
          if (c0 + lane < t.cnt) {
            float Ef[27];
            uint32_t cam, lp;
            load_cross_global<float>(erec + (t.e0 + c0 + lane) * 28, Ef, cam, lp);
            TV v[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) v[c] = -((TV)Ef[c] * t0 + (TV)Ef[9 + c] * t1 + (TV)Ef[18 + c] * t2);
            sc.add(cam, v);
          }
        }
      }
    }
    if (((k + 1) & 31) == 0) {  // batch used up: the next becomes current, load the one after
      ba = bb;
      ++cbatch;
      bb = ring_batch(tiles, first, G, nmine, 32 * (cbatch + 1), lane);
    }
  }
  if (failed) {
    // drain: wait (bounded) for every copy this warp still has in flight
    // (tiles k .. k+R-1: the slot refill happens only after a successful wait)
    if (lane == 0) atomicExch(error, 1);
    for (int j = 0; j < R; ++j) {
      const int64_t kj = k + j;
      if (kj < nmine) warp_wait(&wbar[kj % R], (unsigned)((kj / R) & 1), RING_POLL_LIMIT);
    }
  }
  if (ACC != RACC_SHARED || !SCATTER) return;
  __syncthreads();
  TV* out = partials + (int64_t)blockIdx.x * ny;
  if (FIXED) {
    const double unit = fx_unit_s;
    for (int64_t i = tid; i < ny; i += NTHR) {
      const long long q = (long long)(((unsigned long long)yhi[i] << 32) | (unsigned long long)ylo[i]);
      out[i] = (TV)((double)q * unit);
    }
  } else {
    for (int64_t i = tid; i < ny; i += NTHR) out[i] = (TV)yds[i];
  }
}

// q = lambda x + B x + the global accumulator (summed over its copies in FP64,
// then cleared for the next application); optional p.q -> alpha as
// k_fast_reduce. FP32 copies: GACC_COPIES x ncam x GACC_STRIDE floats; FP64:
// one copy of ncam x 9 doubles.
template <class TV>
__global__ void __launch_bounds__(256) k_gacc_reduce(int64_t ncam, void* gacc, int fp64, const float* gram,
                                                      const uint8_t* observed, const TV* z, const TV* pv,
                                                      const double* beta, double lambda, const double* lam_dev,
                                                      int use_gram, TV* q, double* dparts, PcgState* st,
                                                      const int* gate) {
  if (st && st->done) return;
  if (gate && !*gate) return;
  const int64_t ny = ncam * 9;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double dot = 0;
  if (i < ny) {
    const int64_t cam = i / 9;
    const int r = (int)(i % 9);
    double sum = 0;
    if (fp64) {
      double* g = reinterpret_cast<double*>(gacc);
      sum = g[i];
      g[i] = 0;
    } else {
      float* g = reinterpret_cast<float*>(gacc);
#pragma unroll
      for (int k = 0; k < GACC_COPIES; ++k) {
        float* p = g + ((int64_t)k * ncam + cam) * GACC_STRIDE + r;
        sum += (double)*p;
        *p = 0.f;
      }
    }
    const TV bv = pv ? (TV)*beta : (TV)0;
    const TV xi = pv ? z[i] + bv * pv[i] : z[i];
    const double lam = lam_dev ? *lam_dev : lambda;
    TV v = (TV)lam * xi;
    if (use_gram && observed[cam]) {
      const float* gb = gram + cam * 81;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        const int64_t kk = cam * 9 + j;
        const TV xj = pv ? z[kk] + bv * pv[kk] : z[kk];
        const float gv = j >= r ? gb[r * 9 + j] : gb[j * 9 + r];
        v += (TV)gv * xj;
      }
    }
    v += (TV)sum;
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

}  // namespace fg
