// Stable device ordering by bounded keys (LSD radix sort) and key offsets.
#include "sort.cuh"

namespace fg {

namespace {
constexpr int RS_THREADS = 256;             // 8 warps
constexpr int RS_WARP_ITEMS = 256;          // consecutive keys per warp, 8 rounds of 32
constexpr int RS_TILE = 8 * RS_WARP_ITEMS;  // 2,048 keys per tile

// counts[d * ntiles + tile] = keys of the tile with digit d.
__global__ void __launch_bounds__(RS_THREADS) k_radix_count(const uint32_t* keys, int64_t n, int shift, int nbits,
                                                            int64_t ntiles, uint32_t* counts) {
  __shared__ uint32_t h[256];
  const int nd = 1 << nbits;
  const uint32_t mask = (uint32_t)nd - 1;
  for (int d = threadIdx.x; d < nd; d += RS_THREADS) h[d] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * RS_TILE;
  for (int j = threadIdx.x; j < RS_TILE; j += RS_THREADS) {
    const int64_t i = base + j;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & mask], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < nd; d += RS_THREADS) counts[(int64_t)d * ntiles + blockIdx.x] = h[d];
}

// Stable scatter of one digit pass. Keys of a tile are visited in index order
// (warp w owns items [256w, 256w + 256), in rounds of 32 lanes); the rank of a
// key among equal digits is: earlier warps (prefix of per-warp digit counts),
// earlier rounds of its warp (running count), earlier lanes of its round
// (match mask below the lane).
__global__ void __launch_bounds__(RS_THREADS) k_radix_scatter(const uint32_t* kin, const uint32_t* vin, int64_t n,
                                                              int shift, int nbits, int64_t ntiles,
                                                              const uint32_t* offs, uint32_t* kout, uint32_t* vout) {
  __shared__ uint32_t wcnt[8][256];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t mask = (1u << nbits) - 1;
  for (int d = lane; d < 256; d += 32) wcnt[w][d] = 0;
  __syncwarp();
  const unsigned below = (1u << lane) - 1u;
  const int64_t base = (int64_t)blockIdx.x * RS_TILE + (int64_t)w * RS_WARP_ITEMS;
  uint32_t key[8], val[8], loc[8], dig[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t i = base + r * 32 + lane;
    const bool valid = i < n;
    key[r] = valid ? kin[i] : 0u;
    val[r] = valid ? (vin ? vin[i] : (uint32_t)i) : 0u;
    const uint32_t d = valid ? (key[r] >> shift) & mask : 0xFFFFFFFFu;  // padding lanes match only each other
    dig[r] = d;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
    const unsigned rank = __popc(peers & below);
    const uint32_t old = valid ? wcnt[w][d] : 0u;
    __syncwarp();
    if (valid && rank == 0) wcnt[w][d] = old + (uint32_t)__popc(peers);
    __syncwarp();
    loc[r] = old + rank;
  }
  __syncthreads();
  {  // per digit: exclusive prefix over the warps of the tile
    const int d = threadIdx.x;
    uint32_t s = 0;
#pragma unroll
    for (int ww = 0; ww < 8; ++ww) {
      const uint32_t c = wcnt[ww][d];
      wcnt[ww][d] = s;
      s += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    if (base + r * 32 + lane >= n) break;
    const uint32_t d = dig[r];
    const int64_t pos = (int64_t)offs[(int64_t)d * ntiles + blockIdx.x] + wcnt[w][d] + loc[r];
    kout[pos] = key[r];
    vout[pos] = val[r];
  }
}

__global__ void k_iota_copy(int64_t n, const uint32_t* keys, uint32_t* order, uint32_t* sorted) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  order[i] = (uint32_t)i;
  if (sorted) sorted[i] = keys[i];
}

// Thread i in [0, n] writes the offsets of the keys in (sorted[i-1], sorted[i]].
__global__ void k_key_offsets(const uint32_t* sorted, int64_t n, uint32_t bound, int64_t* off) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i > n) return;
  const int64_t prev = i == 0 ? -1 : (int64_t)min(sorted[i - 1], bound);
  const int64_t cur = i == n ? (int64_t)bound : (int64_t)min(sorted[i], bound);
  for (int64_t k = prev + 1; k <= cur; ++k) off[k] = i;
}
}  // namespace

__global__ void __launch_bounds__(1024) k_scan_exclusive_u32(uint32_t* a, int64_t m, uint32_t* total) {
  __shared__ uint32_t warp_sums[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int64_t chunk = (m + 1023) / 1024, lo = min((int64_t)t * chunk, m), hi = min(lo + chunk, m);
  uint32_t s = 0;
#pragma unroll 8
  for (int64_t i = lo; i < hi; ++i) s += a[i];
  uint32_t incl = s;  // inclusive scan of the chunk sums across the block
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
    if (lane >= off) incl += v;
  }
  if (lane == 31) warp_sums[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t ws = warp_sums[lane], wi = ws;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, wi, off);
      if (lane >= off) wi += v;
    }
    warp_sums[lane] = wi - ws;  // exclusive prefix of the warp sums
    if (lane == 31 && total) *total = wi;
  }
  __syncthreads();
  uint32_t run = warp_sums[w] + incl - s;
#pragma unroll 8
  for (int64_t i = lo; i < hi; ++i) {
    const uint32_t v = a[i];
    a[i] = run;
    run += v;
  }
}

fg_status stable_order(const uint32_t* keys, size_t n, uint32_t bound, uint32_t* order, uint32_t* sorted,
                       SortScratch& s, cudaStream_t st) {
  if (n == 0) return FG_OK;
  if (n >= ((size_t)1 << 32)) {
    set_error("at most 2^32 - 1 keys can be ordered");
    return FG_UNSUPPORTED_STRUCTURE;
  }
  const int bits = bound > 1 ? 32 - __builtin_clz(bound - 1) : 0;
  if (bits == 0) {
    FG_LAUNCH(k_iota_copy, grid_for(n, 256), 256, 0, st, (int64_t)n, keys, order, sorted);
    return FG_OK;
  }
  const int passes = (bits + 7) / 8, per = (bits + passes - 1) / passes;
  const int64_t ntiles = ((int64_t)n + RS_TILE - 1) / RS_TILE;
  FG_TRY(s.counts.resize((size_t)ntiles << per));
  for (int b = 0; b < 2; ++b) {
    FG_TRY(s.keys[b].resize(n));
    FG_TRY(s.vals[b].resize(n));
  }
  const uint32_t* kin = keys;
  const uint32_t* vin = nullptr;
  for (int p = 0; p < passes; ++p) {
    const int shift = p * per, nb = std::min(per, bits - shift);
    const bool last = p == passes - 1;
    uint32_t* kout = last ? (sorted ? sorted : s.keys[p & 1].get()) : s.keys[p & 1].get();
    uint32_t* vout = last ? order : s.vals[p & 1].get();
    FG_LAUNCH(k_radix_count, (unsigned)ntiles, RS_THREADS, 0, st, kin, (int64_t)n, shift, nb, ntiles,
              s.counts.get());
    FG_LAUNCH(k_scan_exclusive_u32, 1, 1024, 0, st, s.counts.get(), ntiles << nb, (uint32_t*)nullptr);
    FG_LAUNCH(k_radix_scatter, (unsigned)ntiles, RS_THREADS, 0, st, kin, vin, (int64_t)n, shift, nb, ntiles,
              s.counts.get(), kout, vout);
    kin = kout;
    vin = vout;
  }
  return FG_OK;
}

fg_status key_offsets(const uint32_t* sorted, size_t n, uint32_t bound, int64_t* off, cudaStream_t st) {
  FG_LAUNCH(k_key_offsets, grid_for(n + 1, 256), 256, 0, st, sorted, (int64_t)n, bound, off);
  return FG_OK;
}

}  // namespace fg
