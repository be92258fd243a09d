// Device ordering of observations by bounded 32-bit keys: the stable counting
// sorts that turn insertion-ordered observations into emission order (one
// Frame batch per camera, examples/bal/model.rs:187-200) and into the per-variable and
// per-point edge lists of the Schur structure, done on the device instead of
// in host loops.
//
// stable_order is an LSD radix sort over the bits the key bound needs (8-bit
// digits at most, as many passes as the bound takes). Each pass is a stable
// counting scatter over tiles of 2,048 keys: a per-tile digit histogram, one
// exclusive scan of the digit-major count table, and a scatter whose in-tile
// ranks come from warp match masks and per-warp running digit counts, so
// equal keys keep their input order.
#pragma once
#include "common.cuh"

namespace fg {

struct SortScratch {
  DBuf<uint32_t> keys[2], vals[2], counts;
};

// order[i] = index of the i-th key in nondecreasing key order, ties in index
// order; sorted (optional) receives keys[order[i]]. Every key must be below
// `bound`; a larger key is ordered by its low bits only. n < 2^32.
fg_status stable_order(const uint32_t* keys, size_t n, uint32_t bound, uint32_t* order, uint32_t* sorted,
                       SortScratch& s, cudaStream_t st);

// off[k] = number of sorted keys below k, for k in [0, bound] (so off[bound] = n),
// from nondecreasing keys below `bound`.
fg_status key_offsets(const uint32_t* sorted, size_t n, uint32_t bound, int64_t* off, cudaStream_t st);

// In-place exclusive scan of m 32-bit counts in one block; *total (optional,
// device) receives the sum.
__global__ void k_scan_exclusive_u32(uint32_t* a, int64_t m, uint32_t* total);

}  // namespace fg
