// Space-filling-curve key of a point of the 1024^3 grid, for the spatial
// ordering of active targets (anchor offsets: an i-block's targets must be
// compact for its anchor-relative FP32 offsets to be accurate).
//
// Hilbert index by Skilling's method (J. Skilling, "Programming the Hilbert
// curve", AIP Conf. Proc. 707, 381 (2004)): the coordinates are transformed to
// the curve's "transpose" form (inverse undo of the excess rotations, then Gray
// encoding), and the index is the bit interleave of the transpose with axis 0
// most significant at every level.  Consecutive keys are adjacent grid cells,
// so a run of consecutive targets never jumps across the cluster the way a
// Morton (Z-order) run does at octant boundaries.
#pragma once
#include <cstdint>

#if !defined(__CUDACC__)
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#endif

namespace abyss {

// 10 low bits of v spread to every third bit (bit k -> bit 3k).
__host__ __device__ inline uint32_t spread_bits10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Hilbert index (30 bits) of grid point (x0, x1, x2), each in [0, 1024).
__host__ __device__ inline uint32_t hilbert_key10(uint32_t x0, uint32_t x1, uint32_t x2) {
  uint32_t X[3] = {x0 & 0x3ffu, x1 & 0x3ffu, x2 & 0x3ffu};
  const uint32_t top = 1u << 9;
  for (uint32_t q = top; q > 1; q >>= 1) {
    const uint32_t p = q - 1;
    for (int i = 0; i < 3; ++i) {
      if (X[i] & q) {
        X[0] ^= p;  // invert the low bits of axis 0
      } else {      // exchange the low bits of axes 0 and i
        const uint32_t t = (X[0] ^ X[i]) & p;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];  // Gray encode
  X[2] ^= X[1];
  uint32_t t = 0;
  for (uint32_t q = top; q > 1; q >>= 1)
    if (X[2] & q) t ^= q - 1;
  X[0] ^= t;
  X[1] ^= t;
  X[2] ^= t;
  return (spread_bits10(X[0]) << 2) | (spread_bits10(X[1]) << 1) | spread_bits10(X[2]);
}

}  // namespace abyss
