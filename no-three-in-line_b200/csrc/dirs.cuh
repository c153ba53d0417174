// Primitive undirected directions and per-warp direction histograms.
//
// Two distinct points a, b lie on one line with a third point x iff the
// gcd-reduced, sign-normalised directions x->a and x->b are equal
// (src/no_three_75/verifier_b.py:8-19 is the reference's normalisation: divide
// by gcd(|dx|,|dy|), then make dx > 0, or dy > 0 when dx == 0).  For the grid
// bound n <= 75 there are kDirCount = 6784 such directions; the table
// dir_lut[dx * kLutW + dy + kMaxN - 1] (dx in [0, 74], dy in [-74, 74]) maps a
// difference vector to the compact id of its direction.  It is built once per
// device by build_dir_lut_kernel (gcd on the device, ids in (p, q) order).
//
// A direction histogram holds one 8-bit counter per id (4 per 32-bit word) in
// shared memory.  Inserting a point returns how many earlier points share its
// direction, so the sum over insertions is sum_dir C(count, 2): the number of
// point pairs collinear with the histogram's centre.  Counts never exceed
// 2 * kMaxN - 2 = 148 < 256.
#pragma once

#include "n3_common.cuh"

namespace n3 {

constexpr int kDirCount = 6784;
constexpr int kDirWords = kDirCount / 4;

// Compact id of the direction of (dx, dy) != (0, 0), |dx|, |dy| <= kMaxN - 1.
__device__ __forceinline__ int dir_id(const uint16_t* __restrict__ lut, int dx, int dy) {
  if (dx < 0 || (dx == 0 && dy < 0)) {
    dx = -dx;
    dy = -dy;
  }
  return lut[dx * kLutW + dy + (kMaxN - 1)];
}

// Adds one point with direction `id`; returns the count before the insertion.
__device__ __forceinline__ int hist_add(uint32_t* hist, int id) {
  const int sh = (id & 3) << 3;
  const uint32_t old = atomicAdd(hist + (id >> 2), 1u << sh);
  return (int)((old >> sh) & 0xFFu);
}

__device__ __forceinline__ int hist_get(const uint32_t* hist, int id) {
  return (int)((hist[id >> 2] >> ((id & 3) << 3)) & 0xFFu);
}

__device__ __forceinline__ void hist_clear(uint32_t* hist, int id) { hist[id >> 2] = 0u; }

}  // namespace n3

namespace n3host {
// Device address of the direction table on the current device (set-up on
// first use by ensure_device_tables).
const uint16_t* dir_lut_device_ptr();
}  // namespace n3host
