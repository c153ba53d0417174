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

constexpr int kSlotsPerLane = (kMaxM + 31) / 32;  // 5

// Full direction table (signed dx, no normalisation at lookup), kept in shared
// memory by the kernels that evaluate moves: entry (dx + kMaxN - 1) * kLutW +
// dy + kMaxN - 1 holds the id of (dx, dy); (0, 0) holds 0 and is never read.
// With key(r, c) = r * kLutW + c the entry of the difference a - b sits at
// key(a) - key(b) + kFullLutCentre, one add per lookup.
constexpr int kFullLutSize = kLutW * kLutW;  // 22,201 entries
constexpr size_t kFullLutBytes = ((sizeof(uint16_t) * kFullLutSize + 15) / 16) * 16;
constexpr int kFullLutCentre = (kMaxN - 1) * kLutW + (kMaxN - 1);

// Copies the full table built once per device (n3host::dir_lut_full_device_ptr)
// into shared memory, 16 bytes at a time; all threads of the block call it.
__device__ __forceinline__ void full_lut_copy(uint16_t* __restrict__ dst, const uint16_t* __restrict__ full) {
  const uint4* s = reinterpret_cast<const uint4*>(full);
  uint4* d = reinterpret_cast<uint4*>(dst);
  for (int i = threadIdx.x; i < (int)(kFullLutBytes / 16); i += blockDim.x) d[i] = s[i];
}

__device__ __forceinline__ int dir_id_full(const uint16_t* __restrict__ lutf, int dx, int dy) {
  return lutf[dx * kLutW + dy + kFullLutCentre];
}

__device__ __forceinline__ void hist_release(uint32_t* hist, const int (&ids)[kSlotsPerLane]) {
#pragma unroll
  for (int t = 0; t < kSlotsPerLane; ++t)
    if (ids[t] >= 0) hist_clear(hist, ids[t]);
}

__device__ __forceinline__ bool legal_swap(const int* cs, int u, int v) {
  const int cu = cs[u], cv = cs[v];
  return (u >> 1) != (v >> 1) && cu != cv && cs[u ^ 1] != cv && cs[v ^ 1] != cu;
}


}  // namespace n3

namespace n3host {
// Device address of the direction table on the current device (set-up on
// first use by ensure_device_tables).
const uint16_t* dir_lut_device_ptr();
// Device address of the full signed table built from it (kFullLutBytes).
const uint16_t* dir_lut_full_device_ptr();
}  // namespace n3host
