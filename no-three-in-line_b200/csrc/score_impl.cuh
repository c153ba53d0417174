// Device bodies of the two population scorers, shared by score.cu (the
// scoring entry points) and tempering.cu (the on-device energy audit).
// See score.cu for the method.
#pragma once

#include "dirs.cuh"
#include "n3_common.cuh"

namespace n3 {

// Tests of the two pivots of row `rho` against all pairs (x, y) with x on the
// larger side (R register slots per lane) and y on the smaller side.
// X=(r_x,c_x), J=(rho,c_j), Y=(r_y,c_y) are collinear iff
//   (r_x-rho)(c_y-c_j) == (c_x-c_j)(r_y-rho)
//   <=>  a_x*c_y == a_y*b_x + a_x*c_j,   a = r - rho, b_x = c_x - c_j.
template <int R, bool BAD>
__device__ __forceinline__ int det_pivot_row(const int* __restrict__ cs, int n, int rho, int lane, int* bad) {
  const int cj0 = cs[2 * rho], cj1 = cs[2 * rho + 1];
  const int above = rho, below = n - 1 - rho;
  const bool lanes_above = above >= below;
  const int L = 2 * (lanes_above ? above : below);
  const int lbase = lanes_above ? 0 : 2 * rho + 2;
  const int rb0 = lanes_above ? rho + 1 : 0;
  const int rb1 = lanes_above ? n : rho;
  int ax[R], bx0[R], bx1[R], k0[R], k1[R], sx[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int x = lane + 32 * r;
    if (x < L) {
      const int s = lbase + x;
      const int a = (s >> 1) - rho, c = cs[s];
      ax[r] = a;
      bx0[r] = c - cj0;
      bx1[r] = c - cj1;
      k0[r] = a * cj0;
      k1[r] = a * cj1;
      sx[r] = s;
    } else {  // idle slot: products are 0, targets -1, never a hit
      ax[r] = 0;
      bx0[r] = 0;
      bx1[r] = 0;
      k0[r] = -1;
      k1[r] = -1;
      sx[r] = 0;
    }
  }
  int cnt = 0;
  const int2* rows2 = reinterpret_cast<const int2*>(cs);
  // Each target T (one per pivot) matches at most one of the row's two
  // products: P0 == P1 needs a_x == 0 (a lane slot always has a_x != 0; an
  // idle slot has target -1).  So every target contributes one OR of two
  // compares, and the count needs no per-test conversion.  Two hits of one
  // register slot in one row do occur (two lines through x, one per pivot).
#pragma unroll 2
  for (int row = rb0; row < rb1; ++row) {
    const int2 cy = rows2[row];
    const int ay = row - rho;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int P0 = ax[r] * cy.x, P1 = ax[r] * cy.y;
      const int T0 = ay * bx0[r] + k0[r], T1 = ay * bx1[r] + k1[r];
      const bool g0 = (P0 == T0) | (P1 == T0), g1 = (P0 == T1) | (P1 == T1);
      cnt += (int)g0 + (int)g1;
      if (BAD && (g0 | g1)) {
        if (g0) {  // x, pivot 2 rho, and slot 2 row or 2 row + 1
          atomicAdd(bad + sx[r], 1);
          atomicAdd(bad + 2 * rho, 1);
          atomicAdd(bad + 2 * row + (P0 == T0 ? 0 : 1), 1);
        }
        if (g1) {
          atomicAdd(bad + sx[r], 1);
          atomicAdd(bad + 2 * rho + 1, 1);
          atomicAdd(bad + 2 * row + (P0 == T1 ? 0 : 1), 1);
        }
      }
    }
  }
  return cnt;
}

template <bool BAD>
__device__ __forceinline__ int det_state(const int* __restrict__ cs, int n, int lane, int* bad) {
  int cnt = 0;
  for (int rho = 1; rho < n - 1; ++rho) {
    const int L = 2 * max(rho, n - 1 - rho);
    switch ((L + 31) >> 5) {
      case 1: cnt += det_pivot_row<1, BAD>(cs, n, rho, lane, bad); break;
      case 2: cnt += det_pivot_row<2, BAD>(cs, n, rho, lane, bad); break;
      case 3: cnt += det_pivot_row<3, BAD>(cs, n, rho, lane, bad); break;
      case 4: cnt += det_pivot_row<4, BAD>(cs, n, rho, lane, bad); break;
      default: cnt += det_pivot_row<5, BAD>(cs, n, rho, lane, bad); break;
    }
  }
  return cnt;
}

// Slope line count of one state.  Returns sum over anchors of badness (3E).
// lutf: the full direction table in shared memory (dirs.cuh).  hist: this
// warp's zeroed direction histogram (kDirWords words); it is left zeroed on
// return.  bad_out (per slot) may be null.
__device__ __forceinline__ int slope_state(const int* __restrict__ cs, int n, const uint16_t* __restrict__ lutf,
                                           uint32_t* __restrict__ hist, int lane, int* __restrict__ bad_out) {
  constexpr int kT = (kMaxM + 31) / 32;
  const int m = 2 * n;
  // this lane's slots b = lane + 32 t: their keys (row * kLutW + column) and rows
  int key[kT], row[kT];
#pragma unroll
  for (int t = 0; t < kT; ++t) {
    const int b = lane + 32 * t;
    row[t] = b < m ? b >> 1 : -1;
    key[t] = b < m ? (b >> 1) * kLutW + cs[b] : 0;
  }
  int total = 0;
  for (int a = 0; a < m; ++a) {
    const int ra = a >> 1;
    const uint16_t* base = lutf + kFullLutCentre - (ra * kLutW + cs[a]);
    int pairs = 0;
    int ids[kT];
#pragma unroll
    for (int t = 0; t < kT; ++t) {
      ids[t] = -1;
      if (row[t] >= 0 && row[t] != ra) {  // the row partner has the lone direction (0,1)
        const int id = base[key[t]];
        ids[t] = id;
        pairs += hist_add(hist, id);  // earlier points on this direction
      }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < kT; ++t)
      if (ids[t] >= 0) hist_clear(hist, ids[t]);
    __syncwarp();
    pairs = warp_sum(pairs);
    if (bad_out != nullptr && lane == (a & 31)) bad_out[a] = pairs;
    total += pairs;
  }
  return total;
}

// The slope count with 4-bit counters (8 per word, kHist4Words words per
// warp): the same pair sums as slope_state in half the shared memory, so twice
// the warps fit beside one direction table.  lutf is the caller's copy of the
// full table with the entry of (0, 0) set to kDirCount, a counter of its own
// (the last word): every slot of the state is inserted, the centre itself into
// that counter (adding 0, once) and its row partner into the (0, 1) class,
// where it is alone (adding 0), so no insertion tests its row.  A counter that
// reaches 16 wraps; by then its direction has added 0 + 1 + ... + 15 = 120
// pairs to the centre's sum, so *overflow is set for every centre whose sum
// reaches 120, and the caller recounts the state with slope_state_halves.
// Every touched word is cleared, so the histogram is zero on return.
constexpr int kDirWords4 = kDirCount / 8;     // 848
constexpr int kHist4Words = kDirWords4 + 1;   // + the word of the centre's own counter
__device__ __forceinline__ int slope_state4(const int* __restrict__ cs, int n, const uint16_t* __restrict__ lutf,
                                            uint32_t* __restrict__ hist, int lane, int* __restrict__ bad_out,
                                            bool* overflow) {
  constexpr int kT = (kMaxM + 31) / 32;
  const int m = 2 * n;
  int key[kT];
#pragma unroll
  for (int t = 0; t < kT; ++t) {
    const int b = lane + 32 * t;
    key[t] = b < m ? (b >> 1) * kLutW + cs[b] : -1;
  }
  int total = 0;
  bool ovf = false;
  for (int a = 0; a < m; ++a) {
    const uint16_t* base = lutf + kFullLutCentre - ((a >> 1) * kLutW + cs[a]);
    int pairs = 0;
    int ids[kT];
#pragma unroll
    for (int t = 0; t < kT; ++t) {
      ids[t] = -1;
      if (key[t] >= 0) {
        const int id = base[key[t]];
        ids[t] = id;
        const int sh = (id & 7) << 2;
        pairs += (int)((atomicAdd(hist + (id >> 3), 1u << sh) >> sh) & 0xFu);
      }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < kT; ++t)
      if (ids[t] >= 0) hist[ids[t] >> 3] = 0u;
    __syncwarp();
    pairs = warp_sum(pairs);
    ovf |= pairs >= 120;
    if (bad_out != nullptr && lane == (a & 31)) bad_out[a] = pairs;
    total += pairs;
  }
  *overflow = ovf;  // uniform: from warp sums
  return total;
}

// The forward slope count (from each centre a only the slots b > a, so every
// collinear triple is counted once, from its first slot) with 4-bit counters,
// as slope_state4; returns E for the whole warp.  A centre whose forward pair
// sum reaches 120 sets *overflow (see slope_state4).
__device__ __forceinline__ int slope_forward_state4(const int* __restrict__ cs, int n,
                                                    const uint16_t* __restrict__ lutf, uint32_t* __restrict__ hist,
                                                    int lane, bool* overflow) {
  constexpr int kT = (kMaxM + 31) / 32;
  const int m = 2 * n;
  int key[kT];
#pragma unroll
  for (int t = 0; t < kT; ++t) {
    const int b = lane + 32 * t;
    key[t] = b < m ? (b >> 1) * kLutW + cs[b] : -1;
  }
  int total = 0;
  bool ovf = false;
  for (int a = 0; a < m - 2; ++a) {
    const uint16_t* base = lutf + kFullLutCentre - ((a >> 1) * kLutW + cs[a]);
    int pairs = 0;
    int ids[kT];
#pragma unroll
    for (int t = 0; t < kT; ++t) {
      ids[t] = -1;
      if (key[t] >= 0 && lane + 32 * t > a) {  // the row partner is alone in its direction
        const int id = base[key[t]];
        ids[t] = id;
        const int sh = (id & 7) << 2;
        pairs += (int)((atomicAdd(hist + (id >> 3), 1u << sh) >> sh) & 0xFu);
      }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < kT; ++t)
      if (ids[t] >= 0) hist[ids[t] >> 3] = 0u;
    __syncwarp();
    pairs = warp_sum(pairs);
    ovf |= pairs >= 120;
    total += pairs;
  }
  *overflow = ovf;
  return total;
}

// The exact slope count in the 4-bit histogram's space (kDirWords4 words):
// 8-bit counters for the direction ids of each half, [0, kDirCount / 2) then
// [kDirCount / 2, kDirCount), one pass per half.  Same results as slope_state.
static __device__ __noinline__ int slope_state_halves(const int* __restrict__ cs, int n, const uint16_t* __restrict__ lutf,
                                               uint32_t* __restrict__ hist, int lane, int* __restrict__ bad_out) {
  constexpr int kT = (kMaxM + 31) / 32;
  constexpr int kHalf = kDirCount / 2;
  static_assert(kHalf == 4 * kDirWords4, "one half of the ids fills the 4-bit histogram as 8-bit counters");
  const int m = 2 * n;
  int total = 0;
  for (int a = 0; a < m; ++a) {
    const int ra = a >> 1;
    const uint16_t* base = lutf + kFullLutCentre - (ra * kLutW + cs[a]);
    int ids[kT];
#pragma unroll
    for (int t = 0; t < kT; ++t) {
      const int b = lane + 32 * t;
      ids[t] = (b < m && (b >> 1) != ra) ? (int)base[(b >> 1) * kLutW + cs[b]] : -1;
    }
    int pairs = 0;
    for (int h = 0; h < 2; ++h) {
#pragma unroll
      for (int t = 0; t < kT; ++t) {
        const int local = ids[t] - h * kHalf;
        if (ids[t] >= 0 && local >= 0 && local < kHalf) pairs += hist_add(hist, local);
      }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < kT; ++t) {
        const int local = ids[t] - h * kHalf;
        if (ids[t] >= 0 && local >= 0 && local < kHalf) hist_clear(hist, local);
      }
      __syncwarp();
    }
    pairs = warp_sum(pairs);
    if (bad_out != nullptr && lane == (a & 31)) bad_out[a] = pairs;
    total += pairs;
  }
  return total;
}


}  // namespace n3
