// CPython's random.Random on the device: MT19937 (Matsumoto & Nishimura,
// 1998) and random.shuffle, draw for draw.  Shared by the device beam search
// (beam.cu) and the exhaustive beam (exhaustive.cu).
#pragma once

#include <stdint.h>

namespace n3 {
namespace beam {

// --------------------------------------------------------------------------
// MT19937 as CPython's random.Random uses it (Matsumoto & Nishimura, 1998;
// seeding by init_by_array, 2002), and CPython's shuffle: for i = len-1 .. 1,
// j = _randbelow(i + 1) with getrandbits(bit_length(i + 1)) and rejection.
// --------------------------------------------------------------------------
constexpr int kMT = 624;

// The state twist by one warp: ordered chunks of 32 words reproduce the
// sequential update exactly (word k reads words k + 1 and k + 397 before they
// are updated and word k - 227 after, as the one-thread loop does, because
// 397 and 227 both exceed the chunk width).
__device__ inline void mt_twist_warp(uint32_t* mt, int lane) {
  for (int k0 = 0; k0 < kMT; k0 += 32) {
    const int k = k0 + lane;
    uint32_t nv = 0u;
    if (k < kMT) {
      const uint32_t y = (mt[k] & 0x80000000u) | (mt[(k + 1) % kMT] & 0x7fffffffu);
      nv = mt[(k + 397) % kMT] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    __syncwarp();
    if (k < kMT) mt[k] = nv;
    __syncwarp();
  }
}

__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

// random.Random.shuffle by one warp, draw for draw the same as CPython.  The
// 624 tempered outputs of the current state block sit in `out`.  Each round
// takes the next (up to) 32 draws at once.  Step i (descending) draws
// r = getrandbits(k), k = bit_length(i + 1), until r <= i (_randbelow).  A
// round covers the next m <= 32 steps that share k; a draw with r <= i - m + 1
// is accepted and one with r > i rejected whatever the earlier lanes decide, so
// the lanes' decisions and, by a prefix count, their steps follow at once; the
// round stops after the first draw that needs its exact step (i - m + 1 < r <= i,
// decided then) or at the m-th acceptance.  A round's accepted swaps (s, j) cover consecutive steps s_max .. s_min;
// they commute when no j lies in [s_min, s_max] (other than j = s) and no two j
// coincide (a bit per position in `seen`, zero on entry and on return, finds
// repeats), and are then made by all lanes at once, otherwise by lane 0 in step
// order.  idx: position in the block (warp-uniform).
template <class T>
__device__ void py_shuffle_warp(uint32_t* mt, uint32_t* out, int& idx, T* values, int count, uint32_t* seen,
                                int lane) {
  for (int k = lane; k < kMT; k += 32) out[k] = mt_temper(mt[k]);
  __syncwarp();
  const unsigned below = (1u << lane) - 1u;
  int i = count - 1;
  while (i >= 1) {
    if (idx >= kMT) {
      mt_twist_warp(mt, lane);
      for (int k = lane; k < kMT; k += 32) out[k] = mt_temper(mt[k]);
      __syncwarp();
      idx = 0;
    }
    const int shift = __clz((uint32_t)i + 1u);  // 32 - bit_length(i + 1)
    // steps i .. i - m + 1 share the draw width: their ranges are >= 2^(bit_length(i + 1) - 1)
    const int m = min(32, i + 2 - (1 << (31 - shift)));
    const int draws = min(32, kMT - idx);
    uint32_t r = 0u;
    bool acc = false, amb = false;
    if (lane < draws) {
      r = out[idx + lane] >> shift;
      acc = (int)r <= i - (m - 1);
      amb = !acc && (int)r <= i;
    }
    const unsigned amb_mask = __ballot_sync(0xffffffffu, amb);
    const int a = amb_mask ? __ffs(amb_mask) - 1 : draws;  // first draw that needs its exact step
    unsigned acc_mask = __ballot_sync(0xffffffffu, acc) & ((a < 32 ? (1u << a) : 0u) - 1u);
    int used = a;
    if (__popc(acc_mask) < m && a < draws) {  // decide draw a with its step i - (accepted draws before it)
      const int sa = i - __popc(acc_mask);
      if ((int)__shfl_sync(0xffffffffu, r, a) <= sa) acc_mask |= 1u << a;
      used = a + 1;
    }
    if (__popc(acc_mask) >= m) {  // the m-th acceptance ends the round (the next step draws wider or
                                  // narrower, or there is none); later draws stay unused
      const int z = __ffs(__ballot_sync(0xffffffffu, ((acc_mask >> lane) & 1u) &&
                                                      __popc(acc_mask & ((2u << lane) - 1u)) == m)) - 1;
      acc_mask &= (2u << z) - 1u;  // 2u << 31 wraps to 0: all bits
      used = z + 1;
    }
    const int nb = __popc(acc_mask);
    const int s_max = i, s_min = s_max - nb + 1;
    // an accepted draw swaps its step s = s_max - (accepted draws before it) with j = r;
    // a j inside [s_min, s_max] (other than s) or met twice orders the swaps
    const bool mine = (acc_mask >> lane) & 1u;
    const int sm = s_max - __popc(acc_mask & below), jm = (int)r;
    bool conflict = false;
    if (mine) {
      conflict = jm >= s_min && jm != sm;
      const uint32_t bit = 1u << (jm & 31);
      conflict |= (atomicOr(&seen[jm >> 5], bit) & bit) != 0u;
    }
    if (!__any_sync(0xffffffffu, conflict)) {
      if (mine && jm != sm) {
        const T t = values[sm];
        values[sm] = values[jm];
        values[jm] = t;
      }
    } else {
      for (int l = 0; l < 32; ++l) {  // in step order: lane order of the accepted draws
        const int sl = __shfl_sync(0xffffffffu, sm, l), jl = __shfl_sync(0xffffffffu, jm, l);
        if (lane == 0 && ((acc_mask >> l) & 1u)) {
          const T t = values[sl];
          values[sl] = values[jl];
          values[jl] = t;
        }
      }
    }
    if (mine) atomicAnd(&seen[jm >> 5], ~(1u << (jm & 31)));
    __syncwarp();
    i -= nb;
    idx += used;
  }
}

}  // namespace beam
}  // namespace n3
