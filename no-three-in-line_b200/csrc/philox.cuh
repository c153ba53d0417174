// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11): ten rounds of two
// 32x32->64 multiplies with the published multipliers and Weyl key bumps.
// Known-answer vectors of the paper's reference implementation are checked by
// the tests (ctr = key = 0 -> 6627e8d5 e169c58d bc57ac4c 9b00dbd8).
#pragma once

#include <stdint.h>

namespace n3 {

struct U4 {
  uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {  // fully unrolled by the compiler (constant trip count)
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    const U4 o = {(uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k1, (uint32_t)p0};
    c = o;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Stream tags (fourth counter word) separating the uses of one seed.
enum : uint32_t {
  kTagPropose = 0x50000000u,   // proposal slots u, v and the Metropolis uniform
  kTagExchange = 0xE0000000u,  // neighbour temperature exchanges
  kTagCandidate = 0xC0000000u, // learned-proposal candidate slots and sampling
  kTagBias = 0xB0000000u,      // badness-weighted slot draw of a walk proposal
};

}  // namespace n3
