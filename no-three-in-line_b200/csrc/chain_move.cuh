// Exact move evaluation and application for one chain held by a warp, shared
// by the tempering kernel (uniform proposals) and the learned-proposal step.
#pragma once

#include "dirs.cuh"
#include "n3_common.cuh"
#include "philox.cuh"

namespace n3 {

// Exact dE of the move (u, v) of the chain held by this warp (state in shared
// memory: columns cs, badness bs, m slots; lutf the full direction table in
// shared memory), Metropolis test against the
// threshold row `thr` (width W) with the 32-bit uniform z, and on acceptance
// the exact update of every slot's badness, the columns and E.  The caller
// has checked legality.  Returns 1 if accepted; *dE_out receives dE.
// FORCE: the move is applied whatever its dE (no Metropolis test).
template <bool FORCE>
__device__ __forceinline__ int move_exact_t(int* __restrict__ cs, int* __restrict__ bs, int m,
                                            const uint16_t* __restrict__ lutf, uint32_t* __restrict__ hist, int lane,
                                            int u, int v, uint32_t z, const uint32_t* __restrict__ thr, int W, int& E,
                                            uint32_t& err, int* dE_out) {
  const int ru = u >> 1, rv = v >> 1, cu = cs[u], cv = cs[v];
  int ids[kSlotsPerLane], cnt_new[kSlotsPerLane];
  // centre u' = (r_u, c_v)
  const int part_a = hist_build_full(cs, m, ru, cv, u, v, lutf, hist, lane, ids);
  __syncwarp();
  const int line_new = dir_id_full(lutf, rv - ru, cu - cv);
  const int j_new = hist_get(hist, line_new);
#pragma unroll
  for (int t = 0; t < kSlotsPerLane; ++t)
    cnt_new[t] = ids[t] >= 0 ? hist_get(hist, ids[t]) - 1 + (ids[t] == line_new) : 0;
  __syncwarp();
  hist_release(hist, ids);
  __syncwarp();
  // centre v' = (r_v, c_u)
  const int part_b = hist_build_full(cs, m, rv, cu, u, v, lutf, hist, lane, ids);
  __syncwarp();
#pragma unroll
  for (int t = 0; t < kSlotsPerLane; ++t) cnt_new[t] += ids[t] >= 0 ? hist_get(hist, ids[t]) - 1 : 0;
  __syncwarp();
  hist_release(hist, ids);
  // points of A on the old line (u, v)
  int joint = 0;
#pragma unroll
  for (int t = 0; t < kSlotsPerLane; ++t) {
    const int k = lane + 32 * t;
    if (k < m && k != u && k != v) joint += (rv - ru) * (cs[k] - cu) == (cv - cu) * ((k >> 1) - ru);
  }
  const int sum_ab = warp_sum(part_a + (part_b << 16));
  const int sum_joint = warp_sum(joint);
  const int t_a = sum_ab & 0xFFFF, t_b = sum_ab >> 16;
  const int dE = (t_a + t_b + j_new) - (bs[u] + bs[v] - sum_joint);
  *dE_out = dE;
  const bool accept = FORCE || dE <= 0 || (dE < W && z < thr[dE]);
  if (!accept) {
    __syncwarp();
    return 0;
  }
  // Old-side histograms: exact badness change of every other point.
  __syncwarp();
  int dB[kSlotsPerLane];
  const int part_c = hist_build_full(cs, m, ru, cu, u, v, lutf, hist, lane, ids);
  __syncwarp();
  const int line_old = dir_id_full(lutf, rv - ru, cv - cu);
  const int j_old = hist_get(hist, line_old);
#pragma unroll
  for (int t = 0; t < kSlotsPerLane; ++t)
    dB[t] = cnt_new[t] - (ids[t] >= 0 ? hist_get(hist, ids[t]) - 1 + (ids[t] == line_old) : 0);
  __syncwarp();
  hist_release(hist, ids);
  __syncwarp();
  const int part_d = hist_build_full(cs, m, rv, cv, u, v, lutf, hist, lane, ids);
  __syncwarp();
#pragma unroll
  for (int t = 0; t < kSlotsPerLane; ++t) dB[t] -= ids[t] >= 0 ? hist_get(hist, ids[t]) - 1 : 0;
  __syncwarp();
  hist_release(hist, ids);
  const int sum_cd = warp_sum(part_c + (part_d << 16));
  const int t_c = sum_cd & 0xFFFF, t_d = sum_cd >> 16;
  if (bs[u] != t_c + j_old || bs[v] != t_d + j_old || j_old != sum_joint) err |= kErrAudit;
  __syncwarp();
#pragma unroll
  for (int t = 0; t < kSlotsPerLane; ++t) {
    const int k = lane + 32 * t;
    if (k < m && k != u && k != v) bs[k] += dB[t];
  }
  if (lane == 0) {
    bs[u] = t_a + j_new;
    bs[v] = t_b + j_new;
    cs[u] = cv;
    cs[v] = cu;
  }
  __syncwarp();
  E += dE;
  return 1;
}

__device__ __forceinline__ int move_exact(int* __restrict__ cs, int* __restrict__ bs, int m,
                                          const uint16_t* __restrict__ lutf, uint32_t* __restrict__ hist, int lane,
                                          int u, int v, uint32_t z, const uint32_t* __restrict__ thr, int W, int& E,
                                          uint32_t& err, int* dE_out) {
  return move_exact_t<false>(cs, bs, m, lutf, hist, lane, u, v, z, thr, W, E, err, dE_out);
}

// One uniform proposal (tempering.py:50-58 draws u, v uniformly; here from a
// Philox block).  Returns 1 if accepted.
__device__ __forceinline__ int propose(int* __restrict__ cs, int* __restrict__ bs, int m,
                                       const uint16_t* __restrict__ lutf, uint32_t* __restrict__ hist, int lane,
                                       U4 rnd, const uint32_t* __restrict__ thr, int W, int& E, uint32_t& err) {
  const int u = (int)__umulhi(rnd.x, (unsigned)m);
  const int v = (int)__umulhi(rnd.y, (unsigned)m);
  if (!legal_swap(cs, u, v)) return 0;
  int dE;
  return move_exact(cs, bs, m, lutf, hist, lane, u, v, rnd.z, thr, W, E, err, &dE);
}

}  // namespace n3
