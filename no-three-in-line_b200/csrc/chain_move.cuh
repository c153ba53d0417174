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
// Metropolis test of an acceptance energy e = dE + umb_q / 2^24 (umb_q: an
// umbrella restraint term in units of 2^-24): accept iff e <= 0 or z is below
// thr[a] x f1[b >> 16] x f2[(b >> 8) & 255] x f3[b & 255] (32-bit fixed-point
// products), where e = a + b / 2^24.  thr[a] = floor(2^32 exp(-a/T)); frac
// holds f1, f2, f3 (256 each): floor(2^32 exp(-k/(2^8 T))), exp(-k/(2^16 T)),
// exp(-k/(2^24 T)).  A factor whose index is 0 is skipped, so umb_q = 0 is the
// plain test.
__device__ __forceinline__ bool umbrella_accept(int dE, int64_t umb_q, uint32_t z, const uint32_t* __restrict__ thr,
                                                int W, const uint32_t* __restrict__ frac) {
  const int64_t e = ((int64_t)dE << 24) + umb_q;
  if (e <= 0) return true;
  const int64_t a = e >> 24;
  if (a >= W) return false;
  uint32_t t = thr[a];
  const int b = (int)(e & 0xFFFFFF);
  if (b >> 16) t = (uint32_t)(((uint64_t)t * frac[b >> 16]) >> 32);
  if ((b >> 8) & 255) t = (uint32_t)(((uint64_t)t * frac[256 + ((b >> 8) & 255)]) >> 32);
  if (b & 255) t = (uint32_t)(((uint64_t)t * frac[512 + (b & 255)]) >> 32);
  return z < t;
}

// FORCE: the move is applied whatever its dE (no Metropolis test).
// UMB: the test adds the umbrella term umb_q (umbrella_accept).
// The threads that evaluate one chain's moves: WPC warps, 32 WPC threads.
// Thread t of the team owns slots t, t + 32 WPC, ... (kSlots of them).  With
// WPC = 1 the team is a warp (__syncwarp, warp reductions); with WPC > 1 the
// team meets at the named barrier `bar` (ids 1..15; id 0 is __syncthreads)
// and reduces through `red`, 2 WPC ints of shared memory used alternately, so
// a reduction's buffer is rewritten only after every thread has passed the
// next reduction's barrier.  Every decision a team takes (legality, dE,
// acceptance) is computed from team-wide values, so all its threads follow
// the same path through barriers and reductions.
template <int WPC>
struct Team {
  static constexpr int kThreads = 32 * WPC;
  static constexpr int kSlots = (kMaxM + kThreads - 1) / kThreads;  // 5, 3, 2, 1
  int t;         // rank in the team
  int bar;       // named barrier id (WPC > 1)
  int* red;      // reduction scratch (WPC > 1)
  int phase;     // which half of red the next reduction uses
  // KEYED moves only: the direction-table key row * kLutW + column of each of
  // this thread's slots (set by the caller from the state; a KEYED move keeps
  // it up to date)
  int key[kSlots];
  __device__ __forceinline__ void sync() const {
    if constexpr (WPC == 1) {
      __syncwarp();
    } else {
      // non-.aligned form: correct even where a warp has not reconverged
      asm volatile("barrier.sync %0, %1;" ::"r"(bar), "n"(kThreads) : "memory");
    }
  }
  __device__ __forceinline__ int sum(int v) {
    const int w = warp_sum(v);
    if constexpr (WPC == 1) {
      return w;
    } else {
      int* buf = red + phase * WPC;
      phase ^= 1;
      if ((t & 31) == 0) buf[t >> 5] = w;
      sync();
      int s = 0;
#pragma unroll
      for (int i = 0; i < WPC; ++i) s += buf[i];
      return s;
    }
  }
};

// Direction histogram of centre (rx, cx) on the full signed table, by a team:
// slot k = t + 32 WPC j, j < kSlots, except skip0, skip1 and row rx; KEYED: the
// slots' table keys come from tm.key instead of the columns in cs.
template <int WPC, bool KEYED = false>
__device__ __forceinline__ int team_hist_build(const Team<WPC>& tm, const int* __restrict__ cs, int m, int rx, int cx,
                                               int skip0, int skip1, const uint16_t* __restrict__ lutf,
                                               uint32_t* __restrict__ hist, int (&ids)[Team<WPC>::kSlots]) {
  const uint16_t* base = lutf + kFullLutCentre - (rx * kLutW + cx);
  int pairs = 0;
#pragma unroll
  for (int j = 0; j < Team<WPC>::kSlots; ++j) {
    const int k = tm.t + Team<WPC>::kThreads * j;
    ids[j] = -1;
    if (k < m && k != skip0 && k != skip1 && (k >> 1) != rx) {
      const int id = base[KEYED ? tm.key[j] : (k >> 1) * kLutW + cs[k]];
      ids[j] = id;
      pairs += hist_add(hist, id);
    }
  }
  return pairs;
}

// tm.key from this thread's own slots of the state in cs (the thread reads
// only the slots it owns, so it needs no barrier after storing them itself).
template <int WPC>
__device__ __forceinline__ void team_load_keys(Team<WPC>& tm, const int* __restrict__ cs, int m) {
#pragma unroll
  for (int j = 0; j < Team<WPC>::kSlots; ++j) {
    const int k = tm.t + Team<WPC>::kThreads * j;
    tm.key[j] = k < m ? (k >> 1) * kLutW + cs[k] : 0;
  }
}

template <int WPC>
__device__ __forceinline__ void team_hist_release(uint32_t* hist, const int (&ids)[Team<WPC>::kSlots]) {
#pragma unroll
  for (int j = 0; j < Team<WPC>::kSlots; ++j)
    if (ids[j] >= 0) hist_clear(hist, ids[j]);
}

// EARLY (plain Metropolis only): after the first new-side histogram,
//   dE >= d1 = t(u') + j(u', v') - (bad[u] + bad[v] - joint)
// because t(v') >= 0, and thr is non-increasing, so a proposal with d1 >= 1 and
// (d1 >= W or z >= thr[d1]) is rejected exactly as the full test would reject
// it, without the second histogram; *dE_out then holds d1.
// KEYED: the histograms and the joint count take the slots' table keys from
// tm.key (see Team), and an accepted move updates them.
template <int WPC, bool FORCE, bool UMB = false, bool EARLY = false, bool KEYED = false>
__device__ __forceinline__ int team_move(Team<WPC>& tm, int* __restrict__ cs, int* __restrict__ bs, int m,
                                         const uint16_t* __restrict__ lutf, uint32_t* __restrict__ hist, int u, int v,
                                         uint32_t z, const uint32_t* __restrict__ thr, int W, int& E, uint32_t& err,
                                         int* dE_out, int64_t umb_q = 0, const uint32_t* __restrict__ frac = nullptr) {
  static_assert(!(EARLY && (FORCE || UMB)), "the early rejection needs the plain Metropolis test");
  constexpr int S = Team<WPC>::kSlots, TT = Team<WPC>::kThreads;
  const int ru = u >> 1, rv = v >> 1, cu = cs[u], cv = cs[v];
  int ids[S], cnt_new[S];
  // centre u' = (r_u, c_v)
  const int part_a = team_hist_build<WPC, KEYED>(tm, cs, m, ru, cv, u, v, lutf, hist, ids);
  tm.sync();
  const int line_new = dir_id_full(lutf, rv - ru, cu - cv);
  const int j_new = hist_get(hist, line_new);
  // points of A on the old line (u, v)
  int joint = 0;
#pragma unroll
  for (int j = 0; j < S; ++j) {
    const int k = tm.t + TT * j;
    if (k < m && k != u && k != v) {
      const int ck = KEYED ? tm.key[j] - (k >> 1) * kLutW : cs[k];
      joint += (rv - ru) * (ck - cu) == (cv - cu) * ((k >> 1) - ru);
    }
  }
  int t_a, sum_joint;
  if constexpr (EARLY) {
    const int s1 = tm.sum(part_a + (joint << 16));
    t_a = s1 & 0xFFFF;
    sum_joint = s1 >> 16;
    const int d1 = t_a + j_new - (bs[u] + bs[v] - sum_joint);
    if (d1 >= 1 && (d1 >= W || z >= thr[d1])) {
      tm.sync();
      team_hist_release<WPC>(hist, ids);
      tm.sync();
      *dE_out = d1;
      return 0;
    }
  }
#pragma unroll
  for (int j = 0; j < S; ++j) cnt_new[j] = ids[j] >= 0 ? hist_get(hist, ids[j]) - 1 + (ids[j] == line_new) : 0;
  tm.sync();
  team_hist_release<WPC>(hist, ids);
  tm.sync();
  // centre v' = (r_v, c_u)
  const int part_b = team_hist_build<WPC, KEYED>(tm, cs, m, rv, cu, u, v, lutf, hist, ids);
  tm.sync();
#pragma unroll
  for (int j = 0; j < S; ++j) cnt_new[j] += ids[j] >= 0 ? hist_get(hist, ids[j]) - 1 : 0;
  tm.sync();
  team_hist_release<WPC>(hist, ids);
  int t_b;
  if constexpr (EARLY) {
    t_b = tm.sum(part_b);
  } else {
    const int sum_ab = tm.sum(part_a + (part_b << 16));
    sum_joint = tm.sum(joint);
    t_a = sum_ab & 0xFFFF;
    t_b = sum_ab >> 16;
  }
  const int dE = (t_a + t_b + j_new) - (bs[u] + bs[v] - sum_joint);
  *dE_out = dE;
  const bool accept = FORCE || (UMB ? umbrella_accept(dE, umb_q, z, thr, W, frac)
                                     : (dE <= 0 || (dE < W && z < thr[dE])));
  if (!accept) {
    tm.sync();
    return 0;
  }
  // Old-side histograms: exact badness change of every other point.
  tm.sync();
  int dB[S];
  const int part_c = team_hist_build<WPC, KEYED>(tm, cs, m, ru, cu, u, v, lutf, hist, ids);
  tm.sync();
  const int line_old = dir_id_full(lutf, rv - ru, cv - cu);
  const int j_old = hist_get(hist, line_old);
#pragma unroll
  for (int j = 0; j < S; ++j)
    dB[j] = cnt_new[j] - (ids[j] >= 0 ? hist_get(hist, ids[j]) - 1 + (ids[j] == line_old) : 0);
  tm.sync();
  team_hist_release<WPC>(hist, ids);
  tm.sync();
  const int part_d = team_hist_build<WPC, KEYED>(tm, cs, m, rv, cv, u, v, lutf, hist, ids);
  tm.sync();
#pragma unroll
  for (int j = 0; j < S; ++j) dB[j] -= ids[j] >= 0 ? hist_get(hist, ids[j]) - 1 : 0;
  tm.sync();
  team_hist_release<WPC>(hist, ids);
  const int sum_cd = tm.sum(part_c + (part_d << 16));
  const int t_c = sum_cd & 0xFFFF, t_d = sum_cd >> 16;
  if (bs[u] != t_c + j_old || bs[v] != t_d + j_old || j_old != sum_joint) err |= kErrAudit;
  tm.sync();
#pragma unroll
  for (int j = 0; j < S; ++j) {
    const int k = tm.t + TT * j;
    if (k < m && k != u && k != v) bs[k] += dB[j];
    if (KEYED) tm.key[j] += k == u ? cv - cu : (k == v ? cu - cv : 0);
  }
  if (tm.t == 0) {
    bs[u] = t_a + j_new;
    bs[v] = t_b + j_new;
    cs[u] = cv;
    cs[v] = cu;
  }
  tm.sync();
  E += dE;
  return 1;
}

// Slot of a badness-weighted draw (tempering.py:52-54): the first slot whose
// running badness sum exceeds `target` (target < 3E = the sum of all badness),
// and at most m - 1.  Lane l sums slots 5l .. 5l + 4 (stride-5 shared-memory
// reads, no bank conflicts); one warp scan gives the running sums, and the
// slot is the number of running sums not above the target.
__device__ __forceinline__ int bias_pick(const int* __restrict__ bs, int m, uint32_t target, int lane) {
  const int s0 = lane * kSlotsPerLane;
  int val[kSlotsPerLane];
  int local = 0;
#pragma unroll
  for (int t = 0; t < kSlotsPerLane; ++t) {
    val[t] = s0 + t < m ? bs[s0 + t] : 0;
    local += val[t];
  }
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  int run = incl - local, cnt = 0;
#pragma unroll
  for (int t = 0; t < kSlotsPerLane; ++t) {
    run += val[t];
    cnt += (s0 + t < m && (uint32_t)run <= target) ? 1 : 0;
  }
  cnt = warp_sum(cnt);
  return cnt < m - 1 ? cnt : m - 1;
}

// Change of the umbrella distance `removed` (reference points missing from the
// state) when slot u takes column c_v and slot v takes c_u: the reference's
// distance_delta (tempering.py:59-63) over the reference state's rows.
__device__ __forceinline__ int umbrella_distance_delta(const int16_t* __restrict__ ref, int u, int v, int cu, int cv) {
  const int ur = u & ~1, vr = v & ~1;
  const int a0 = ref[ur], a1 = ref[ur + 1], b0 = ref[vr], b1 = ref[vr + 1];
  return (int)(cu == a0 || cu == a1) + (int)(cv == b0 || cv == b1) - (int)(cv == a0 || cv == a1) -
         (int)(cu == b0 || cu == b1);
}

// What a walk proposal needs beyond the chain's state.
struct WalkParams {
  int bad_bias;                  // percent of proposals with a badness-weighted u
  uint32_t k0, k1;               // Philox key
  const int16_t* ref;            // umbrella reference slot columns (UMB)
  const uint32_t* frac;          // fraction factors of this chain's temperature (UMB)
  int64_t s_q, c2s_q;            // round(2^24 s), round(2^24 * 2 s center) of this chain's position (UMB)
};

// One walk proposal (tempering.py:49-58): u uniform, or with probability
// bad_bias/100 drawn by badness (second Philox block, counter `ctr`, tag
// kTagBias); v uniform; legal iff E > 0 and no point is duplicated.  rnd is
// the proposal's Philox block: x -> u, y -> v, z the Metropolis uniform,
// w the bias coin.  With UMB the acceptance energy carries the umbrella
// restraint s((off + dd)^2 - off^2), off = removed - center (tempering.py:93-94),
// and an accepted move adds dd to `removed`.  Returns 1 if accepted.
template <int WPC, bool BIAS, bool UMB>
__device__ __forceinline__ int propose_walk(Team<WPC>& tm, int* __restrict__ cs, int* __restrict__ bs, int m,
                                            const uint16_t* __restrict__ lutf, uint32_t* __restrict__ hist, U4 rnd,
                                            uint64_t ctr, int chain, const uint32_t* __restrict__ thr, int W, int& E,
                                            uint32_t& err, const WalkParams& P, int& removed) {
  if (E <= 0) return 0;
  int u = (int)__umulhi(rnd.x, (unsigned)m);
  const int v = (int)__umulhi(rnd.y, (unsigned)m);
  if (BIAS && __umulhi(rnd.w, 100u) < (unsigned)P.bad_bias) {
    // every warp of the team draws the same slot from the same badness
    const U4 r2 = philox4x32_10(U4{(uint32_t)ctr, (uint32_t)(ctr >> 32), (uint32_t)chain, kTagBias}, P.k0, P.k1);
    u = bias_pick(bs, m, __umulhi(r2.x, 3u * (unsigned)E), tm.t & 31);
  }
  if (!legal_swap(cs, u, v)) return 0;
  int dE;
  if (!UMB)
    return team_move<WPC, false, false, true, true>(tm, cs, bs, m, lutf, hist, u, v, rnd.z, thr, W, E, err, &dE);
  const int dd = umbrella_distance_delta(P.ref, u, v, cs[u], cs[v]);
  const int64_t umb = P.s_q * (int64_t)(2 * removed * dd + dd * dd) - P.c2s_q * (int64_t)dd;
  const int acc = team_move<WPC, false, true, false, true>(tm, cs, bs, m, lutf, hist, u, v, rnd.z, thr, W, E, err,
                                                           &dE, umb, P.frac);
  if (acc) removed += dd;
  return acc;
}

}  // namespace n3
