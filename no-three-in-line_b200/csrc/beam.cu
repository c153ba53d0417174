// Device-resident beam search: the generation loop of
// src/no_three_75/gpu_device_search.py:254-432 (gpu_device_beam_search) on the
// GPU.  Per generation, five launches on one stream and no host round trip:
//   mutate_kernel      children from the ranked elites (gpu_device_search.py:27-114),
//                      recording each child's parent and swaps
//   child_delta_kernel E and badness of every child from its parent's by the exact
//                      delta of each swap (the reference rescores every child)
//   select_kernel      stable score order prefix, the children within the energy
//                      window in index order, their random.Random shuffle, the
//                      pick of elite_size children (gpu_device_search.py:343-373)
//   gather_kernel      the picked children's rows, E and badness
//   rank_kernel        rank_elites order (gpu_device_search.py:185-197) and the
//                      best-so-far update by elite_key (:200-203, :388-396)
// The reference does the selection and ranking on the host with a copy of
// every child's score each generation.  Here the selection is one CTA: a
// one-pass histogram (or radix) select of the elite_size-th smallest score, a
// bitonic sort of the scores below it, ordered compactions by per-warp counts,
// the MT19937 state blocks twisted by the whole CTA, the shuffle's draws
// (exactly CPython's: by the whole CTA for the wide draw widths, by one warp
// for the last ones), and the first elite_size shuffled positions traced back
// through the draws.
#include <stdint.h>

#include <climits>

#include "chain_move.cuh"
#include "dirs.cuh"
#include "pyrandom.cuh"
#include "n3_common.cuh"

namespace n3 {
namespace beam {

// --------------------------------------------------------------------------
// xorshift64* (Vigna), the reference's per-child RNG (gpu_device_search.py:18-25).
// --------------------------------------------------------------------------
__device__ __forceinline__ uint64_t xs64(uint64_t& s) {
  uint64_t x = s;
  x ^= x >> 12;
  x ^= x << 25;
  x ^= x >> 27;
  s = x;
  return x * 2685821657736338717ULL;
}

struct MutArgs {
  const int32_t* pp;
  const int32_t* pq;
  const int32_t* pbad;
  int parent_count, quality_count, active_strength;  // used when status == nullptr
  const int64_t* status;                              // beam status: counts and strength derive from it
  int elite_size, n, population, max_strength, bad_bias, generation;
  uint64_t seed;
  int32_t* cp;
  int32_t* cq;
  int32_t* child_parent;  // optional: each child's parent and swaps (u | v << 8), for the delta scoring
  int32_t* child_moves;
  int32_t* child_nmoves;
  int moves_cap;
  int prefix_cap;  // parents whose badness prefix sums the CTA stages in shared memory
};

// One thread per child, the reference's draws in the reference's order.  The
// CTA's 64 children live in shared memory (slot layout s = 2 * row + layer)
// from the parent copy to one coalesced write of their rows.  When the parents'
// badness prefix sums fit in shared memory (prefix_cap parents), the CTA builds
// them once and the roulette draw becomes a binary search: with no negative
// badness, the linear scan `t -= bad[u]` stops at the first u whose inclusive
// prefix exceeds t, which the search finds.  A negative badness anywhere, or
// one large enough for a sum to overflow (neither is a state's badness), sends
// the CTA back to the linear scan, so every draw and result stays the
// reference's for any input.  The parent's total badness is taken once per
// child instead of once per attempt (it does not change).
constexpr int kMutThreads = 64;
constexpr size_t kMutPrefixMaxBytes = 96 * 1024;

constexpr size_t kMutSmemMax = sizeof(int32_t) * kMutThreads * kMaxM + kMutPrefixMaxBytes;

__global__ void __launch_bounds__(kMutThreads) mutate_kernel(const MutArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_parent[kMutThreads];
  int parent_count = A.parent_count, quality_count = A.quality_count, active = A.active_strength;
  if (A.status != nullptr) {
    if (A.status[1] == 0) return;  // uniform: the search has reached E = 0
    parent_count = (int)A.status[0];
    quality_count = max(1, min(parent_count, A.elite_size / 4));
    active = min(A.max_strength, 2 + (A.generation - (int)A.status[4]) / 10);
  }
  const int n = A.n, m = 2 * n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int child0 = blockIdx.x * kMutThreads, child = child0 + tid;
  const int nc = min(kMutThreads, A.population - child0);
  int32_t* rows = reinterpret_cast<int32_t*>(smem);  // [kMutThreads][m]
  int32_t* prefix = rows + kMutThreads * m;          // [prefix_cap][m] inclusive prefix sums
  uint64_t rng = A.seed ^ (0x9e3779b97f4a7c15ULL * (uint64_t)(child + 1)) ^
                 (0xbf58476d1ce4e5b9ULL * (uint64_t)(A.generation + 1));
  int parent = child;
  if (child < A.population && child >= parent_count) {
    const uint64_t pick = xs64(rng);
    const int pool = (pick & 255ULL) < 160ULL ? quality_count : parent_count;
    parent = (int)(xs64(rng) % (uint64_t)pool);
  }
  s_parent[tid] = parent;
  bool use_prefix = parent_count <= A.prefix_cap;  // uniform
  if (use_prefix) {
    const int count = parent_count * m;
#pragma unroll 8
    for (int i = tid; i < count; i += kMutThreads) prefix[i] = A.pbad[i];  // coalesced, loads in flight together
    __syncthreads();
    bool negative = false;
    for (int p = tid; p < parent_count; p += kMutThreads) {  // in place, a thread per parent
      int32_t* row = prefix + p * m;
      int acc = 0;
#pragma unroll 10
      for (int e = 0; e < m; ++e) {
        const int b = row[e];
        negative |= b < 0 || b > 0x7fffffff / kMaxM;  // keeps every prefix sum below 2^31
        row[e] = acc += b;
      }
    }
    use_prefix = !__syncthreads_or(negative);
  } else {
    __syncthreads();
  }
  for (int c = warp; c < nc; c += kMutThreads / 32) {  // the parents' rows into the children's, a warp per child
    const int32_t* src_p = A.pp + (size_t)s_parent[c] * n;
    const int32_t* src_q = A.pq + (size_t)s_parent[c] * n;
    int32_t* dst = rows + c * m;
    for (int r = lane; r < n; r += 32) {
      dst[2 * r] = src_p[r];
      dst[2 * r + 1] = src_q[r];
    }
  }
  __syncthreads();
  const bool record = A.child_moves != nullptr;
  if (child < A.population) {
    if (record) A.child_parent[child] = parent;
    if (child < parent_count) {
      if (record) A.child_nmoves[child] = 0;
    } else {
      int32_t* cs = rows + tid * m;
      const int32_t* bad = A.pbad + (size_t)parent * m;
      const int32_t* pre = prefix + parent * m;
      int total = 0;
      if (use_prefix) {
        total = pre[m - 1];
      } else {
        for (int e = 0; e < m; ++e) total += bad[e];
      }
      int strength, nmoves = 0;
      if ((xs64(rng) & 31ULL) == 0ULL)
        strength = 1 + (int)(xs64(rng) % (uint64_t)A.max_strength);
      else
        strength = 1 + (int)(xs64(rng) % (uint64_t)active);
      for (int step = 0; step < strength; ++step) {
        for (int attempt = 0; attempt < 32; ++attempt) {
          int u;
          if ((int)(xs64(rng) % 100ULL) < A.bad_bias) {
            if (total) {
              const int t = (int)(xs64(rng) % (uint64_t)total);
              if (use_prefix) {  // first u with prefix[u] > t; prefix[m - 1] = total > t
                int lo = 0, hi = m - 1;
                while (lo < hi) {
                  const int mid = (lo + hi) >> 1;
                  if (pre[mid] > t) hi = mid;
                  else lo = mid + 1;
                }
                u = lo;
              } else {
                int r = t;
                for (u = 0; u < m - 1; ++u) {
                  r -= bad[u];
                  if (r < 0) break;
                }
              }
            } else {
              u = (int)(xs64(rng) % (uint64_t)m);
            }
          } else {
            u = (int)(xs64(rng) % (uint64_t)m);
          }
          const int v = (int)(xs64(rng) % (uint64_t)m);
          if ((u >> 1) == (v >> 1)) continue;
          const int cu = cs[u], cv = cs[v];
          if (cu == cv) continue;
          if (cv == cs[u ^ 1] || cu == cs[v ^ 1]) continue;  // the other point of each row
          cs[u] = cv;
          cs[v] = cu;
          if (record && nmoves < A.moves_cap) A.child_moves[(size_t)child * A.moves_cap + nmoves] = u | (v << 8);
          ++nmoves;
          break;
        }
      }
      if (record) A.child_nmoves[child] = nmoves;
    }
  }
  __syncthreads();
  for (int c = warp; c < nc; c += kMutThreads / 32) {  // coalesced rows, a warp per child
    const int32_t* src = rows + c * m;
    int32_t* dst_p = A.cp + (size_t)(child0 + c) * n;
    int32_t* dst_q = A.cq + (size_t)(child0 + c) * n;
    for (int r = lane; r < n; r += 32) {
      dst_p[r] = src[2 * r];
      dst_q[r] = src[2 * r + 1];
    }
  }
}

// --------------------------------------------------------------------------
// Children's scores by exact deltas: warp per child, the parent's columns and
// badness in shared memory, then each recorded swap applied with its exact dE
// and the exact update of every badness (team_move<1, true>: the tempering
// move by one warp, without the Metropolis test).  E and badness equal a full
// recount.
// --------------------------------------------------------------------------
constexpr int kDeltaWarps = 22;
constexpr size_t kDeltaSmem = kFullLutBytes + kDeltaWarps * (sizeof(uint32_t) * kDirWords + 2 * sizeof(int) * kMaxM);

struct DeltaArgs {
  const int32_t* ep;
  const int32_t* eq;
  const int32_t* ebad;
  const int32_t* es;
  const int32_t* parent;
  const int32_t* moves;
  const int32_t* nmoves;
  int moves_cap, n, population;
  const int64_t* status;
  const uint16_t* lutf;
  int32_t* scores;
  int32_t* badness;
  uint32_t* error_word;
};

__global__ void __launch_bounds__(kDeltaWarps * 32, 1) child_delta_kernel(const DeltaArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (A.status[1] == 0) return;  // uniform: the search has reached E = 0
  uint16_t* lutf = reinterpret_cast<uint16_t*>(smem);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + kFullLutBytes);
  int* cs_all = reinterpret_cast<int*>(hist_all + kDeltaWarps * kDirWords);
  int* bs_all = cs_all + kDeltaWarps * kMaxM;
  full_lut_copy(lutf, A.lutf);
  for (int i = threadIdx.x; i < kDeltaWarps * kDirWords / 4; i += blockDim.x)
    reinterpret_cast<uint4*>(hist_all)[i] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = A.n, m = 2 * n;
  int* cs = cs_all + warp * kMaxM;
  int* bs = bs_all + warp * kMaxM;
  uint32_t* hist = hist_all + warp * kDirWords;
  uint32_t err = 0;
  for (int c = blockIdx.x * kDeltaWarps + warp; c < A.population; c += gridDim.x * kDeltaWarps) {
    const int par = A.parent[c];
    for (int s = lane; s < m; s += 32) {
      cs[s] = (s & 1) ? A.eq[(size_t)par * n + (s >> 1)] : A.ep[(size_t)par * n + (s >> 1)];
      bs[s] = A.ebad[(size_t)par * m + s];
    }
    __syncwarp();
    Team<1> tm{lane, 0, nullptr, 0, {}};
    team_load_keys(tm, cs, m);  // the slots' table keys, kept in registers across the moves
    int E = A.es[par];
    const int k_end = min(A.nmoves[c], A.moves_cap);
    for (int k = 0; k < k_end; ++k) {
      const int mv = A.moves[(size_t)c * A.moves_cap + k];
      int dE;
      team_move<1, true, false, false, true>(tm, cs, bs, m, lutf, hist, mv & 0xFF, (mv >> 8) & 0xFF, 0u, nullptr, 0,
                                             E, err, &dE);
    }
    if (lane == 0) A.scores[c] = E;
    for (int s = lane; s < m; s += 32) A.badness[(size_t)c * m + s] = bs[s];
    __syncwarp();
  }
  if (lane == 0 && err && A.error_word) atomicOr(A.error_word, err);
}


__global__ void py_seed_kernel(uint32_t* state, uint64_t seed) {
  uint32_t* mt = state;
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const int len = (seed >> 32) ? 2 : 1;
  mt[0] = 19650218u;
  for (int i = 1; i < kMT; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
  int i = 1, j = 0;
  for (int k = kMT > len ? kMT : len; k; --k) {
    mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1664525u)) + key[j] + (uint32_t)j;
    ++i;
    ++j;
    if (i >= kMT) {
      mt[0] = mt[kMT - 1];
      i = 1;
    }
    if (j >= len) j = 0;
  }
  for (int k = kMT - 1; k; --k) {
    mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1566083941u)) - (uint32_t)i;
    ++i;
    if (i >= kMT) {
      mt[0] = mt[kMT - 1];
      i = 1;
    }
  }
  mt[0] = 0x80000000u;
  state[kMT] = kMT;  // position: the first draw twists
}

__global__ void py_shuffle_kernel(uint32_t* state, int32_t* values, int count) {
  __shared__ uint32_t mt[kMT], out[kMT], seen[65536 / 32];
  for (int i = threadIdx.x; i < kMT; i += blockDim.x) mt[i] = state[i];
  for (int i = threadIdx.x; i < 65536 / 32; i += blockDim.x) seen[i] = 0u;
  __syncthreads();
  if (threadIdx.x < 32) {
    int idx = (int)state[kMT];
    py_shuffle_warp(mt, out, idx, values, count, seen, threadIdx.x);
    if (threadIdx.x == 0) state[kMT] = (uint32_t)idx;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kMT; i += blockDim.x) state[i] = mt[i];
}

// The state twist by a whole CTA, out of place: dst = twist(src).  Word k of the
// sequential in-place update reads the old words k, k + 1 and k + 397 (k < 227)
// or the new word k - 227 (k >= 227; for k = 623 also the new word 0), so three
// phases of at most 227 words each reproduce it.  Every thread calls it.
__device__ __forceinline__ uint32_t mt_mix(uint32_t hi_word, uint32_t lo_word, uint32_t far) {
  const uint32_t y = (hi_word & 0x80000000u) | (lo_word & 0x7fffffffu);
  return far ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

__device__ void mt_twist_cta(const uint32_t* src, uint32_t* dst) {
  const int t = threadIdx.x;
  if (t < 227) dst[t] = mt_mix(src[t], src[t + 1], src[t + 397]);
  __syncthreads();
  if (t < 227) dst[227 + t] = mt_mix(src[227 + t], src[228 + t], dst[t]);
  __syncthreads();
  if (t < 170) {
    const int k = 454 + t;
    dst[k] = mt_mix(src[k], k == kMT - 1 ? dst[0] : src[k + 1], dst[k - 227]);
  }
  __syncthreads();
}

// The shuffle's draws by one warp from the tempered outputs out[0, avail)
// (consecutive blocks of the stream; out holds 32 more words, read and
// ignored), starting at output pos, for steps i, i - 1, ... >= 1: the j of
// step s goes to jstep[s] and no swap is made.  A round takes the next 32
// words: word l serves step i - A_l (A_l: accepted words before it), so with
// bounds A_lo <= A_l <= A_hi it is accepted for sure when r <= i - A_hi and
// rejected for sure when r > i - A_lo.  Ballots of the decided words give the
// bounds (A_lo: accepted below the lane; A_hi: the lane less the rejected
// below it), and the lowest undecided lane always has exact bounds, so a few
// iterations decide all 32.  The round keeps the words up to the m-th
// acceptance (m: the steps left in this draw width, at most 32).  Stops when
// the steps end or the outputs do; i and pos advance.
__device__ void shuffle_draws_warp(const uint32_t* out, int avail, int& pos, int& i, uint16_t* jstep, int lane) {
  const unsigned below = (1u << lane) - 1u;
  while (i >= 1 && pos < avail) {
    const int shift = __clz((uint32_t)i + 1u);
    const int lo = max(1, (int)(0x80000000u >> shift) - 1);  // the width's last step
    const int m = min(32, i - lo + 1);
    const int draws = min(32, avail - pos);
    const int r = (int)(out[pos + lane] >> shift);
    unsigned accm = 0u, rejm = draws < 32 ? ~0u << draws : 0u;  // lanes past the outputs: decided, unused
    for (;;) {
      const bool und = !(((accm | rejm) >> lane) & 1u);
      const int a_lo = __popc(accm & below), a_hi = lane - __popc(rejm & below);
      accm |= __ballot_sync(0xffffffffu, und && r <= i - a_hi);
      rejm |= __ballot_sync(0xffffffffu, und && r > i - a_lo);
      if ((accm | rejm) == 0xffffffffu) break;  // uniform
    }
    int used = draws;
    if (__popc(accm) >= m) {  // the m-th acceptance ends this width
      const int z = __ffs(__ballot_sync(0xffffffffu, ((accm >> lane) & 1u) &&
                                                      __popc(accm & ((2u << lane) - 1u)) == m)) - 1;
      used = z + 1;
    }
    const unsigned take = used < 32 ? accm & ((1u << used) - 1u) : accm;
    if ((take >> lane) & 1u) jstep[i - __popc(take & below)] = (uint16_t)r;
    i -= __popc(take);
    pos += used;
  }
}

// Exclusive scan over the CTA (thread order) of a 32-bit value, with the total.
// wsum: 32 words of shared memory; consecutive calls must alternate between
// two such buffers (a call's buffer is rewritten only after every thread has
// passed the next call's barriers).  blockDim.x == 1024.
__device__ __forceinline__ uint32_t cta_exscan32(uint32_t v, uint32_t* wsum, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    wsum[lane] = w;
  }
  __syncthreads();
  total = wsum[31];
  return (warp ? wsum[warp - 1] : 0u) + x - v;
}

// The shuffle's draws for the steps i, i - 1, ... that share i's draw width
// (down to 2^(k-1) - 1, k = bit_length(i + 1)), resolved by the whole CTA from
// the tempered outputs out[pos, avail), the same as shuffle_draws_warp: step s
// takes words in order until one has r = word >> (32 - k) <= s, and j = r.
// Word w (w = 0, 1, ... from pos) serves step i - A_w, A_w the number of
// accepted words before it, so it is accepted for sure when r <= i - A_hi and
// rejected for sure when r > i - A_lo, for any bounds A_lo <= A_w <= A_hi.
// Each pass bounds A_w by prefix counts over the CTA of the words decided so
// far (A_lo: accepted before w; A_hi: w less the rejected before w) and
// decides what the bounds allow; the first undecided word always has exact
// bounds, so a pass never ends without progress.  Thread t holds words
// kDrawPer t .. kDrawPer t + kDrawPer - 1.  After at most kDrawPasses passes
// the call stops at the first undecided word, or after the acceptance of the
// width's last step, or at the end of the outputs; i and pos advance.  All
// threads call it with the same i and pos (>= 1 step, >= 1 word left).  A
// call takes at most 2 need + 64 words (a draw is accepted with probability
// above 1/2): more words per call mean more passes, as a word's bounds widen
// with the number of words before it.
constexpr int kDrawPer = 5;       // 5120 words per call: one batch of kSelBatch blocks
constexpr int kDrawPasses = 48;
__device__ void shuffle_draws_cta(const uint32_t* out, int avail, int& pos, int& i, uint16_t* jstep,
                                  uint32_t* wsum /* [2][32] */, int* cut /* [3] */) {
  const int tid = threadIdx.x;
  const int shift = __clz((uint32_t)i + 1u);
  const int lo = max(1, (int)(0x80000000u >> shift) - 1);  // the width's last step
  const int need = i - lo + 1;
  const int nw = min(min(avail - pos, (int)blockDim.x * kDrawPer), 2 * need + 64);
  const int w0 = tid * kDrawPer;
  uint32_t r[kDrawPer];
  uint32_t st = 0u;  // 2 bits per word: 0 undecided, 1 accepted, 2 rejected, 3 absent
#pragma unroll
  for (int e = 0; e < kDrawPer; ++e) {
    const int w = w0 + e;
    r[e] = w < nw ? out[pos + w] >> shift : 0u;
    if (w >= nw) st |= 3u << (2 * e);
  }
  // scanned counts: accepted | rejected << 16 (at most 5120 each); undecided = words - both
  uint32_t before = 0u, total = 0u;
  int la = 0, lu = 0;
  for (int pass = 0; pass < kDrawPasses; ++pass) {
    int a = (int)(before & 0xFFFFu), rj = (int)(before >> 16);
    la = 0;
    lu = 0;
    int lr = 0;
#pragma unroll
    for (int e = 0; e < kDrawPer; ++e) {
      uint32_t d = (st >> (2 * e)) & 3u;
      if (d == 0u) {
        const int w = w0 + e;
        if ((int)r[e] <= i - (w - rj)) d = 1u;
        else if ((int)r[e] > i - a) d = 2u;
        st |= d << (2 * e);
      }
      if (d == 1u) { ++a; ++la; }
      else if (d == 2u) { ++rj; ++lr; }
      else if (d == 0u) ++lu;
    }
    before = cta_exscan32((uint32_t)la | ((uint32_t)lr << 16), wsum + 32 * (pass & 1), total);
    if ((int)(total & 0xFFFFu) + (int)(total >> 16) == nw) break;  // uniform: every word decided
  }
  // `before` counts exactly for the words before the first undecided one, F.
  if (tid == 0) {
    cut[0] = nw;       // F
    cut[1] = INT_MAX;  // the word after the need-th acceptance
  }
  __syncthreads();
  const int a0 = (int)(before & 0xFFFFu);
  // no undecided word before this thread's (words before it: min(w0, nw))
  const bool clean = a0 + (int)(before >> 16) == min(w0, nw);
  if (clean && lu > 0) {  // this thread holds F
    int acc = a0;
    for (int e = 0; e < kDrawPer; ++e) {
      const uint32_t d = (st >> (2 * e)) & 3u;
      if (d == 0u) {
        cut[0] = w0 + e;
        cut[2] = acc;  // acceptances before F
        break;
      }
      acc += d == 1u;
    }
  }
  if (a0 < need && a0 + la >= need) {  // this thread holds the need-th acceptance (exact if before F)
    int acc = a0;
    for (int e = 0; e < kDrawPer; ++e) {
      if (((st >> (2 * e)) & 3u) == 1u && ++acc == need) {
        cut[1] = w0 + e + 1;
        break;
      }
    }
  }
  __syncthreads();
  const int F = cut[0], cA = cut[1];
  const int used = min(F, cA);
  const int accepted = cA <= F ? need : (F == nw ? (int)(total & 0xFFFFu) : cut[2]);
  {
    int acc = a0;
#pragma unroll
    for (int e = 0; e < kDrawPer; ++e) {
      if (((st >> (2 * e)) & 3u) == 1u) {
        if (w0 + e < used) jstep[i - acc] = (uint16_t)r[e];
        ++acc;
      }
    }
  }
  i -= accepted;
  pos += used;
}

// --------------------------------------------------------------------------
// Selection (one CTA of kSelThreads threads).
// --------------------------------------------------------------------------
constexpr int kSelThreads = 1024;
constexpr int kMaxPopulation = 65536;
constexpr int kMaxElite = 2048;
constexpr int kSelBatch = 8;  // MT state blocks generated per batch for the shuffle's draws
constexpr int kCtaDrawMin = 2048;  // steps from which the CTA resolves the draws (below: one warp)
constexpr int kSelHistBins = 4096;  // one-pass selection when every score is below this
static_assert(kSelBatch * kMT <= kSelThreads * kDrawPer, "one resolver call covers a batch");
static_assert(kSelHistBins <= kSelBatch * kMT && kSelHistBins % 1024 == 0, "histogram in the MT words' space");

constexpr int kSelWarps = kSelThreads / 32;
static_assert(kSelWarps == 32, "the per-warp offsets are scanned by one warp, one lane per warp");

struct SelArgs {
  const int32_t* scores;  // [population]
  int population, elite_size, energy_window;
  int64_t* status;
  uint32_t* rng;          // [625]
  int32_t* selected;      // [elite_size]
};

// The draws of random.shuffle over `count` items (steps s = count - 1 .. 1,
// j_s = _randbelow(s + 1)) into jstep[s], from the state in shared memory (mt,
// the current block; idx the position in it, 624 when it is used up), with
// no swap made.  The CTA twists and tempers the state blocks kSelBatch at a
// time (words: kSelBatch blocks; out: their outputs and 32 words of padding);
// the CTA resolves the draws while many steps are left (shuffle_draws_cta) and
// warp 0 the last ones (shuffle_draws_warp).  On return mt and idx are the
// state CPython leaves: the block of the last draw and the position after it.
// Every thread calls it; idx is uniform.
__device__ void shuffle_steps_cta(uint32_t* mt, int& idx, int count, uint16_t* jstep, uint32_t* words, uint32_t* out,
                                  uint32_t* wsum, int* cut, int* s_misc) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int steps_left = count - 1;
  if (steps_left >= 1) {
    int pos = idx;
    if (pos < kMT) {
      for (int k = tid; k < kMT; k += blockDim.x) words[k] = mt[k];
      __syncthreads();
    } else {  // the current block is used up: the first draw twists
      mt_twist_cta(mt, words);
      pos = 0;
    }
    if (tid < 32) out[kSelBatch * kMT + tid] = 0u;  // the padding a last warp round reads
    for (;;) {
      for (int g = 1; g < kSelBatch; ++g) mt_twist_cta(words + (g - 1) * kMT, words + g * kMT);
      for (int k = tid; k < kSelBatch * kMT; k += blockDim.x) out[k] = mt_temper(words[k]);
      __syncthreads();
      while (steps_left >= kCtaDrawMin && pos < kSelBatch * kMT)
        shuffle_draws_cta(out, kSelBatch * kMT, pos, steps_left, jstep, wsum, cut);
      if (steps_left >= 1 && pos < kSelBatch * kMT) {  // uniform
        if (warp == 0) {
          shuffle_draws_warp(out, kSelBatch * kMT, pos, steps_left, jstep, lane);
          if (lane == 0) {
            s_misc[0] = steps_left;
            s_misc[1] = pos;
          }
        }
        __syncthreads();
        steps_left = s_misc[0];
        pos = s_misc[1];
        __syncthreads();
      }
      if (steps_left < 1) break;  // uniform
      mt_twist_cta(words + (kSelBatch - 1) * kMT, words);  // the next batch starts after the last block
      pos = 0;
    }
    const int last = pos - 1;  // >= 0: every round uses at least one word
    for (int k = tid; k < kMT; k += blockDim.x) mt[k] = words[(last / kMT) * kMT + k];
    idx = last % kMT + 1;
  }
  __syncthreads();
}

// Shuffled position p traced back through the steps after it: the item moves
// to step s wherever j_s equals its position (s > its current step).  The warp
// reads 256 steps at a time (8 packed 16-bit j per lane, compared two at a
// time); a chunk with a match is re-read after each move, in step order.
// jstep is 16-byte aligned and holds kMaxPopulation entries.
__device__ __forceinline__ int trace_position(const uint16_t* jstep, int p, int n_window, int lane) {
  int pos = p == 0 ? 0 : (int)jstep[p];
  int cur = p;  // the steps up to cur are behind the item
  const uint4* j8 = reinterpret_cast<const uint4*>(jstep);
  for (int b = (p + 1) & ~7; b < n_window; b += 256) {
    const int s0 = b + 8 * lane;
    const uint4 v = s0 < kMaxPopulation ? j8[s0 >> 3] : make_uint4(0u, 0u, 0u, 0u);
    for (;;) {
      const uint32_t pp = (uint32_t)pos * 0x10001u;
      const uint32_t e0 = __vcmpeq2(v.x, pp), e1 = __vcmpeq2(v.y, pp), e2 = __vcmpeq2(v.z, pp),
                     e3 = __vcmpeq2(v.w, pp);
      // bit h: step s0 + h has j == pos
      uint32_t hits = (e0 & 1u) | ((e0 >> 15) & 2u) | ((e1 & 1u) << 2) | ((e1 >> 13) & 8u) | ((e2 & 1u) << 4) |
                      ((e2 >> 11) & 32u) | ((e3 & 1u) << 6) | ((e3 >> 9) & 128u);
      // only steps after cur and inside the window count
      const int lo_h = cur + 1 - s0, hi_h = n_window - s0;  // valid h in [lo_h, hi_h)
      if (lo_h > 0) hits &= lo_h >= 8 ? 0u : ~((1u << lo_h) - 1u);
      if (hi_h < 8) hits &= hi_h <= 0 ? 0u : (1u << hi_h) - 1u;
      const unsigned any = __ballot_sync(0xffffffffu, hits != 0u);
      if (!any) break;  // uniform
      const int fl = __ffs(any) - 1;
      const uint32_t hm = __shfl_sync(0xffffffffu, hits, fl);
      cur = b + 8 * fl + __ffs(hm) - 1;
      pos = cur;
    }
  }
  return pos;
}

// Warp w owns the children [w * seg, (w + 1) * seg) (seg a multiple of 32) and
// reads them 32 at a time, so every pass over the scores is coalesced and every
// ordered compaction is a per-warp running count plus one scan over the warps.
__global__ void __launch_bounds__(kSelThreads, 1) select_kernel(const SelArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int P = A.population, E = A.elite_size, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const unsigned below = (1u << lane) - 1u;
  uint64_t* keys = reinterpret_cast<uint64_t*>(smem);                 // [kMaxElite]
  uint32_t* mt = reinterpret_cast<uint32_t*>(keys + kMaxElite);       // [624]
  int32_t* order = reinterpret_cast<int32_t*>(mt + kMT);              // [kMaxElite] score-order prefix
  uint32_t* mark = reinterpret_cast<uint32_t*>(order + kMaxElite);    // [kMaxPopulation / 32]
  uint32_t* words = mark + kMaxPopulation / 32;                        // [kSelBatch][624] untempered MT blocks
  uint32_t* tw = words + kSelBatch * kMT;                              // [kSelBatch * 624 + 32] their outputs
  uint16_t* jstep = reinterpret_cast<uint16_t*>(tw + kSelBatch * kMT + 32);  // [population] j of shuffle step s
  __shared__ uint32_t hist[256];
  __shared__ int tie_off[kSelWarps], win_off[kSelWarps];
  __shared__ int s_misc[4];
  __shared__ uint32_t draw_wsum[64];
  __shared__ int draw_cut[3];
  if (A.status[1] == 0) return;  // uniform: the search has reached E = 0
  const int64_t limit = A.status[1] + (int64_t)A.energy_window;
  for (int i = tid; i < kMaxPopulation / 32; i += kSelThreads) mark[i] = 0u;
  for (int i = tid; i < kMT; i += kSelThreads) mt[i] = A.rng[i];
  const int seg = (P + kSelThreads - 1) / kSelThreads * 32;
  const int s_lo = min(P, warp * seg), s_hi = min(P, s_lo + seg);
  if (tid == 0) s_misc[2] = 0;

  // 1. T = the E-th smallest score: radix select over the 32-bit scores, 8 bits
  //    a pass, from the highest byte that any score uses
  uint32_t top = 0u;
  for (int b = s_lo; b < s_hi; b += 32)
    if (b + lane < s_hi) top = max(top, (uint32_t)A.scores[b + lane]);
  top = __reduce_max_sync(0xffffffffu, top);
  if (lane == 0) hist[warp] = top;
  __syncthreads();
  if (warp == 0) {
    const uint32_t m = __reduce_max_sync(0xffffffffu, hist[lane]);
    if (lane == 0) s_misc[3] = (int)m;
  }
  __syncthreads();
  top = (uint32_t)s_misc[3];
  int shift = 24;
  while (shift > 0 && (top >> shift) == 0u) shift -= 8;  // the skipped high bytes are zero in every score
  uint32_t prefix = 0u, mask = 0u;
  int remaining = E;  // 1-based rank of the E-th element among those matching prefix
  if (top < (uint32_t)kSelHistBins) {
    // every score below 4096: one pass, one bin per score value (in the MT words'
    // space, free until the shuffle), then a scan over the bins
    uint32_t* h12 = words;
    for (int i = tid; i < kSelHistBins; i += kSelThreads) h12[i] = 0u;
    __syncthreads();
#pragma unroll 4
    for (int b = s_lo; b < s_hi; b += 32) {
      const int i = b + lane;
      const bool valid = i < s_hi;
      const uint32_t x = valid ? (uint32_t)A.scores[i] : 0u;
      const unsigned act = __ballot_sync(0xffffffffu, valid);
      if (valid) {
        const unsigned peers = __match_any_sync(act, x);
        if (lane == __ffs(peers) - 1) atomicAdd(&h12[x], (uint32_t)__popc(peers));
      }
    }
    __syncthreads();
    constexpr int kPerT = kSelHistBins / kSelThreads;
    uint32_t c[kPerT], local = 0u;
#pragma unroll
    for (int k = 0; k < kPerT; ++k) {
      c[k] = h12[kPerT * tid + k];
      local += c[k];
    }
    uint32_t tot;
    int run = (int)cta_exscan32(local, draw_wsum, tot);
    if (run < E && run + (int)local >= E) {  // this thread's bins hold the E-th smallest score
#pragma unroll
      for (int k = 0; k < kPerT; ++k) {
        if (run + (int)c[k] >= E) {
          s_misc[0] = kPerT * tid + k;
          s_misc[1] = E - run;
          break;
        }
        run += (int)c[k];
      }
    }
    __syncthreads();
    prefix = (uint32_t)s_misc[0];
    remaining = s_misc[1];
    shift = -8;  // done
    __syncthreads();
  }
  for (; shift >= 0; shift -= 8) {
    for (int i = tid; i < 256; i += kSelThreads) hist[i] = 0u;
    __syncthreads();
#pragma unroll 4
    for (int b = s_lo; b < s_hi; b += 32) {  // warp-uniform trip count; equal digits add once per warp
      const int i = b + lane;
      const uint32_t x = i < s_hi ? (uint32_t)A.scores[i] : 0u;
      const bool valid = i < s_hi && (x & mask) == prefix;
      const unsigned act = __ballot_sync(0xffffffffu, valid);
      if (valid) {
        const uint32_t digit = (x >> shift) & 255u;
        const unsigned peers = __match_any_sync(act, digit);
        if (lane == __ffs(peers) - 1) atomicAdd(&hist[digit], (uint32_t)__popc(peers));
      }
    }
    __syncthreads();
    if (tid == 0) {
      int before = 0, d = 0;
      for (; d < 255; ++d) {
        if (before + (int)hist[d] >= remaining) break;
        before += (int)hist[d];
      }
      s_misc[0] = d;
      s_misc[1] = remaining - before;
    }
    __syncthreads();
    prefix |= (uint32_t)s_misc[0] << shift;
    mask |= 255u << shift;
    remaining = s_misc[1];
    __syncthreads();
  }
  const uint32_t T = prefix;
  const int n_less = E - remaining;  // scores below T; then `remaining` ties at T by index

  // 2. one pass: the keys below T (at most E - 1), and per warp the ties at T
  //    and the children within the energy window
  int c_tie = 0, c_win = 0;
#pragma unroll 4
  for (int b = s_lo; b < s_hi; b += 32) {
    const int i = b + lane;
    const int x = i < s_hi ? A.scores[i] : 0;
    const unsigned lt = __ballot_sync(0xffffffffu, i < s_hi && (uint32_t)x < T);
    if (lt) {
      int at = 0;
      if (lane == 0) at = atomicAdd(&s_misc[2], __popc(lt));
      at = __shfl_sync(0xffffffffu, at, 0);
      if ((lt >> lane) & 1u) keys[at + __popc(lt & below)] = ((uint64_t)(uint32_t)x << 32) | (uint32_t)i;
    }
    c_tie += __popc(__ballot_sync(0xffffffffu, i < s_hi && (uint32_t)x == T));
    c_win += __popc(__ballot_sync(0xffffffffu, i < s_hi && (int64_t)x <= limit));
  }
  if (lane == 0) {
    tie_off[warp] = c_tie;
    win_off[warp] = c_win;
  }
  __syncthreads();
  if (warp == 0) {  // exclusive scans over the warps
    int t = tie_off[lane], w = win_off[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int yt = __shfl_up_sync(0xffffffffu, t, o), yw = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) {
        t += yt;
        w += yw;
      }
    }
    tie_off[lane] = t - tie_off[lane];
    if (lane == 31) s_misc[0] = w;  // the window's size
    win_off[lane] = w - win_off[lane];
  }
  int width = 1;
  while (width < n_less) width <<= 1;
  for (int i = n_less + tid; i < width; i += kSelThreads) keys[i] = ~0ull;
  __syncthreads();
  const int n_window = s_misc[0];

  // 3. the first `remaining` ties at T in index order; the keys below T sorted
  //    by (score, index) with a bitonic sort
  {
    int o = tie_off[warp];
    for (int b = s_lo; b < s_hi && o < remaining; b += 32) {
      const int i = b + lane;
      const unsigned m = __ballot_sync(0xffffffffu, i < s_hi && (uint32_t)A.scores[i] == T);
      if ((m >> lane) & 1u) {
        const int r = o + __popc(m & below);
        if (r < remaining) order[n_less + r] = i;
      }
      o += __popc(m);
    }
  }
  for (int size = 2; size <= width; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < width; i += kSelThreads) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const uint64_t a = keys[i], b = keys[j];
          if ((a > b) == up) {
            keys[i] = b;
            keys[j] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < n_less; i += kSelThreads) order[i] = (int32_t)(uint32_t)keys[i];

  // 4. the draws of the window list's shuffle (gpu_device_search.py:340-373):
  //    the j of every step s in jstep[s], no swap made (shuffle_steps_cta).
  {
    int idx = (int)A.rng[kMT];  // uniform
    shuffle_steps_cta(mt, idx, n_window, jstep, words, tw, draw_wsum, draw_cut, s_misc);
    if (tid == 0) A.rng[kMT] = (uint32_t)idx;
  }

  // 5. the first K = min(E, window) shuffled positions, one warp each.  Step s
  //    fixes position s for good, so position p holds what sat at j_p before
  //    step p; going back through the later steps p+1, p+2, ... (applied before
  //    it), the item moves only where a step's j equals its position, to that
  //    step.  The window position found is then mapped to its child through
  //    the per-warp window offsets.
  const int K = min(E, n_window);
  int32_t* picked = reinterpret_cast<int32_t*>(keys);  // [K]; keys is free once order is written
  for (int p = warp; p < K; p += kSelWarps) {
    const int pos = trace_position(jstep, p, n_window, lane);
    const unsigned owners = __ballot_sync(0xffffffffu, win_off[lane] <= pos);  // bit 0 always set
    const int w = 31 - __clz(owners);
    int rank = pos - win_off[w];
    const int w_lo = min(P, w * seg), w_hi = min(P, w_lo + seg);
    int child = -1;
    for (int b = w_lo; b < w_hi; b += 32) {
      const int i = b + lane;
      const unsigned m = __ballot_sync(0xffffffffu, i < w_hi && (int64_t)A.scores[i] <= limit);
      const int c = __popc(m);
      if (rank < c) {  // uniform
        const unsigned hitl = __ballot_sync(0xffffffffu, ((m >> lane) & 1u) && __popc(m & below) == rank);
        child = b + __ffs(hitl) - 1;
        break;
      }
      rank -= c;
    }
    if (lane == 0) picked[p] = child;
  }
  __syncthreads();

  // 6. thread 0: the pick (gpu_device_search.py:340-373)
  if (tid == 0) {
    int sel = 0;
    const int quality_keep = max(1, E / 4);
    for (int r = 0; r < quality_keep; ++r) {
      const int c = order[r];
      mark[c >> 5] |= 1u << (c & 31);
      A.selected[sel++] = c;
    }
    for (int k = 0; k < K && sel < E; ++k) {
      const int c = picked[k];
      if (c >= 0 && !(mark[c >> 5] & (1u << (c & 31)))) {
        mark[c >> 5] |= 1u << (c & 31);
        A.selected[sel++] = c;
      }
    }
    for (int r = 0; r < E && sel < E; ++r) {
      const int c = order[r];
      if (!(mark[c >> 5] & (1u << (c & 31)))) {
        mark[c >> 5] |= 1u << (c & 31);
        A.selected[sel++] = c;
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < kMT; i += kSelThreads) A.rng[i] = mt[i];
}

// The shuffle's draws alone (shuffle_steps_cta), for callers that apply the
// permutation themselves and for tests: j of step s in jout[s], jout[0] = 0.
constexpr size_t kStepsSmem = sizeof(uint32_t) * (kMT + 2 * kSelBatch * kMT + 32) + sizeof(uint16_t) * kMaxPopulation;
__global__ void __launch_bounds__(kSelThreads, 1) py_steps_kernel(uint32_t* state, int count, int32_t* jout) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* mt = reinterpret_cast<uint32_t*>(smem);
  uint32_t* words = mt + kMT;
  uint32_t* out = words + kSelBatch * kMT;
  uint16_t* jstep = reinterpret_cast<uint16_t*>(out + kSelBatch * kMT + 32);
  __shared__ uint32_t wsum[64];
  __shared__ int cut[3], s_misc[4];
  for (int i = threadIdx.x; i < kMT; i += blockDim.x) mt[i] = state[i];
  __syncthreads();
  int idx = (int)state[kMT];
  shuffle_steps_cta(mt, idx, count, jstep, words, out, wsum, cut, s_misc);
  for (int s = threadIdx.x; s < count; s += blockDim.x) jout[s] = s == 0 ? 0 : (int32_t)jstep[s];
  for (int i = threadIdx.x; i < kMT; i += blockDim.x) state[i] = mt[i];
  if (threadIdx.x == 0) state[kMT] = (uint32_t)idx;
}

constexpr size_t kSelSmem = sizeof(uint64_t) * kMaxElite + sizeof(uint32_t) * kMT + sizeof(int32_t) * kMaxElite +
                            sizeof(uint32_t) * (kMaxPopulation / 32) + sizeof(uint32_t) * (2 * kSelBatch * kMT + 32) +
                            sizeof(uint16_t) * kMaxPopulation;
static_assert(kSelSmem <= 227 * 1024 - 2048, "select_kernel shared memory");

// pick rows r = child rows selected[r]
__global__ void gather_kernel(const int32_t* __restrict__ cp, const int32_t* __restrict__ cq,
                              const int32_t* __restrict__ cs, const int32_t* __restrict__ cbad,
                              const int32_t* __restrict__ selected, int n, const int64_t* status, int32_t* pp,
                              int32_t* pq, int32_t* ps, int32_t* pbad) {
  if (status[1] == 0) return;
  const int r = blockIdx.x, c = selected[r];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    pp[(size_t)r * n + i] = cp[(size_t)c * n + i];
    pq[(size_t)r * n + i] = cq[(size_t)c * n + i];
  }
  for (int i = threadIdx.x; i < 2 * n; i += blockDim.x) pbad[(size_t)r * 2 * n + i] = cbad[(size_t)c * 2 * n + i];
  if (threadIdx.x == 0) ps[r] = cs[c];
}

// --------------------------------------------------------------------------
// Ranking (one CTA): rank_elites (gpu_device_search.py:185-197) is a stable
// sort by elite_key = (E, max badness, sum of squared badness); each element's
// rank is the number of keys before it.  Then the best-so-far update
// (gpu_device_search.py:388-396; set-up: :305-310).
// --------------------------------------------------------------------------
constexpr int kRankThreads = 1024;

struct RankArgs {
  const int32_t* pp;
  const int32_t* pq;
  const int32_t* pbad;
  const int32_t* ps;
  int count;       // picks to rank (set-up: the base count; a generation: elite_size)
  int n, generation;
  int32_t* ep;
  int32_t* eq;
  int32_t* ebad;
  int32_t* es;
  int64_t* status;
  int32_t* best_p;
  int32_t* best_q;
  int32_t* history;
  int history_len;
};

__global__ void __launch_bounds__(kRankThreads, 1) rank_kernel(const RankArgs A) {
  __shared__ int32_t s_score[kMaxElite], s_max[kMaxElite], s_rank[kMaxElite];
  __shared__ int64_t s_ss[kMaxElite];
  __shared__ int s_first, s_improved;
  if (A.generation > 0 && A.status[1] == 0) return;  // uniform
  const int C = A.count, m = 2 * A.n, tid = threadIdx.x;
  for (int i = tid; i < C; i += kRankThreads) {
    int mx = INT32_MIN;
    int64_t ss = 0;
    for (int s = 0; s < m; ++s) {
      const int b = A.pbad[(size_t)i * m + s];
      mx = max(mx, b);
      ss += (int64_t)b * b;
    }
    s_score[i] = A.ps[i];
    s_max[i] = mx;
    s_ss[i] = ss;
  }
  __syncthreads();
  for (int i = tid; i < C; i += kRankThreads) {
    const int a0 = s_score[i], a1 = s_max[i];
    const int64_t a2 = s_ss[i];
    int r = 0;
    for (int j = 0; j < C; ++j) {
      const int b0 = s_score[j], b1 = s_max[j];
      const int64_t b2 = s_ss[j];
      const bool less = b0 < a0 || (b0 == a0 && (b1 < a1 || (b1 == a1 && (b2 < a2 || (b2 == a2 && j < i)))));
      r += less;
    }
    s_rank[i] = r;
    if (r == 0) s_first = i;
  }
  __syncthreads();
  for (int e = tid; e < C * A.n; e += kRankThreads) {
    const int i = e / A.n, k = e % A.n;
    A.ep[(size_t)s_rank[i] * A.n + k] = A.pp[e];
    A.eq[(size_t)s_rank[i] * A.n + k] = A.pq[e];
  }
  for (int e = tid; e < C * m; e += kRankThreads) {
    const int i = e / m, k = e % m;
    A.ebad[(size_t)s_rank[i] * m + k] = A.pbad[e];
  }
  for (int i = tid; i < C; i += kRankThreads) A.es[s_rank[i]] = s_score[i];
  if (tid == 0) {
    const int f = s_first;
    const int64_t k0 = s_score[f], k1 = s_max[f], k2 = s_ss[f];
    int64_t* st = A.status;
    const bool improved = A.generation == 0 || k0 < st[1] || (k0 == st[1] && (k1 < st[2] || (k1 == st[2] && k2 < st[3])));
    if (improved) {
      st[1] = k0;
      st[2] = k1;
      st[3] = k2;
      if (A.generation > 0) st[4] = A.generation;
    }
    st[0] = C;
    if (A.generation == 0) st[4] = 0;
    st[5] = A.generation;
    st[6] = k0;
    st[7] = improved && A.generation > 0;
    if (A.history != nullptr && A.generation >= 1 && A.generation <= A.history_len) {
      A.history[2 * (A.generation - 1)] = (int32_t)k0;
      A.history[2 * (A.generation - 1) + 1] = (int32_t)st[1];
    }
    s_improved = improved;
  }
  __syncthreads();
  if (s_improved) {
    const int f = s_first;
    for (int k = tid; k < A.n; k += kRankThreads) {
      A.best_p[k] = A.pp[(size_t)f * A.n + k];
      A.best_q[k] = A.pq[(size_t)f * A.n + k];
    }
  }
}

}  // namespace beam
}  // namespace n3

namespace n3host {

// mutate_kernel over `population` children; the parents' prefix sums are staged
// when at most `parents_bound` parents fit in kMutPrefixMaxBytes.
static int launch_mutate(n3::beam::MutArgs A, int parents_bound, cudaStream_t st) {
  using namespace n3::beam;
  const int m = 2 * A.n;
  const int cap = (int)(kMutPrefixMaxBytes / (sizeof(int32_t) * (size_t)m));
  A.prefix_cap = parents_bound <= cap ? parents_bound : 0;
  const size_t bytes = sizeof(int32_t) * (size_t)m * (kMutThreads + A.prefix_cap);
  N3_TRY(allow_smem(reinterpret_cast<const void*>(mutate_kernel), kMutSmemMax));
  mutate_kernel<<<(A.population + kMutThreads - 1) / kMutThreads, kMutThreads, bytes, st>>>(A);
  return check_launch("beam mutate_kernel");
}

static int check_beam(const n3_beam* b) {
  if (b == nullptr) return set_error(N3_ERR_ARG, "null beam descriptor");
  if (b->n < 3 || b->n > N3_MAX_N) return set_error(N3_ERR_RANGE, "beam: n must lie in [3, %d]", N3_MAX_N);
  if (b->elite_size < 2 || b->elite_size > n3::beam::kMaxElite)
    return set_error(N3_ERR_RANGE, "beam: elite_size must lie in [2, %d]", n3::beam::kMaxElite);
  if (b->population < b->elite_size || b->population > n3::beam::kMaxPopulation)
    return set_error(N3_ERR_RANGE, "beam: population must lie in [elite_size, %d]", n3::beam::kMaxPopulation);
  if (b->max_strength < 1 || b->max_strength > 4096)
    return set_error(N3_ERR_RANGE, "beam: max_strength must lie in [1, 4096]");
  if (b->bad_bias < 0 || b->bad_bias > 100) return set_error(N3_ERR_RANGE, "beam: bad_bias must lie in [0, 100]");
  if (b->energy_window < 0) return set_error(N3_ERR_RANGE, "beam: energy_window must be non-negative");
  const void* ptrs[] = {b->elite_p, b->elite_q, b->elite_badness, b->elite_scores, b->child_p, b->child_q,
                        b->child_scores, b->pick_p, b->pick_q, b->pick_badness, b->pick_scores, b->selected,
                        b->rng, b->status, b->best_p, b->best_q, b->child_parent, b->child_moves,
                        b->child_nmoves, b->child_badness};
  for (const void* p : ptrs)
    if (p == nullptr) return set_error(N3_ERR_ARG, "beam: null buffer");
  return N3_OK;
}

static n3::beam::RankArgs rank_args(const n3_beam* b, int count, int generation) {
  n3::beam::RankArgs R;
  R.pp = b->pick_p;
  R.pq = b->pick_q;
  R.pbad = b->pick_badness;
  R.ps = b->pick_scores;
  R.count = count;
  R.n = b->n;
  R.generation = generation;
  R.ep = b->elite_p;
  R.eq = b->elite_q;
  R.ebad = b->elite_badness;
  R.es = b->elite_scores;
  R.status = b->status;
  R.best_p = b->best_p;
  R.best_q = b->best_q;
  R.history = b->history;
  R.history_len = b->history_len;
  return R;
}

}  // namespace n3host

extern "C" {

int n3_beam_mutate(const int32_t* parent_p, const int32_t* parent_q, const int32_t* parent_badness,
                   int parent_count, int quality_count, int n, int population, int active_strength,
                   int max_strength, int bad_bias, uint64_t seed, int generation, int32_t* child_p,
                   int32_t* child_q, void* stream) {
  if (!parent_p || !parent_q || !parent_badness || !child_p || !child_q)
    return n3host::set_error(N3_ERR_ARG, "beam mutate: null buffer");
  if (n < 2 || n > N3_MAX_N || parent_count < 1 || population < 0 || quality_count < 1 ||
      quality_count > parent_count || active_strength < 1 || max_strength < 1 || bad_bias < 0 || bad_bias > 100)
    return n3host::set_error(N3_ERR_RANGE, "beam mutate: argument out of range");
  if (population == 0) return N3_OK;
  n3::beam::MutArgs A;
  A.pp = parent_p;
  A.pq = parent_q;
  A.pbad = parent_badness;
  A.parent_count = parent_count;
  A.quality_count = quality_count;
  A.active_strength = active_strength;
  A.status = nullptr;
  A.elite_size = parent_count;
  A.n = n;
  A.population = population;
  A.max_strength = max_strength;
  A.bad_bias = bad_bias;
  A.generation = generation;
  A.seed = seed;
  A.cp = child_p;
  A.cq = child_q;
  A.child_parent = A.child_moves = A.child_nmoves = nullptr;
  A.moves_cap = 0;
  return n3host::launch_mutate(A, parent_count, (cudaStream_t)stream);
}

int n3_py_random_seed(uint32_t* state, uint64_t seed, void* stream) {
  if (!state) return n3host::set_error(N3_ERR_ARG, "null RNG state");
  n3::beam::py_seed_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(state, seed);
  return n3host::check_launch("py_seed_kernel");
}

int n3_py_random_shuffle(uint32_t* state, int32_t* values, int count, void* stream) {
  if (!state || (!values && count > 0)) return n3host::set_error(N3_ERR_ARG, "null shuffle buffer");
  if (count < 0 || count > n3::beam::kMaxPopulation) return n3host::set_error(N3_ERR_RANGE, "shuffle: bad count");
  n3::beam::py_shuffle_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(state, values, count);
  return n3host::check_launch("py_shuffle_kernel");
}

int n3_py_shuffle_steps(uint32_t* state, int count, int32_t* steps_j, void* stream) {
  if (!state || (!steps_j && count > 0)) return n3host::set_error(N3_ERR_ARG, "null shuffle-steps buffer");
  if (count < 0 || count > n3::beam::kMaxPopulation)
    return n3host::set_error(N3_ERR_RANGE, "shuffle steps: count %d outside [0, %d]", count, n3::beam::kMaxPopulation);
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(n3::beam::py_steps_kernel), n3::beam::kStepsSmem));
  n3::beam::py_steps_kernel<<<1, n3::beam::kSelThreads, n3::beam::kStepsSmem, (cudaStream_t)stream>>>(state, count,
                                                                                                      steps_j);
  return n3host::check_launch("py_steps_kernel");
}

int n3_beam_init(const n3_beam* b, int base_count, void* stream) {
  N3_TRY(n3host::check_beam(b));
  if (base_count < 1 || base_count > b->elite_size) return n3host::set_error(N3_ERR_RANGE, "beam: bad base count");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t rows = sizeof(int32_t) * (size_t)base_count * b->n;
  if (cudaMemcpyAsync(b->pick_p, b->elite_p, rows, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(b->pick_q, b->elite_q, rows, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return n3host::set_error(N3_ERR_CUDA, "beam init: copy failed");
  N3_TRY(n3_score_population(b->pick_p, b->pick_q, base_count, b->n, b->pick_scores, b->pick_badness, stream));
  n3::beam::rank_kernel<<<1, n3::beam::kRankThreads, 0, st>>>(n3host::rank_args(b, base_count, 0));
  N3_TRY(n3host::check_launch("beam rank_kernel"));
  return n3_py_random_seed(b->rng, b->seed, stream);
}

int n3_beam_generation(const n3_beam* b, int generation, void* stream) {
  N3_TRY(n3host::check_beam(b));
  if (generation < 1) return n3host::set_error(N3_ERR_RANGE, "beam: generations count from 1");
  cudaStream_t st = (cudaStream_t)stream;
  n3::beam::MutArgs M;
  M.pp = b->elite_p;
  M.pq = b->elite_q;
  M.pbad = b->elite_badness;
  M.parent_count = M.quality_count = M.active_strength = 0;
  M.status = b->status;
  M.elite_size = b->elite_size;
  M.n = b->n;
  M.population = b->population;
  M.max_strength = b->max_strength;
  M.bad_bias = b->bad_bias;
  M.generation = generation;
  M.seed = b->seed;
  M.cp = b->child_p;
  M.cq = b->child_q;
  M.child_parent = b->child_parent;
  M.child_moves = b->child_moves;
  M.child_nmoves = b->child_nmoves;
  M.moves_cap = b->max_strength;
  N3_TRY(n3host::launch_mutate(M, b->elite_size, st));
  N3_TRY(n3host::ensure_device_tables());
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(n3::beam::child_delta_kernel), n3::beam::kDeltaSmem));
  n3::beam::DeltaArgs D;
  D.ep = b->elite_p;
  D.eq = b->elite_q;
  D.ebad = b->elite_badness;
  D.es = b->elite_scores;
  D.parent = b->child_parent;
  D.moves = b->child_moves;
  D.nmoves = b->child_nmoves;
  D.moves_cap = b->max_strength;
  D.n = b->n;
  D.population = b->population;
  D.status = b->status;
  D.lutf = n3host::dir_lut_full_device_ptr();
  D.scores = b->child_scores;
  D.badness = b->child_badness;
  D.error_word = b->error_word;
  const int dgrid = (b->population + n3::beam::kDeltaWarps - 1) / n3::beam::kDeltaWarps;
  n3::beam::child_delta_kernel<<<dgrid < n3host::sm_count() ? dgrid : n3host::sm_count(), n3::beam::kDeltaWarps * 32,
                                 n3::beam::kDeltaSmem, st>>>(D);
  N3_TRY(n3host::check_launch("beam child_delta_kernel"));
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(n3::beam::select_kernel), n3::beam::kSelSmem));
  n3::beam::SelArgs S;
  S.scores = b->child_scores;
  S.population = b->population;
  S.elite_size = b->elite_size;
  S.energy_window = b->energy_window;
  S.status = b->status;
  S.rng = b->rng;
  S.selected = b->selected;
  n3::beam::select_kernel<<<1, n3::beam::kSelThreads, n3::beam::kSelSmem, st>>>(S);
  N3_TRY(n3host::check_launch("beam select_kernel"));
  n3::beam::gather_kernel<<<b->elite_size, 128, 0, st>>>(b->child_p, b->child_q, b->child_scores, b->child_badness,
                                                          b->selected, b->n, b->status, b->pick_p, b->pick_q,
                                                          b->pick_scores, b->pick_badness);
  N3_TRY(n3host::check_launch("beam gather_kernel"));
  n3::beam::rank_kernel<<<1, n3::beam::kRankThreads, 0, st>>>(n3host::rank_args(b, b->elite_size, generation));
  return n3host::check_launch("beam rank_kernel");
}

}  // extern "C"
