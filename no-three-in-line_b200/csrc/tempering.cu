// (c) Replica-exchange tempering: one persistent kernel over thousands of
// chains, ladders of neighbouring temperatures exchanged on the device.
//
// Reference: the per-replica walk kernel and host-side exchange of
// src/no_three_75/tempering.py:29-191.  Layout and scheduling here:
//
// * One team of WPC warps per chain (WPC = threads_per_chain / 32: 1, 2, 4, 8;
//   the team shares the chain's histogram and splits its slots).  A CTA
//   holds `cpb` chains (cpb * WPC <= 16 warps).  A ladder of L
//   temperatures lives either inside one CTA (cpb a multiple of L) or across a
//   thread-block cluster of L / cpb CTAs; its exchange step uses the CTA
//   barrier or the cluster barrier and distributed shared memory, never a
//   global spin-wait.
// * Every chain keeps its columns and badness in shared memory and proposes
//   row-pair column swaps (slots u, v from Philox4x32-10 with counter
//   (proposal index, chain), key = seed; u badness-weighted for bad_bias
//   percent of proposals, tempering.py:50-55).  An optional umbrella restraint
//   on the distance to a reference state enters the acceptance energy in
//   2^-24 fixed point (tempering.py:59-63, 93-94).  The exact dE uses the maintained
//   badness for the old side (the reference identity bad[u]+bad[v]-joint,
//   accelerated.py:78) and two direction histograms for the new side; an
//   accepted move rebuilds the old-side histograms to update every point's
//   badness exactly and checks the old side against the maintained badness.
// * Metropolis acceptance compares a 32-bit uniform with a per-temperature
//   integer threshold table floor(2^32 exp(-dE/T)) built on the host, so the
//   CPU oracle replays every chain bit for bit.  Exchanges swap temperature
//   labels (not states) between neighbours with the reference's rule
//   (tempering.py:178-184, even/odd alternation), thresholds likewise tabled.
// * Results depend only on the seed, the chain index and the round structure,
//   not on cpb or on how rounds are split over launches.
#include <cooperative_groups.h>

#include "dirs.cuh"
#include "n3_common.cuh"
#include "philox.cuh"
#include "chain_move.cuh"
#include "score_impl.cuh"

namespace cg = cooperative_groups;

namespace n3 {

struct TemperArgs {
  n3_chains ch;
  n3_temper_config cfg;
  const uint16_t* lut;  // full signed direction table (device)
  int cluster;          // CTAs per ladder (1: whole ladders per CTA)
};

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Shared-memory layout of the tempering kernel (dynamic): the full direction
// table, then per chain a histogram, columns and badness, then the leader
// arrays, then the teams' reduction scratch (2 WPC ints per chain).
constexpr int kTeamScratch = 2 * 16;
struct TemperSmem {
  static constexpr size_t lut_bytes = kFullLutBytes;
  static __host__ __device__ size_t bytes(int cpb) {
    return lut_bytes + (size_t)cpb * (sizeof(uint32_t) * kDirWords + 2 * sizeof(int) * kMaxM) +
           3 * sizeof(int) * 64 + 16 + sizeof(int) * kTeamScratch;
  }
};

// Exchange step of one ladder (run by its leader thread).  tmp_chain[t] is the
// ladder-local chain at temperature t, tmp_temp[i] the temperature of chain i,
// e[i] the energy of chain i.
__device__ void exchange_ladder(int* tmp_chain, int* tmp_temp, const int* e, int L, int ladder, uint32_t round,
                                const uint32_t* __restrict__ xthr, int XW, uint32_t k0, uint32_t k1,
                                uint32_t& accepted) {
  for (int t = (int)(round & 1u); t < L - 1; t += 2) {
    const int a = tmp_chain[t], b = tmp_chain[t + 1];
    const int D = e[a] - e[b];  // chain a holds the lower temperature
    bool swap = D >= 0;
    if (!swap) {
      const U4 r = philox4x32_10(U4{round, (uint32_t)t, (uint32_t)ladder, kTagExchange}, k0, k1);
      const int d = -D;
      swap = d < XW && r.x < xthr[(size_t)t * XW + d];
    }
    if (swap) {
      tmp_chain[t] = b;
      tmp_chain[t + 1] = a;
      tmp_temp[a] = t + 1;
      tmp_temp[b] = t;
      ++accepted;
    }
  }
}

template <int WPC, bool BIAS, bool UMB>
__global__ void __launch_bounds__(512, 1) temper_kernel(const TemperArgs A) {
  constexpr int TT = Team<WPC>::kThreads;
  extern __shared__ __align__(16) unsigned char smem[];
  const n3_chains& ch = A.ch;
  const n3_temper_config& cfg = A.cfg;
  const int cpb = cfg.chains_per_block, L = ch.ladder_size, CS = A.cluster;
  uint16_t* lut = reinterpret_cast<uint16_t*>(smem);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + TemperSmem::lut_bytes);
  int* cs_all = reinterpret_cast<int*>(hist_all + (size_t)cpb * kDirWords);
  int* bs_all = cs_all + cpb * kMaxM;
  int* ld_e = bs_all + cpb * kMaxM;  // leader arrays (64 entries each)
  int* ld_temp = ld_e + 64;
  int* ld_chain = ld_temp + 64;
  int* ld_stop = ld_chain + 64;
  int* team_red = ld_stop + 4;  // 16-byte aligned: ld_stop's block holds 4 ints

  cg::cluster_group cluster = cg::this_cluster();
  const int rank = CS > 1 ? (int)cluster.block_rank() : 0;
  auto barrier = [&]() {
    if (CS > 1)
      cluster.sync();
    else
      __syncthreads();
  };
  // leader arrays: CTA rank 0 of the cluster (CS > 1) or this CTA (CS == 1)
  int* L_e = CS > 1 ? cluster.map_shared_rank(ld_e, 0) : ld_e;
  int* L_temp = CS > 1 ? cluster.map_shared_rank(ld_temp, 0) : ld_temp;
  int* L_stop = CS > 1 ? cluster.map_shared_rank(ld_stop, 0) : ld_stop;

  const int warp = threadIdx.x / TT;  // this chain's index in the CTA
  Team<WPC> tm{(int)threadIdx.x % TT, 1 + warp, team_red + 2 * WPC * warp, 0, {}};
  const int c = blockIdx.x * cpb + warp;
  const int lad = c / L;
  const int li = c % L;
  const int lidx = CS > 1 ? li : warp;              // index into the leader arrays
  const int lbase = CS > 1 ? 0 : (warp / L) * L;    // this ladder's block in them
  const int n = ch.ladder_n[lad], m = 2 * n;
  int* cs = cs_all + warp * kMaxM;
  int* bs = bs_all + warp * kMaxM;
  uint32_t* hist = hist_all + (size_t)warp * kDirWords;

  full_lut_copy(lut, A.lut);
  for (int i = threadIdx.x; i < cpb * kDirWords; i += blockDim.x) hist_all[i] = 0u;
  for (int s = tm.t; s < m; s += TT) {
    cs[s] = ch.cols[(size_t)c * kMaxM + s];
    bs[s] = ch.badness[(size_t)c * kMaxM + s];
  }
#pragma unroll
  for (int j = 0; j < Team<WPC>::kSlots; ++j) {  // this thread's slots (the ones it loaded)
    const int k = tm.t + TT * j;
    tm.key[j] = k < m ? (k >> 1) * kLutW + (int)ch.cols[(size_t)c * kMaxM + k] : 0;
  }
  int E = ch.energy[c], bestE = ch.best_energy[c];
  int removed = UMB ? ch.removed[c] : 0;
  uint64_t counter = ch.counter[c];
  uint32_t accepted = ch.accepted[c];
  uint32_t err = 0;
  bool hit_done = false;

  // The leader CTA loads the ladder bookkeeping of its ladder(s).
  const bool leader_cta = rank == 0;
  const int lad_first = (blockIdx.x * cpb) / L;          // first ladder of this CTA
  const int n_lad_here = CS > 1 ? 1 : cpb / L;
  if (leader_cta) {
    for (int i = threadIdx.x; i < n_lad_here * L; i += blockDim.x) {
      const int gl = lad_first + i / L;
      ld_chain[i] = ch.chain_at[(size_t)gl * L + i % L];
      ld_temp[i] = ch.temp_of[(size_t)gl * L + i % L];
    }
    if (threadIdx.x == 0) *ld_stop = 0;
  }
  uint32_t lround = 0, lexch = 0;  // leader-thread copies (one leader per ladder)
  const bool ladder_leader = leader_cta && tm.t == 0 && (CS > 1 ? warp == 0 : (warp % L) == 0);
  if (ladder_leader) {
    lround = ch.ladder_round[lad];
    lexch = ch.ladder_exchanges[lad];
  }
  barrier();

  const int rounds = cfg.ladder_rounds ? cfg.ladder_rounds[lad] : cfg.rounds;
  const int per_round = cfg.round_proposals > 0 ? cfg.round_proposals : cfg.round_sweeps * m;
  const uint32_t k0 = (uint32_t)cfg.seed, k1 = (uint32_t)(cfg.seed >> 32);
  const int W = ch.acc_width;
  WalkParams wp;
  wp.bad_bias = cfg.bad_bias;
  wp.k0 = k0;
  wp.k1 = k1;
  wp.ref = ch.reference;
  wp.frac = nullptr;
  wp.s_q = 0;
  wp.c2s_q = 0;
  for (int r = 0; r < rounds; ++r) {
    const int temp = L_temp[lidx];
    const uint32_t* thr = ch.acc_thresh + (size_t)temp * W;
    if (UMB) {
      const size_t pos = (size_t)lad * L + temp;  // the replica position (temperature slot) of this chain
      wp.frac = ch.acc_frac + (size_t)temp * 768;
      wp.s_q = ch.umbrella[2 * pos];
      wp.c2s_q = ch.umbrella[2 * pos + 1];
    }
    // The proposals' Philox blocks 32 at a time: lane l makes the block of
    // proposal p + l (counter + l), and proposal p + j takes lane j's by shuffle.
    U4 batch = {0u, 0u, 0u, 0u};
    for (int p = 0; p < per_round; ++p) {
      const int j = p & 31;
      if (j == 0) {
        const uint64_t cl = counter + (uint64_t)(tm.t & 31);
        batch = philox4x32_10(U4{(uint32_t)cl, (uint32_t)(cl >> 32), (uint32_t)c, kTagPropose}, k0, k1);
      }
      const U4 rnd = {__shfl_sync(0xffffffffu, batch.x, j), __shfl_sync(0xffffffffu, batch.y, j),
                      __shfl_sync(0xffffffffu, batch.z, j), __shfl_sync(0xffffffffu, batch.w, j)};
      const int acc = propose_walk<WPC, BIAS, UMB>(tm, cs, bs, m, lut, hist, rnd, counter, c, thr, W, E, err, wp,
                                                   removed);
      ++counter;
      if (acc) {
        ++accepted;
        if (E < bestE) {
          bestE = E;
          for (int s = tm.t; s < m; s += TT) ch.best_cols[(size_t)c * kMaxM + s] = (int16_t)cs[s];
        }
        if (cfg.target_energy >= 0 && E <= cfg.target_energy && !hit_done) {
          hit_done = true;
          if (tm.t == 0 && ch.hit != nullptr && atomicCAS(ch.hit, -1, c) == -1) {
            const uint64_t now = global_ns();
            ch.hit[1] = (int32_t)(uint32_t)counter;
            ch.hit[2] = (int32_t)(uint32_t)now;
            ch.hit[3] = (int32_t)(uint32_t)(now >> 32);
            if (ch.stop) atomicExch(ch.stop, 1);
          }
        }
      }
    }
    if (!cfg.exchange) continue;
    if (tm.t == 0) L_e[lidx] = E;
    barrier();
    if (ladder_leader) {
      exchange_ladder(ld_chain + lbase, ld_temp + lbase, ld_e + lbase, L, lad, lround, ch.exch_thresh,
                      ch.exch_width, k0, k1, lexch);
      ++lround;
      if (ch.stop != nullptr && warp == 0) *ld_stop = *((volatile int*)ch.stop);
    }
    barrier();
    if (*((volatile int*)L_stop)) break;
  }

  // write back
  for (int s = tm.t; s < m; s += TT) {
    ch.cols[(size_t)c * kMaxM + s] = (int16_t)cs[s];
    ch.badness[(size_t)c * kMaxM + s] = bs[s];
  }
  if (err && ch.error_word) atomicOr(ch.error_word, err);
  if (tm.t == 0) {
    ch.energy[c] = E;
    ch.best_energy[c] = bestE;
    ch.counter[c] = counter;
    ch.accepted[c] = accepted;
    if (UMB) ch.removed[c] = removed;
    if (ch.global_best) atomicMin(ch.global_best, bestE);
  }
  if (ladder_leader) {
    ch.ladder_round[lad] = lround;
    ch.ladder_exchanges[lad] = lexch;
  }
  if (leader_cta) {
    __syncthreads();  // leader threads finished their exchanges above
    for (int i = threadIdx.x; i < n_lad_here * L; i += blockDim.x) {
      const int gl = lad_first + i / L;
      ch.chain_at[(size_t)gl * L + i % L] = ld_chain[i];
      ch.temp_of[(size_t)gl * L + i % L] = ld_temp[i];
    }
  }
  barrier();  // keep the leader's shared memory alive until every CTA is done with it
}

// Full recompute of every chain's energy (determinant count) and badness
// (slope count) compared with the maintained values.  One warp per chain.
constexpr int kAuditWarps = 4;
constexpr size_t kAuditSmem = kFullLutBytes + kAuditWarps * (sizeof(uint32_t) * kDirWords + 2 * sizeof(int) * kMaxM);

__global__ void __launch_bounds__(kAuditWarps * 32) audit_kernel(const n3_chains ch, const uint16_t* __restrict__ g_lut,
                                                                   int32_t* mismatch) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t* lut = reinterpret_cast<uint16_t*>(smem);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + kFullLutBytes);
  int* cs_all = reinterpret_cast<int*>(hist_all + kAuditWarps * kDirWords);
  int* bs_all = cs_all + kAuditWarps * kMaxM;
  full_lut_copy(lut, g_lut);
  for (int i = threadIdx.x; i < kAuditWarps * kDirWords; i += blockDim.x) hist_all[i] = 0u;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* cs = cs_all + warp * kMaxM;
  int* bs = bs_all + warp * kMaxM;
  uint32_t* hist = hist_all + warp * kDirWords;
  for (int c = blockIdx.x * kAuditWarps + warp; c < ch.n_chains; c += gridDim.x * kAuditWarps) {
    const int n = ch.ladder_n[c / ch.ladder_size], m = 2 * n;
    for (int s = lane; s < m; s += 32) cs[s] = ch.cols[(size_t)c * kMaxM + s];
    __syncwarp();
    const int e = warp_sum(det_state<false>(cs, n, lane, nullptr));
    slope_state(cs, n, lut, hist, lane, bs);
    __syncwarp();
    int bad_ok = 1;
    for (int s = lane; s < m; s += 32) bad_ok &= bs[s] == ch.badness[(size_t)c * kMaxM + s];
    bad_ok = __all_sync(0xffffffffu, bad_ok);
    if (lane == 0 && (e != ch.energy[c] || !bad_ok)) {
      atomicAdd(mismatch, 1);
      if (ch.error_word) atomicOr(ch.error_word, kErrAudit);
    }
    __syncwarp();
  }
}

}  // namespace n3

namespace n3host {

static int check_chains(const n3_chains* ch) {
  if (ch == nullptr) return set_error(N3_ERR_ARG, "null chains descriptor");
  const int L = ch->ladder_size;
  if (L < 2 || L > 64) return set_error(N3_ERR_ARG, "ladder_size %d outside [2, 64]", L);
  if (ch->n_chains <= 0 || ch->n_chains % L)
    return set_error(N3_ERR_ARG, "n_chains %d is not a positive multiple of ladder_size %d", ch->n_chains, L);
  if (!ch->cols || !ch->badness || !ch->energy || !ch->best_energy || !ch->best_cols || !ch->temp_of ||
      !ch->chain_at || !ch->counter || !ch->accepted || !ch->ladder_n || !ch->ladder_round ||
      !ch->ladder_exchanges || !ch->acc_thresh || !ch->exch_thresh)
    return set_error(N3_ERR_ARG, "null device pointer in chains descriptor");
  if (ch->acc_width < 2 || ch->exch_width < 2) return set_error(N3_ERR_ARG, "threshold tables too narrow");
  return N3_OK;
}

using TemperKernel = void (*)(const n3::TemperArgs);

template <int WPC>
static TemperKernel temper_instance_w(bool bias, bool umb) {
  return umb ? (bias ? n3::temper_kernel<WPC, true, true> : n3::temper_kernel<WPC, false, true>)
             : (bias ? n3::temper_kernel<WPC, true, false> : n3::temper_kernel<WPC, false, false>);
}

static TemperKernel temper_instance(int wpc, bool bias, bool umb) {
  switch (wpc) {
    case 8: return temper_instance_w<8>(bias, umb);
    case 4: return temper_instance_w<4>(bias, umb);
    case 2: return temper_instance_w<2>(bias, umb);
    default: return temper_instance_w<1>(bias, umb);
  }
}

int temper_launch(const n3_chains* ch, const n3_temper_config* cfg, cudaStream_t st) {
  N3_TRY(check_chains(ch));
  if (cfg == nullptr) return set_error(N3_ERR_ARG, "null config");
  const int L = ch->ladder_size, cpb = cfg->chains_per_block;
  const int tpc = cfg->threads_per_chain == 0 ? 32 : cfg->threads_per_chain;
  if (tpc != 32 && tpc != 64 && tpc != 128 && tpc != 256)
    return set_error(N3_ERR_ARG, "threads_per_chain %d is not 32, 64, 128 or 256", cfg->threads_per_chain);
  const int wpc = tpc / 32;
  if (cpb < 1 || cpb * wpc > 16)
    return set_error(N3_ERR_ARG, "chains_per_block %d x %d warps per chain outside [1, 16] warps", cpb, wpc);
  int cluster = 1;
  if (cpb < L) {
    if (L % cpb) return set_error(N3_ERR_ARG, "chains_per_block %d does not divide ladder_size %d", cpb, L);
    cluster = L / cpb;
    if (cluster > 8) return set_error(N3_ERR_ARG, "a ladder would span %d CTAs (max 8)", cluster);
  } else if (cpb % L) {
    return set_error(N3_ERR_ARG, "chains_per_block %d is not a multiple of ladder_size %d", cpb, L);
  }
  if (ch->n_chains % cpb) return set_error(N3_ERR_ARG, "n_chains not a multiple of chains_per_block");
  if (cfg->rounds < 0 || cfg->round_proposals < 0 || cfg->round_sweeps < 0)
    return set_error(N3_ERR_ARG, "negative round count or length");
  if (!cfg->exchange && cfg->round_proposals == 0 && cfg->round_sweeps == 0)
    return set_error(N3_ERR_ARG, "a round without exchange needs proposals");
  if (cfg->bad_bias < 0 || cfg->bad_bias > 100) return set_error(N3_ERR_ARG, "bad_bias %d outside [0, 100]", cfg->bad_bias);
  const bool umb = ch->umbrella != nullptr;
  if (umb) {
    if (!ch->reference || !ch->removed || !ch->acc_frac)
      return set_error(N3_ERR_ARG, "umbrella needs reference, removed and acc_frac");
    if (cfg->exchange)
      return set_error(N3_ERR_ARG, "temperature-only exchange is disabled with umbrella potentials");
  }
  N3_TRY(ensure_device_tables());
  n3::TemperArgs args;
  args.ch = *ch;
  args.lut = dir_lut_full_device_ptr();
  args.cfg = *cfg;
  args.cluster = cluster;
  const size_t smem = n3::TemperSmem::bytes(cpb);
  const bool bias = cfg->bad_bias > 0;
  void (*kern)(const n3::TemperArgs) = temper_instance(wpc, bias, umb);
  N3_TRY(allow_smem(reinterpret_cast<const void*>(kern), n3::TemperSmem::bytes(16)));
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(ch->n_chains / cpb);
  lc.blockDim = dim3(cpb * tpc);
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&lc, kern, args);
  if (e != cudaSuccess) return set_error(N3_ERR_CUDA, "temper_kernel launch: %s", cudaGetErrorString(e));
  return check_launch("temper_kernel");
}

}  // namespace n3host

namespace n3host {
int prepare_tempering() {
  for (int wpc : {1, 2, 4, 8})
    for (int b = 0; b < 2; ++b)
      for (int u = 0; u < 2; ++u)
        N3_TRY(allow_smem(reinterpret_cast<const void*>(temper_instance(wpc, b, u)), n3::TemperSmem::bytes(16)));
  return allow_smem(reinterpret_cast<const void*>(n3::audit_kernel), n3::kAuditSmem);
}
}  // namespace n3host

extern "C" {

int n3_temper_run(const n3_chains* chains, const n3_temper_config* config, void* stream) {
  return n3host::temper_launch(chains, config, (cudaStream_t)stream);
}

int n3_temper_audit(const n3_chains* chains, int32_t* mismatch, void* stream) {
  N3_TRY(n3host::check_chains(chains));
  if (mismatch == nullptr) return n3host::set_error(N3_ERR_ARG, "null mismatch counter");
  N3_TRY(n3host::ensure_device_tables());
  const n3_chains ch = *chains;
  const size_t smem = n3::kAuditSmem;
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(n3::audit_kernel), smem));
  const int want = (ch.n_chains + n3::kAuditWarps - 1) / n3::kAuditWarps;
  const int grid = want < n3host::sm_count() * 4 ? want : n3host::sm_count() * 4;
  n3::audit_kernel<<<grid, n3::kAuditWarps * 32, smem, (cudaStream_t)stream>>>(ch, n3host::dir_lut_full_device_ptr(),
                                                                                 mismatch);
  return n3host::check_launch("audit_kernel");
}

}  // extern "C"

namespace n3 {
__global__ void clock_kernel(int64_t* out) { out[0] = (int64_t)global_ns(); }
}  // namespace n3

extern "C" int n3_device_clock_ns(int64_t* out, void* stream) {
  if (out == nullptr) return n3host::set_error(N3_ERR_ARG, "null output");
  n3::clock_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(out);
  return n3host::check_launch("clock_kernel");
}
