// Exhaustive 2-switch beam on the device: every legal 2-switch of every elite
// that touches a bad slot (or every slot, on global generations), scored
// exactly from the parent without building the children, then ordered and
// sampled the way the reference's host loop orders and samples them.
//
// Reference: gpu_exhaustive_beam.py:17-325 (enumerate_switches,
// candidate_descriptors, gpu_exhaustive_beam_search).  The reference builds
// every child on the device, rescores each in full (551,300 triple tests at
// n = 75), copies all scores to the host and sorts, filters and shuffles there.
// Here, per generation:
//
//  1. anchors_kernel (one CTA): the anchors of each elite in (elite, slot)
//     order, and for each anchor u its first candidate index.  Candidate order
//     is the reference's descriptor order: elite, anchor u ascending, partner v
//     ascending, skipping u's row and anchors v < u.
//  2. n3_two_switch_scores: the exact score after each (elite, u, v) swap, from
//     the elite's maintained badness and two direction histograms per partner.
//  3. compact_kernel (a warp per anchor): each kept partner's score at its
//     candidate index, 2^29 where the swap is illegal (the reference's marker
//     for invalid children, gpu_exhaustive_beam.py:179), plus its descriptor.
//  4. select_kernel (one CTA): the legal count, the first min(legal, 24 E)
//     candidates of the stable score order (the quality pool), and every legal
//     candidate within energy_window of the best score, in index order (the
//     diverse pool).
//  5. shuffle_kernel: CPython's random.shuffle of the diverse pool, draw for
//     draw, from the search's random.Random state (pyrandom.cuh).
//  6. prospect kernels: the quality pool, then the first 24 E shuffled diverse
//     candidates not already in it; each prospect's position in the shuffled
//     diverse pool (-1 if absent); the prospects' states as P/Q rows.
//
// The host then applies the reference's retention rules (signatures and the
// `seen` set over at most 48 E prospects, gpu_exhaustive_beam.py:223-260).
#include "dirs.cuh"
#include "n3_common.cuh"
#include "pyrandom.cuh"

namespace n3 {
namespace exh {

constexpr int kInvalid = 1 << 29;
constexpr int kMaxElites = 2048;
constexpr int kSelThreads = 1024;
constexpr int kBins = 8192;          // score bins per histogram pass of the selection
constexpr int kMaxPool = 1 << 20;    // diverse pool entries the device shuffle takes

// Status words (int64) written by the kernels and read by the host.
enum { kStAnchors = 0, kStCandidates = 1, kStLegal = 2, kStQuality = 3, kStDiverse = 4, kStProspects = 5,
       kStError = 6, kStWords = 8 };

// 1. Anchors and candidate offsets; 160 threads (5 warps), one slot each,
// elites in order.  For an anchor u with rank r among its elite's anchors, the
// kept partners number m - 2 - (r - [u odd and u - 1 an anchor]).
__global__ void __launch_bounds__(160) anchors_kernel(const int32_t* __restrict__ bad, int E, int m, int global,
                                                     int32_t* __restrict__ anchors, int32_t* __restrict__ start,
                                                     int64_t* __restrict__ status) {
  __shared__ int wflag[5], wcnt[5];
  const int s = threadIdx.x, warp = s >> 5, lane = s & 31;
  int a_off = 0, c_off = 0;
  for (int p = 0; p < E; ++p) {
    const bool flag = s < m && (global || bad[(size_t)p * m + s] > 0);
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    const bool partner = (bal >> (lane ^ 1)) & 1u;
    const int rank_w = __popc(bal & ((1u << lane) - 1u));
    int cnt = flag ? m - 2 - rank_w : 0;  // warp-local part of the rank for now
    if (lane == 0) wflag[warp] = __popc(bal);
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; ++w) before += wflag[w];
    const int rank = rank_w + before;
    cnt = flag ? m - 2 - (rank - ((s & 1) && partner ? 1 : 0)) : 0;
    // exclusive scan of cnt over the slots
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wcnt[warp] = incl;
    __syncthreads();
    int cbefore = 0, total_c = 0, total_a = 0;
    for (int w = 0; w < 5; ++w) {
      if (w < warp) cbefore += wcnt[w];
      total_c += wcnt[w];
      total_a += wflag[w];
    }
    if (flag) {
      anchors[2 * (size_t)(a_off + rank)] = p;
      anchors[2 * (size_t)(a_off + rank) + 1] = s;
      start[a_off + rank] = c_off + cbefore + incl - cnt;
    }
    a_off += total_a;
    c_off += total_c;
    __syncthreads();
  }
  if (s == 0) {
    status[kStAnchors] = a_off;
    status[kStCandidates] = c_off;
  }
}

// 3. Candidate scores and descriptors, a warp per anchor.
__global__ void compact_kernel(const int16_t* __restrict__ cols, const int32_t* __restrict__ bad, int m, int global,
                               const int32_t* __restrict__ anchors, const int32_t* __restrict__ start,
                               const int64_t* __restrict__ status, const int32_t* __restrict__ partner_scores,
                               int32_t* __restrict__ cand_score, int32_t* __restrict__ cand_code) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int A = (int)status[kStAnchors];
  if (warp >= A) return;
  const int p = anchors[2 * warp], u = anchors[2 * warp + 1];
  const int cu = cols[(size_t)p * m + u];
  int pos = start[warp];
  for (int v0 = 0; v0 < m; v0 += 32) {
    const int v = v0 + lane;
    bool keep = false;
    if (v < m && (v >> 1) != (u >> 1)) {
      const bool anchor_v = global || bad[(size_t)p * m + v] > 0;
      keep = !(anchor_v && v < u);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      const int at = pos + __popc(bal & ((1u << lane) - 1u));
      const int sc = partner_scores[(size_t)warp * m + v];
      // the reference's enumeration also rejects equal columns (identity swaps)
      const bool legal = sc != N3_SENTINEL && cols[(size_t)p * m + v] != cu;
      cand_score[at] = legal ? sc : kInvalid;
      cand_code[at] = warp * 256 + v;
    }
    pos += __popc(bal);
  }
}

// Block-wide exclusive scan of one int per thread (kSelThreads threads);
// returns the exclusive prefix and writes the total to *total.
__device__ int block_scan(int x, int* wsum, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = lane < kSelThreads / 32 ? wsum[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < kSelThreads / 32) wsum[lane] = wi - w;
    if (lane == 31) wsum[32] = wi;
  }
  __syncthreads();
  const int ex = incl - x + wsum[warp];
  *total = wsum[32];
  __syncthreads();
  return ex;
}

// 4. Quality and diverse pools, one CTA of kSelThreads threads.
__global__ void __launch_bounds__(kSelThreads, 1) select_kernel(const int32_t* __restrict__ cand_score,
                                                                int64_t* __restrict__ status, int elite_size,
                                                                int best, int window, int32_t* __restrict__ quality,
                                                                int32_t* __restrict__ diverse) {
  __shared__ unsigned hist[kBins];
  __shared__ int wsum[33];
  __shared__ int red_min, red_cnt;
  __shared__ int qlist[kSelThreads];
  __shared__ int sh_base, sh_tb, sh_need, sh_less;
  const int C = (int)status[kStCandidates];
  const int t = threadIdx.x;
  if (t == 0) {
    red_min = kInvalid;
    red_cnt = 0;
    status[kStError] = 0;
  }
  __syncthreads();
  // pass 0: legal count and the lowest score
  int cnt = 0, mn = kInvalid;
  for (int i = t; i < C; i += kSelThreads) {
    const int s = cand_score[i];
    if (s < kInvalid) {
      ++cnt;
      mn = min(mn, s);
    }
  }
  atomicAdd(&red_cnt, cnt);
  atomicMin(&red_min, mn);
  __syncthreads();
  const int L = red_cnt;
  const int K = min(L, 24 * elite_size);
  // pass 1: the score bin of the K-th smallest (scores >= base and < base + kBins per pass)
  if (t == 0) {
    sh_base = red_min;
    sh_tb = -1;
    sh_less = 0;
  }
  __syncthreads();
  while (K > 0 && sh_tb < 0) {
    const int base = sh_base;
    for (int b = t; b < kBins; b += kSelThreads) hist[b] = 0u;
    __syncthreads();
    for (int i = t; i < C; i += kSelThreads) {
      const int s = cand_score[i];
      if (s < kInvalid && s >= base && s - base < kBins) atomicAdd(&hist[s - base], 1u);
    }
    __syncthreads();
    if (t == 0) {
      int cum = sh_less;
      for (int b = 0; b < kBins; ++b) {
        if (cum + (int)hist[b] >= K) {
          sh_tb = b;
          sh_need = K - cum;
          sh_less = cum;
          break;
        }
        cum += (int)hist[b];
      }
      if (sh_tb < 0) {  // the K smallest scores span more than kBins: not supported (reported)
        sh_less = cum;
        sh_base = base + kBins;
        status[kStError] = 1;
      }
    }
    __syncthreads();
  }
  // bin starts: exclusive prefix over bins < tb (tb itself starts at sh_less)
  const int base = sh_base, tb = sh_tb, need = sh_need;
  if (K > 0 && t == 0) {
    unsigned run = (unsigned)(sh_less);
    // rewrite hist[b] (b <= tb) as the start position of bin b, from the top down
    for (int b = tb; b >= 0; --b) {
      const unsigned c = b == tb ? (unsigned)need : hist[b];
      run -= b == tb ? 0u : c;
      hist[b] = b == tb ? (unsigned)sh_less : run;
    }
  }
  __syncthreads();
  // pass 2: stable placement of the quality pool; tiles in index order, the
  // qualifying items of a tile compacted in order, then placed by warp 0 32 at
  // a time (match-any ranks) with per-bin running positions in hist[]
  int taken_tb = 0;  // warp 0's count of bin-tb items placed
  for (int tile = 0; K > 0 && tile < C; tile += kSelThreads) {
    const int i = tile + t;
    int bin = -1;
    if (i < C) {
      const int s = cand_score[i];
      if (s < kInvalid && s >= base && s - base <= tb) bin = s - base;
    }
    int total;
    const int ex = block_scan(bin >= 0 ? 1 : 0, wsum, &total);
    if (bin >= 0) qlist[ex] = i;
    __syncthreads();
    if (t < 32) {
      for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + t;
        int item = -1, b = -1;
        if (k < total) {
          item = qlist[k];
          b = cand_score[item] - base;
        }
        const unsigned peers = __match_any_sync(0xffffffffu, b);
        const int rank = __popc(peers & ((1u << t) - 1u));
        const int first = __ffs(peers) - 1;
        if (b >= 0) {
          const int at = (int)hist[b] + rank;
          const bool place = b < tb || (taken_tb + rank < need);
          if (place) quality[at] = item;
        }
        __syncwarp();
        if (b >= 0 && t == first) hist[b] += (unsigned)__popc(peers);
        // bin tb items seen by this round (uniform across the warp)
        const unsigned tbmask = __ballot_sync(0xffffffffu, b == tb);
        taken_tb += __popc(tbmask);
        __syncwarp();
      }
    }
    __syncthreads();
  }
  // pass 3: the diverse pool, legal and within the window, in index order
  int dcount = 0;
  const int limit = best + window;
  for (int tile = 0; tile < C; tile += kSelThreads) {
    const int i = tile + t;
    const bool in = i < C && cand_score[i] < kInvalid && cand_score[i] <= limit;
    int total;
    const int ex = block_scan(in ? 1 : 0, wsum, &total);
    if (in) diverse[dcount + ex] = i;
    dcount += total;
  }
  if (t == 0) {
    if (sh_tb >= 0 && sh_base != red_min) status[kStError] = 1;
    status[kStLegal] = L;
    status[kStQuality] = K;
    status[kStDiverse] = dcount;
  }
}

// 5. CPython's shuffle of the diverse pool (count <= kMaxPool); the bitmap of
// the shuffle's repeated-position check lives in dynamic shared memory.
__global__ void __launch_bounds__(256) shuffle_kernel(uint32_t* state, int32_t* values,
                                                      const int64_t* __restrict__ status) {
  extern __shared__ uint32_t seen[];
  __shared__ uint32_t mt[beam::kMT], out[beam::kMT];
  const int count = (int)status[kStDiverse];
  const int words = (count + 31) / 32;
  for (int i = threadIdx.x; i < beam::kMT; i += blockDim.x) mt[i] = state[i];
  for (int i = threadIdx.x; i < words; i += blockDim.x) seen[i] = 0u;
  __syncthreads();
  if (threadIdx.x < 32 && count > 1) {
    int idx = (int)state[beam::kMT];
    beam::py_shuffle_warp(mt, out, idx, values, count, seen, threadIdx.x);
    if (threadIdx.x == 0) state[beam::kMT] = (uint32_t)idx;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < beam::kMT; i += blockDim.x) state[i] = mt[i];
}

// 6a. Marks the quality pool (flag 1, position -1) before the diverse positions.
__global__ void mark_quality_kernel(const int32_t* __restrict__ quality, const int64_t* __restrict__ status,
                                    uint8_t* __restrict__ in_quality, int32_t* __restrict__ dpos) {
  const int K = (int)status[kStQuality];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
    in_quality[quality[k]] = 1;
    dpos[quality[k]] = -1;
  }
}

// 6b. Position of each shuffled diverse candidate.
__global__ void diverse_positions_kernel(const int32_t* __restrict__ diverse, const int64_t* __restrict__ status,
                                         int32_t* __restrict__ dpos) {
  const int D = (int)status[kStDiverse];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < D; k += gridDim.x * blockDim.x) dpos[diverse[k]] = k;
}

// 6c. The prospect list (one CTA): quality pool, then the first 24 E shuffled
// diverse candidates not in it; each prospect's diverse position, score and
// descriptor.  Then unmarks the quality pool.
__global__ void __launch_bounds__(kSelThreads, 1) prospects_kernel(
    const int32_t* __restrict__ quality, const int32_t* __restrict__ diverse, int64_t* __restrict__ status,
    int elite_size, uint8_t* __restrict__ in_quality, const int32_t* __restrict__ dpos,
    const int32_t* __restrict__ cand_score, int32_t* __restrict__ prospects, int32_t* __restrict__ p_pos,
    int32_t* __restrict__ p_score) {
  __shared__ int wsum[33];
  const int K = (int)status[kStQuality], D = (int)status[kStDiverse];
  const int Dtake = min(D, 24 * elite_size);
  const int t = threadIdx.x;
  for (int k = t; k < K; k += kSelThreads) prospects[k] = quality[k];
  int np = K;
  for (int tile = 0; tile < Dtake; tile += kSelThreads) {
    const int k = tile + t;
    const bool add = k < Dtake && !in_quality[diverse[k]];
    int total;
    const int ex = block_scan(add ? 1 : 0, wsum, &total);
    if (add) prospects[np + ex] = diverse[k];
    np += total;
  }
  __syncthreads();
  for (int k = t; k < np; k += kSelThreads) {
    const int c = prospects[k];
    p_pos[k] = dpos[c];
    p_score[k] = cand_score[c];
  }
  __syncthreads();
  for (int k = t; k < K; k += kSelThreads) in_quality[quality[k]] = 0;
  if (t == 0) status[kStProspects] = np;
}

// 6d. The prospects' states as P/Q rows (a warp per prospect).
__global__ void build_prospects_kernel(const int16_t* __restrict__ cols, int m, const int32_t* __restrict__ anchors,
                                       const int32_t* __restrict__ cand_code, const int32_t* __restrict__ prospects,
                                       const int64_t* __restrict__ status, int32_t* __restrict__ pp,
                                       int32_t* __restrict__ pq, int32_t* __restrict__ parent_of) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int NP = (int)status[kStProspects];
  if (w >= NP) return;
  const int code = cand_code[prospects[w]];
  const int a = code >> 8, v = code & 0xFF;
  const int p = anchors[2 * a], u = anchors[2 * a + 1];
  const int n = m / 2;
  const int16_t* src = cols + (size_t)p * m;
  const int cu = src[u], cv = src[v];
  for (int s = lane; s < m; s += 32) {
    const int c = s == u ? cv : s == v ? cu : src[s];
    (s & 1 ? pq : pp)[(size_t)w * n + (s >> 1)] = c;
  }
  if (lane == 0) parent_of[w] = p;
}

// Rows of P/Q by index (elites from prospects), and the slot-layout copy.
__global__ void gather_rows_kernel(const int32_t* __restrict__ sp, const int32_t* __restrict__ sq,
                                   const int32_t* __restrict__ idx, int count, int n, int32_t* __restrict__ dp,
                                   int32_t* __restrict__ dq, int16_t* __restrict__ dcols) {
  const int r = blockIdx.x;
  if (r >= count) return;
  const int from = idx[r];
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const int a = sp[(size_t)from * n + k], b = sq[(size_t)from * n + k];
    dp[(size_t)r * n + k] = a;
    dq[(size_t)r * n + k] = b;
    dcols[(size_t)r * 2 * n + 2 * k] = (int16_t)a;
    dcols[(size_t)r * 2 * n + 2 * k + 1] = (int16_t)b;
  }
}

}  // namespace exh
}  // namespace n3

extern "C" {

int n3_two_switch_scores(const int16_t* cols, const int32_t* badness, const int32_t* current, int B, int n,
                         const int32_t* anchors, int A, int32_t* out, void* stream);

int n3_exh_candidates(const int16_t* elite_cols, const int32_t* elite_badness, const int32_t* elite_scores, int E,
                      int n, int global, int32_t* anchors, int32_t* anchor_start, int32_t* partner_scores,
                      int32_t* cand_score, int32_t* cand_code, int64_t* status, void* stream) {
  using namespace n3::exh;
  if (n < 3 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "n=%d outside [3, %d]", n, N3_MAX_N);
  if (E < 1 || E > kMaxElites) return n3host::set_error(N3_ERR_RANGE, "elite count %d outside [1, %d]", E, kMaxElites);
  if (!elite_cols || !elite_badness || !elite_scores || !anchors || !anchor_start || !partner_scores ||
      !cand_score || !cand_code || !status)
    return n3host::set_error(N3_ERR_ARG, "null device pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const int m = 2 * n;
  anchors_kernel<<<1, 160, 0, st>>>(elite_badness, E, m, global, anchors, anchor_start, status);
  N3_TRY(n3host::check_launch("anchors_kernel"));
  // the anchor count decides the partner-score launch: read it (8 bytes)
  int64_t A = 0;
  if (cudaMemcpyAsync(&A, status + kStAnchors, sizeof(A), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return n3host::check_launch("n3_exh_candidates: anchor count");
  if (A == 0) return N3_OK;
  N3_TRY(n3_two_switch_scores(elite_cols, elite_badness, elite_scores, E, n, anchors, (int)A, partner_scores, stream));
  const int warps_per_block = 8;
  compact_kernel<<<(unsigned)((A + warps_per_block - 1) / warps_per_block), warps_per_block * 32, 0, st>>>(
      elite_cols, elite_badness, m, global, anchors, anchor_start, status, partner_scores, cand_score, cand_code);
  return n3host::check_launch("compact_kernel");
}

int n3_exh_select(const int32_t* cand_score, int64_t* status, int elite_size, int best, int window,
                  uint32_t* rng_state, int32_t* quality, int32_t* diverse, uint8_t* in_quality, int32_t* dpos,
                  int32_t* prospects, int32_t* p_pos, int32_t* p_score, int max_candidates, void* stream) {
  using namespace n3::exh;
  if (elite_size < 1 || elite_size > kMaxElites || window < 0)
    return n3host::set_error(N3_ERR_RANGE, "bad elite size or window");
  if (!cand_score || !status || !rng_state || !quality || !diverse || !in_quality || !dpos || !prospects || !p_pos ||
      !p_score)
    return n3host::set_error(N3_ERR_ARG, "null device pointer");
  cudaStream_t st = (cudaStream_t)stream;
  select_kernel<<<1, kSelThreads, 0, st>>>(cand_score, status, elite_size, best, window, quality, diverse);
  N3_TRY(n3host::check_launch("select_kernel"));
  // the diverse count sizes the shuffle's bitmap
  int64_t D = 0;
  if (cudaMemcpyAsync(&D, status + kStDiverse, sizeof(D), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return n3host::check_launch("n3_exh_select: diverse count");
  if (D > kMaxPool)
    return n3host::set_error(N3_ERR_RANGE, "diverse pool of %lld candidates exceeds %d", (long long)D, kMaxPool);
  const size_t smem = sizeof(uint32_t) * (size_t)((D + 31) / 32 + 1);
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(shuffle_kernel), sizeof(uint32_t) * (kMaxPool / 32 + 1)));
  shuffle_kernel<<<1, 256, smem, st>>>(rng_state, diverse, status);
  N3_TRY(n3host::check_launch("shuffle_kernel"));
  const int blocks = 4 * n3host::sm_count();
  mark_quality_kernel<<<blocks, 256, 0, st>>>(quality, status, in_quality, dpos);
  diverse_positions_kernel<<<blocks, 256, 0, st>>>(diverse, status, dpos);
  prospects_kernel<<<1, kSelThreads, 0, st>>>(quality, diverse, status, elite_size, in_quality, dpos, cand_score,
                                               prospects, p_pos, p_score);
  (void)max_candidates;
  return n3host::check_launch("prospect kernels");
}

int n3_exh_build_prospects(const int16_t* elite_cols, int n, const int32_t* anchors, const int32_t* cand_code,
                           const int32_t* prospects, const int64_t* status, int max_prospects, int32_t* pp,
                           int32_t* pq, int32_t* parent_of, void* stream) {
  if (!elite_cols || !anchors || !cand_code || !prospects || !status || !pp || !pq || !parent_of)
    return n3host::set_error(N3_ERR_ARG, "null device pointer");
  if (max_prospects < 1) return N3_OK;
  const int wpb = 8;
  n3::exh::build_prospects_kernel<<<(max_prospects + wpb - 1) / wpb, wpb * 32, 0, (cudaStream_t)stream>>>(
      elite_cols, 2 * n, anchors, cand_code, prospects, status, pp, pq, parent_of);
  return n3host::check_launch("build_prospects_kernel");
}

int n3_exh_gather_rows(const int32_t* src_p, const int32_t* src_q, const int32_t* index, int count, int n,
                       int32_t* dst_p, int32_t* dst_q, int16_t* dst_cols, void* stream) {
  if (count < 0 || n < 1 || n > N3_MAX_N) return n3host::set_error(N3_ERR_ARG, "bad gather sizes");
  if (count == 0) return N3_OK;
  if (!src_p || !src_q || !index || !dst_p || !dst_q || !dst_cols)
    return n3host::set_error(N3_ERR_ARG, "null device pointer");
  n3::exh::gather_rows_kernel<<<count, 96, 0, (cudaStream_t)stream>>>(src_p, src_q, index, count, n, dst_p, dst_q,
                                                                      dst_cols);
  return n3host::check_launch("gather_rows_kernel");
}

}  // extern "C"
