// (b) Exact incremental deltas of row-pair column swaps.
//
// A move exchanges the columns of slots u and v (different rows): u' takes
// (r_u, c_v), v' takes (r_v, c_u).  It is legal iff the columns differ and
// neither new point duplicates the other point of its row
// (src/no_three_75/tempering.py:58, accelerated.py:145-151).  With
// A = S \ {u, v} and, for a centre X, t(X) = number of pairs of A collinear
// with X and j(X, Y) = number of points of A collinear with X and Y:
//
//   dE = t(u') + t(v') + j(u', v') - t(u) - t(v) - j(u, v)
//
// which is the reference's "triples through a moved point" accounting
// (tempering.py:68-89: pairs through one moved point plus triples through
// both).  Only pairs through the moved points are touched, and they are counted
// by direction class: t(X) = sum over directions from X of C(count, 2), one
// direction-histogram insertion per point of A (dirs.cuh).  The same
// histograms give every other point's badness change:
//
//   dbad[k] = sum over new centres (count - 1) - sum over old centres (count - 1)
//             + [k on line(u', v')] - [k on line(u, v)]
//
// and dbad[u] = t(u') + j(u',v') - t(u) - j(u,v) (likewise v).
//
// A second, independent kernel evaluates the reference formulation literally
// (every pair (i<j) outside {u,v} tested against u, u', v, v' with int32 cross
// products, plus every k against (u,v) and (u',v')); tests compare the two.
#include "dirs.cuh"
#include "n3_common.cuh"

namespace n3 {

// Exact dE (and, if dbad != nullptr, this lane's badness changes for slots
// lane + 32 t, plus the moved slots' changes in *dbad_u, *dbad_v) of a legal
// move.  Uses the 4 centres u, v, u', v'; hist must be zeroed, is left zeroed.
// lutf: the full signed direction table; key: this lane's slots' table keys
// row * kLutW + column.
template <bool BAD>
__device__ __forceinline__ int swap_delta_hist(const int* __restrict__ cs, const int (&key)[kSlotsPerLane], int m,
                                               int u, int v, const uint16_t* __restrict__ lutf,
                                               uint32_t* __restrict__ hist, int lane, int (&dbad)[kSlotsPerLane],
                                               int* dbad_u, int* dbad_v) {
  const int ru = u >> 1, rv = v >> 1, cu = cs[u], cv = cs[v];
  // centre order: u, v, u', v'
  const int crow[4] = {ru, rv, ru, rv};
  const int ccol[4] = {cu, cv, cv, cu};
  int tX[4];
  int j_old = 0, j_new = 0;
  if (BAD) {
#pragma unroll
    for (int t = 0; t < kSlotsPerLane; ++t) dbad[t] = 0;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    int ids[kSlotsPerLane];
    int part = 0;
    {
      const int rx = crow[c];
      const uint16_t* base = lutf + kFullLutCentre - (rx * kLutW + ccol[c]);
#pragma unroll
      for (int t = 0; t < kSlotsPerLane; ++t) {
        const int k = lane + 32 * t;
        ids[t] = -1;
        if (k < m && k != u && k != v && (k >> 1) != rx) {
          const int id = base[key[t]];
          ids[t] = id;
          part += hist_add(hist, id);
        }
      }
    }
    __syncwarp();
    tX[c] = warp_sum(part);
    const int sign = c < 2 ? -1 : 1;
    int line_id = -1;  // direction of the other moved point, for centres u and u'
    if (c == 0) {
      line_id = dir_id_full(lutf, rv - ru, cv - cu);
      j_old = hist_get(hist, line_id);
    } else if (c == 2) {
      line_id = dir_id_full(lutf, rv - ru, cu - cv);
      j_new = hist_get(hist, line_id);
    }
    if (BAD) {
#pragma unroll
      for (int t = 0; t < kSlotsPerLane; ++t) {
        if (ids[t] >= 0) dbad[t] += sign * (hist_get(hist, ids[t]) - 1 + (ids[t] == line_id));
      }
    }
    __syncwarp();
    hist_release(hist, ids);
    __syncwarp();
  }
  if (BAD) {
    *dbad_u = (tX[2] + j_new) - (tX[0] + j_old);
    *dbad_v = (tX[3] + j_new) - (tX[1] + j_old);
  }
  return (tX[2] + tX[3] + j_new) - (tX[0] + tX[1] + j_old);
}

// The reference formulation (tempering.py:68-89), pair by pair.  Returns this
// lane's share of dE; badness changes are added to the warp's smem array `db`.
__device__ __forceinline__ int aligned(int a, int ca, int b, int cb, int c, int cc) {
  return (b - a) * (cc - ca) == (cb - ca) * (c - a);
}

__device__ int swap_delta_pairs(const int* __restrict__ cs, int m, int u, int v, int lane, int* db) {
  const int ru = u >> 1, rv = v >> 1, cu = cs[u], cv = cs[v];
  int delta = 0;
  for (int i = 0; i < m - 1; ++i) {
    if (i == u || i == v) continue;
    const int ri = i >> 1, ci = cs[i];
    for (int j = i + 1 + lane; j < m; j += 32) {
      if (j == u || j == v) continue;
      const int rj = j >> 1, cj = cs[j];
      int d = aligned(ru, cv, ri, ci, rj, cj) - aligned(ru, cu, ri, ci, rj, cj);
      if (d) {
        delta += d;
        if (db) {
          atomicAdd(db + u, d);
          atomicAdd(db + i, d);
          atomicAdd(db + j, d);
        }
      }
      d = aligned(rv, cu, ri, ci, rj, cj) - aligned(rv, cv, ri, ci, rj, cj);
      if (d) {
        delta += d;
        if (db) {
          atomicAdd(db + v, d);
          atomicAdd(db + i, d);
          atomicAdd(db + j, d);
        }
      }
    }
  }
  for (int k = lane; k < m; k += 32) {
    if (k == u || k == v) continue;
    const int d = aligned(ru, cv, rv, cu, k >> 1, cs[k]) - aligned(ru, cu, rv, cv, k >> 1, cs[k]);
    if (d) {
      delta += d;
      if (db) {
        atomicAdd(db + u, d);
        atomicAdd(db + v, d);
        atomicAdd(db + k, d);
      }
    }
  }
  return delta;
}

constexpr int kDeltaWarps = 8;

struct DeltaSmem {
  static constexpr size_t lut_bytes = kFullLutBytes;  // the full signed direction table
  static constexpr size_t bytes =
      lut_bytes + sizeof(uint32_t) * kDirWords * kDeltaWarps + sizeof(int) * kMaxM * kDeltaWarps * 2;
};

__device__ __forceinline__ void load_lut_and_clear(unsigned char* smem, const uint16_t* __restrict__ g_lut,
                                                   uint16_t*& lut, uint32_t*& hist_all, int*& cs_all, int*& aux_all) {
  lut = reinterpret_cast<uint16_t*>(smem);
  hist_all = reinterpret_cast<uint32_t*>(smem + DeltaSmem::lut_bytes);
  cs_all = reinterpret_cast<int*>(hist_all + kDirWords * kDeltaWarps);
  aux_all = cs_all + kMaxM * kDeltaWarps;
  full_lut_copy(lut, g_lut);
  for (int i = threadIdx.x; i < kDirWords * kDeltaWarps; i += blockDim.x) hist_all[i] = 0u;
  __syncthreads();
}

// Batched swap deltas: moves[mv] = (state, u, v).  PAIRS selects the literal
// reference formulation.  dE = N3_SENTINEL for illegal moves or bad indices.
template <bool PAIRS>
__global__ void __launch_bounds__(kDeltaWarps * 32) swap_delta_kernel(const int16_t* __restrict__ cols, int B, int n,
                                                                        const int32_t* __restrict__ moves, int M,
                                                                        const uint16_t* __restrict__ g_lut,
                                                                        int32_t* __restrict__ dE,
                                                                        int32_t* __restrict__ dbad) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t* lut;
  uint32_t* hist_all;
  int *cs_all, *aux_all;
  load_lut_and_clear(smem, g_lut, lut, hist_all, cs_all, aux_all);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m = 2 * n;
  int* cs = cs_all + warp * kMaxM;
  int* db = aux_all + warp * kMaxM;
  uint32_t* hist = hist_all + warp * kDirWords;
  for (int mv = blockIdx.x * kDeltaWarps + warp; mv < M; mv += gridDim.x * kDeltaWarps) {
    const int b = moves[3 * mv], u = moves[3 * mv + 1], v = moves[3 * mv + 2];
    const bool in_range = b >= 0 && b < B && u >= 0 && u < m && v >= 0 && v < m;
    int key[kSlotsPerLane];
#pragma unroll
    for (int t = 0; t < kSlotsPerLane; ++t) {  // this lane's slots and their table keys
      const int k = lane + 32 * t;
      const int c = in_range && k < m ? (int)cols[(size_t)b * m + k] : 0;
      if (in_range && k < m) cs[k] = c;
      key[t] = (k >> 1) * kLutW + c;
    }
    __syncwarp();
    if (!in_range || !legal_swap(cs, u, v)) {
      if (lane == 0) dE[mv] = N3_SENTINEL;
      if (dbad)
        for (int s = lane; s < m; s += 32) dbad[(size_t)mv * m + s] = 0;
      __syncwarp();
      continue;
    }
    int d;
    if (PAIRS) {
      if (dbad)
        for (int s = lane; s < m; s += 32) db[s] = 0;
      __syncwarp();
      d = warp_sum(swap_delta_pairs(cs, m, u, v, lane, dbad ? db : nullptr));
      __syncwarp();
      if (dbad)
        for (int s = lane; s < m; s += 32) dbad[(size_t)mv * m + s] = db[s];
    } else {
      int local[kSlotsPerLane];
      int du = 0, dv = 0;
      if (dbad) {
        d = swap_delta_hist<true>(cs, key, m, u, v, lut, hist, lane, local, &du, &dv);
#pragma unroll
        for (int t = 0; t < kSlotsPerLane; ++t) {
          const int k = lane + 32 * t;
          if (k < m) dbad[(size_t)mv * m + k] = k == u ? du : (k == v ? dv : local[t]);
        }
      } else {
        d = swap_delta_hist<false>(cs, key, m, u, v, lut, hist, lane, local, &du, &dv);
      }
    }
    if (lane == 0) dE[mv] = d;
    __syncwarp();
  }
}

// Shared memory of partner_scores_kernel: the full signed direction table, a
// histogram per warp, the anchor's state.
struct PartnerSmem {
  static constexpr size_t bytes = kFullLutBytes + sizeof(uint32_t) * kDirWords * kDeltaWarps + sizeof(int) * kMaxM;
};

// Scores of every partner of anchor slots (the reference plugin
// two_switch_scores, src/no_three_75/gpu_delta.py:19-75, and
// evaluate_two_switches / evaluate_transpositions, accelerated.py:40-195):
//   out = current - (bad[u] + bad[v] - joint(u, v)) + t(u') + t(v') + j(u', v')
// One CTA per anchor; its warps split the partners.  SAME_LAYER restricts
// partners to slots of u's layer and indexes the output by partner row.  The
// anchor's state is fixed for all its partners, so each lane keeps the
// direction-table keys row * kLutW + column of its slots in registers and a
// histogram insertion is one load from the full signed table and one atomic.
template <bool SAME_LAYER>
__global__ void __launch_bounds__(kDeltaWarps * 32) partner_scores_kernel(
    const int16_t* __restrict__ cols, const int32_t* __restrict__ badness, const int32_t* __restrict__ current,
    int B, int n, const int32_t* __restrict__ anchors, int A, const uint16_t* __restrict__ g_lut_full,
    int32_t* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t* lutf = reinterpret_cast<uint16_t*>(smem);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + kFullLutBytes);
  int* cs = reinterpret_cast<int*>(hist_all + kDirWords * kDeltaWarps);  // one state per CTA: shared by all warps
  full_lut_copy(lutf, g_lut_full);
  for (int i = threadIdx.x; i < kDirWords * kDeltaWarps; i += blockDim.x) hist_all[i] = 0u;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m = 2 * n;
  const int width = SAME_LAYER ? n : m;
  uint32_t* hist = hist_all + warp * kDirWords;
  for (int a = blockIdx.x; a < A; a += gridDim.x) {
    const int b = anchors[2 * a], u = anchors[2 * a + 1];
    const bool in_range = b >= 0 && b < B && u >= 0 && u < m;
    __syncthreads();
    if (in_range)
      for (int s = threadIdx.x; s < m; s += blockDim.x) cs[s] = cols[(size_t)b * m + s];
    __syncthreads();
    if (!in_range) {
      for (int s = threadIdx.x; s < width; s += blockDim.x) out[(size_t)a * width + s] = N3_SENTINEL;
      continue;
    }
    const int ru = u >> 1, cu = cs[u];
    const int cur = current[b];
    const int bad_u = badness[(size_t)b * m + u];
    int key[kSlotsPerLane];
#pragma unroll
    for (int t = 0; t < kSlotsPerLane; ++t) {
      const int k = lane + 32 * t;
      key[t] = k < m ? (k >> 1) * kLutW + cs[k] : 0;
    }
    // one histogram of centre (rx, cx) over the slots other than u, v and row rx
    auto build = [&](int rx, int cx, int v, int (&ids)[kSlotsPerLane]) {
      const uint16_t* base = lutf + kFullLutCentre - (rx * kLutW + cx);
      int pairs = 0;
#pragma unroll
      for (int t = 0; t < kSlotsPerLane; ++t) {
        const int k = lane + 32 * t;
        ids[t] = -1;
        if (k < m && k != u && k != v && (k >> 1) != rx) {
          const int id = base[key[t]];
          ids[t] = id;
          pairs += hist_add(hist, id);
        }
      }
      return pairs;
    };
    for (int w = warp; w < width; w += kDeltaWarps) {
      const int v = SAME_LAYER ? 2 * w + (u & 1) : w;
      // The reference's partner rule (accelerated.py:146-151, gpu_delta.py:175-180):
      // another row, and neither new point duplicates its row partner.  Equal
      // columns are allowed there (the move is then the identity, score = current).
      if ((v >> 1) == ru || cs[v] == cs[u ^ 1] || cu == cs[v ^ 1]) {
        if (lane == 0) out[(size_t)a * width + w] = N3_SENTINEL;
        continue;
      }
      const int rv = v >> 1, cv = cs[v];
      // joint(u, v): points other than u, v on the line through u and v
      int joint = 0;
#pragma unroll
      for (int t = 0; t < kSlotsPerLane; ++t) {
        const int k = lane + 32 * t;
        if (k < m && k != u && k != v)
          joint += (rv - ru) * (key[t] - (k >> 1) * kLutW - cu) == (cv - cu) * ((k >> 1) - ru);
      }
      int part = joint << 16;  // two sums in one reduction: joint (high) and pairs (low)
      int ids[kSlotsPerLane];
      part += build(ru, cv, v, ids);  // u' = (r_u, c_v)
      __syncwarp();
      const int j_new = hist_get(hist, dir_id_full(lutf, rv - ru, cu - cv));
      __syncwarp();
      hist_release(hist, ids);
      __syncwarp();
      part += build(rv, cu, v, ids);  // v' = (r_v, c_u)
      __syncwarp();
      hist_release(hist, ids);
      __syncwarp();
      const int sum = warp_sum(part);
      if (lane == 0) {
        const int old_aff = bad_u + badness[(size_t)b * m + v] - (sum >> 16);
        const int new_aff = (sum & 0xFFFF) + j_new;
        out[(size_t)a * width + w] = cur - old_aff + new_aff;
      }
    }
  }
}

}  // namespace n3

namespace n3host {

template <class K>
static int prepare(K kernel, size_t bytes = n3::DeltaSmem::bytes) {
  return allow_smem(reinterpret_cast<const void*>(kernel), bytes);
}

int prepare_delta() {
  N3_TRY(prepare(n3::swap_delta_kernel<true>));
  N3_TRY(prepare(n3::swap_delta_kernel<false>));
  N3_TRY(prepare(n3::partner_scores_kernel<true>, n3::PartnerSmem::bytes));
  return prepare(n3::partner_scores_kernel<false>, n3::PartnerSmem::bytes);
}

static int check_state_args(int B, int n, const void* cols) {
  if (n < 2 || n > N3_MAX_N) return set_error(N3_ERR_RANGE, "n=%d outside [2, %d]", n, N3_MAX_N);
  if (B < 0) return set_error(N3_ERR_ARG, "negative batch size %d", B);
  if (B > 0 && cols == nullptr) return set_error(N3_ERR_ARG, "null state pointer");
  return N3_OK;
}

static int launch_swap(bool pairs, const int16_t* cols, int B, int n, const int32_t* moves, int M, int32_t* dE,
                       int32_t* dbad, cudaStream_t st) {
  N3_TRY(check_state_args(B, n, cols));
  if (M < 0) return set_error(N3_ERR_ARG, "negative move count");
  if (M == 0) return N3_OK;
  if (moves == nullptr || dE == nullptr) return set_error(N3_ERR_ARG, "null move or output pointer");
  N3_TRY(ensure_device_tables());
  const uint16_t* lut = dir_lut_full_device_ptr();
  const int want = (M + n3::kDeltaWarps - 1) / n3::kDeltaWarps;
  const int grid = want < sm_count() * 2 ? want : sm_count() * 2;
  if (pairs) {
    N3_TRY(prepare(n3::swap_delta_kernel<true>));
    n3::swap_delta_kernel<true><<<grid, n3::kDeltaWarps * 32, n3::DeltaSmem::bytes, st>>>(cols, B, n, moves, M, lut,
                                                                                          dE, dbad);
  } else {
    N3_TRY(prepare(n3::swap_delta_kernel<false>));
    n3::swap_delta_kernel<false><<<grid, n3::kDeltaWarps * 32, n3::DeltaSmem::bytes, st>>>(cols, B, n, moves, M, lut,
                                                                                           dE, dbad);
  }
  return check_launch("swap_delta_kernel");
}

static int launch_partners(bool same_layer, const int16_t* cols, const int32_t* badness, const int32_t* current, int B,
                           int n, const int32_t* anchors, int A, int32_t* out, cudaStream_t st) {
  N3_TRY(check_state_args(B, n, cols));
  if (A < 0) return set_error(N3_ERR_ARG, "negative anchor count");
  if (A == 0) return N3_OK;
  if (!badness || !current || !anchors || !out) return set_error(N3_ERR_ARG, "null pointer");
  N3_TRY(ensure_device_tables());
  const uint16_t* lutf = dir_lut_full_device_ptr();
  const int grid = A < sm_count() * 4 ? A : sm_count() * 4;
  if (same_layer) {
    N3_TRY(prepare(n3::partner_scores_kernel<true>, n3::PartnerSmem::bytes));
    n3::partner_scores_kernel<true><<<grid, n3::kDeltaWarps * 32, n3::PartnerSmem::bytes, st>>>(
        cols, badness, current, B, n, anchors, A, lutf, out);
  } else {
    N3_TRY(prepare(n3::partner_scores_kernel<false>, n3::PartnerSmem::bytes));
    n3::partner_scores_kernel<false><<<grid, n3::kDeltaWarps * 32, n3::PartnerSmem::bytes, st>>>(
        cols, badness, current, B, n, anchors, A, lutf, out);
  }
  return check_launch("partner_scores_kernel");
}

}  // namespace n3host

extern "C" {

int n3_swap_delta(const int16_t* cols, int B, int n, const int32_t* moves, int M, int32_t* dE, int32_t* dbad,
                  void* stream) {
  return n3host::launch_swap(false, cols, B, n, moves, M, dE, dbad, (cudaStream_t)stream);
}

int n3_swap_delta_pairs(const int16_t* cols, int B, int n, const int32_t* moves, int M, int32_t* dE, int32_t* dbad,
                        void* stream) {
  return n3host::launch_swap(true, cols, B, n, moves, M, dE, dbad, (cudaStream_t)stream);
}

int n3_two_switch_scores(const int16_t* cols, const int32_t* badness, const int32_t* current, int B, int n,
                         const int32_t* anchors, int A, int32_t* out, void* stream) {
  return n3host::launch_partners(false, cols, badness, current, B, n, anchors, A, out, (cudaStream_t)stream);
}

int n3_transposition_scores(const int16_t* cols, const int32_t* badness, const int32_t* current, int B, int n,
                            const int32_t* anchors, int A, int32_t* out, void* stream) {
  return n3host::launch_partners(true, cols, badness, current, B, n, anchors, A, out, (cudaStream_t)stream);
}

}  // extern "C"
