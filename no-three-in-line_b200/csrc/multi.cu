// Multi-point moves: the three-cycle scores of src/no_three_75/accelerated.py:196-276
// (evaluate_three_cycles) and the four-cycle / double-switch neighbourhood scans
// of src/no_three_75/gpu_neighborhood.py:70-211 (best_four_cycle,
// best_double_switch).
//
// A move that relocates the points of a slot set M (k points in k distinct
// rows; columns permuted among them) changes E by
//   dE = side(new positions) - side(old positions),
//   side(X) = sum_i t_A(x_i) + sum_{i<j} j_A(x_i, x_j) + #collinear triples within X,
// where A = S \ M, t_A(x) = pairs of A collinear with x (a direction histogram
// around x over A) and j_A(x, y) = points of A on the line x-y (the count of
// that direction in x's histogram).  Both sides count exactly the collinear
// triples that contain a point of M, before and after.  The reference scores a
// three-cycle by its O(n^2) pair loops and a four-point move by materialising
// the whole candidate state and rescoring it (O(n^3)); here each is O(n) per
// position, and the scan shares positions: for a slot set (anchor + 3 slots)
// every four-cycle and double switch puts each target at one of 12 possible
// positions, so 4 + 12 histograms score its 6 four-cycles and 3 double switches.
#include <stdint.h>

#include "dirs.cuh"
#include "n3_common.cuh"

namespace n3 {
namespace multi {

constexpr int kT = kSlotsPerLane;  // 5 slots per lane

// This lane's slots' direction-table keys row * kLutW + column (the state is
// fixed for the whole kernel, so the keys stay in registers).
__device__ __forceinline__ void lane_keys(const int* __restrict__ cs, int m, int lane, int (&key)[kT]) {
#pragma unroll
  for (int t = 0; t < kT; ++t) {
    const int k = lane + 32 * t;
    key[t] = k < m ? (k >> 1) * kLutW + cs[k] : 0;
  }
}

// Direction histogram of centre (rx, cx) over A, on the full signed table:
// slots whose bit t is set in `skip` (this lane's slot lane + 32 t is a moved
// one) are left out, and so are the points in row rx.  key: lane_keys of the
// state.
__device__ __forceinline__ int hist_build_excl(const int (&key)[kT], int m, int rx, int cx, uint32_t skip,
                                               const uint16_t* __restrict__ lutf, uint32_t* __restrict__ hist,
                                               int lane, int (&ids)[kT]) {
  const uint16_t* base = lutf + kFullLutCentre - (rx * kLutW + cx);
  int pairs = 0;
#pragma unroll
  for (int t = 0; t < kT; ++t) {
    const int k = lane + 32 * t;
    ids[t] = -1;
    if (k < m && !((skip >> t) & 1u) && (k >> 1) != rx) {
      const int id = base[key[t]];
      ids[t] = id;
      pairs += hist_add(hist, id);
    }
  }
  return pairs;
}

__device__ __forceinline__ uint32_t skip_mask(int lane, const int* moved, int count) {
  uint32_t s = 0;
#pragma unroll
  for (int t = 0; t < kT; ++t) {
    const int k = lane + 32 * t;
    for (int i = 0; i < count; ++i) s |= (uint32_t)(k == moved[i]) << t;
  }
  return s;
}

__device__ __forceinline__ int collinear(int r0, int c0, int r1, int c1, int r2, int c2) {
  return (r1 - r0) * (c2 - c0) == (c1 - c0) * (r2 - r0);
}

// side() of `count` positions (distinct rows) over A; all lanes return the sum.
__device__ __forceinline__ int side_sum(const int (&key)[kT], int m, const int* rows, const int* cols, int count, uint32_t skip,
                        const uint16_t* __restrict__ lutf, uint32_t* __restrict__ hist, int lane) {
  int total = 0;
  for (int i = 0; i < count; ++i) {
    int ids[kT];
    const int part = hist_build_excl(key, m, rows[i], cols[i], skip, lutf, hist, lane, ids);
    __syncwarp();
    int pair_lines = 0;
    if (lane == 0)
      for (int j = i + 1; j < count; ++j)
        pair_lines += hist_get(hist, dir_id_full(lutf, rows[j] - rows[i], cols[j] - cols[i]));
    __syncwarp();
    hist_release(hist, ids);
    __syncwarp();
    total += warp_sum(part) + __shfl_sync(0xffffffffu, pair_lines, 0);
  }
  for (int i = 0; i < count; ++i)
    for (int j = i + 1; j < count; ++j)
      for (int k = j + 1; k < count; ++k) total += collinear(rows[i], cols[i], rows[j], cols[j], rows[k], cols[k]);
  return total;
}

// --------------------------------------------------------------------------
// Three-cycles: warp per candidate (u, v, w, orientation).
// --------------------------------------------------------------------------
constexpr int kWarps = 8;
constexpr size_t kSmem = kFullLutBytes + kWarps * sizeof(uint32_t) * kDirWords + sizeof(int) * kMaxM;

__global__ void __launch_bounds__(kWarps * 32) three_cycle_kernel(const int32_t* __restrict__ p,
                                                                  const int32_t* __restrict__ q, int n,
                                                                  const int32_t* __restrict__ cand, int count,
                                                                  int64_t current, const uint16_t* __restrict__ g_lut,
                                                                  int64_t* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t* lutf = reinterpret_cast<uint16_t*>(smem);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + kFullLutBytes);
  int* cs = reinterpret_cast<int*>(hist_all + kWarps * kDirWords);
  full_lut_copy(lutf, g_lut);
  for (int i = threadIdx.x; i < kWarps * kDirWords; i += blockDim.x) hist_all[i] = 0u;
  const int m = 2 * n;
  for (int s = threadIdx.x; s < m; s += blockDim.x) cs[s] = (s & 1) ? q[s >> 1] : p[s >> 1];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* hist = hist_all + warp * kDirWords;
  int key[kT];
  lane_keys(cs, m, lane, key);
  for (int c = blockIdx.x * kWarps + warp; c < count; c += gridDim.x * kWarps) {
    const int u = cand[4 * c], v = cand[4 * c + 1], w = cand[4 * c + 2], o = cand[4 * c + 3];
    // the moves search.py:38-65 generates: three slots in three rows, three
    // distinct columns, no row left with a repeated column
    bool ok = u >= 0 && v >= 0 && w >= 0 && u < m && v < m && w < m && (o == 0 || o == 1);
    int nu = 0, nv = 0, nw = 0;
    if (ok) {
      const int ru = u >> 1, rv = v >> 1, rw = w >> 1;
      ok = ru != rv && ru != rw && rv != rw && cs[u] != cs[v] && cs[u] != cs[w] && cs[v] != cs[w];
      nu = o == 0 ? cs[v] : cs[w];
      nv = o == 0 ? cs[w] : cs[u];
      nw = o == 0 ? cs[u] : cs[v];
      ok = ok && nu != cs[u ^ 1] && nv != cs[v ^ 1] && nw != cs[w ^ 1];
    }
    if (!ok) {
      if (lane == 0) out[c] = (int64_t)1 << 60;
      continue;
    }
    const int moved[3] = {u, v, w};
    const uint32_t skip = skip_mask(lane, moved, 3);
    const int rows[3] = {u >> 1, v >> 1, w >> 1};
    const int old_cols[3] = {cs[u], cs[v], cs[w]};
    const int new_cols[3] = {nu, nv, nw};
    const int before = side_sum(key, m, rows, old_cols, 3, skip, lutf, hist, lane);
    const int after = side_sum(key, m, rows, new_cols, 3, skip, lutf, hist, lane);
    if (lane == 0) out[c] = current - before + after;
  }
}

// --------------------------------------------------------------------------
// Neighbourhood scan around an anchor slot: warp per (row triple, layer choice).
// Enumeration order and tie rule of gpu_neighborhood.py:108-116 / :181-190: row
// triples in itertools.combinations order, layers in itertools.product order,
// then orderings (itertools.permutations) or the three pairings; the result is
// the first candidate (in that order) with the lowest score, kept only if it
// improves on the base.
// --------------------------------------------------------------------------
struct ScanArgs {
  const int32_t* p;
  const int32_t* q;
  int n, anchor;
  int64_t base;          // E of the state
  int combos;            // C(n - 1, 3)
  const uint16_t* lut;
  unsigned long long* best;   // [2]: (score << 32 | index) for four-cycles, double switches
  unsigned long long* legal;  // [2]
};

// j-th (0-based, lexicographic) 3-subset {a < b < c} of {0 .. N-1}
__device__ __forceinline__ void unrank3(int x, int N, int& a, int& b, int& c) {
  a = 0;
  for (;; ++a) {
    const int k = N - 1 - a, cnt = k * (k - 1) / 2;
    if (x < cnt) break;
    x -= cnt;
  }
  b = a + 1;
  for (;; ++b) {
    const int cnt = N - 1 - b;
    if (x < cnt) break;
    x -= cnt;
  }
  c = b + 1 + x;
}

__global__ void __launch_bounds__(kWarps * 32) scan_kernel(const ScanArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t* lutf = reinterpret_cast<uint16_t*>(smem);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + kFullLutBytes);
  int* cs = reinterpret_cast<int*>(hist_all + kWarps * kDirWords);
  __shared__ int jt_all[kWarps][12][12];  // points of A on the line between two candidate positions
  __shared__ int tn_all[kWarps][12];      // t_A of each candidate position
  full_lut_copy(lutf, A.lut);
  for (int i = threadIdx.x; i < kWarps * kDirWords; i += blockDim.x) hist_all[i] = 0u;
  const int n = A.n, m = 2 * n;
  for (int s = threadIdx.x; s < m; s += blockDim.x) cs[s] = (s & 1) ? A.q[s >> 1] : A.p[s >> 1];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * kWarps + warp;
  if (gw >= A.combos * 8) return;  // no block-level barrier follows
  uint32_t* hist = hist_all + warp * kDirWords;
  int (*jt)[12] = jt_all[warp];
  int* tn = tn_all[warp];
  const int combo = gw >> 3, layers = gw & 7;
  const int arow = A.anchor >> 1;
  int r[3];
  unrank3(combo, n - 1, r[0], r[1], r[2]);
  int T[4];
  T[0] = A.anchor;
  for (int i = 0; i < 3; ++i) {
    const int row = r[i] < arow ? r[i] : r[i] + 1;  // i-th row other than the anchor's
    T[i + 1] = 2 * row + ((layers >> (2 - i)) & 1);
  }
  int rowT[4], colT[4], partner[4];
  for (int i = 0; i < 4; ++i) {
    rowT[i] = T[i] >> 1;
    colT[i] = cs[T[i]];
    partner[i] = cs[T[i] ^ 1];
  }
  const uint32_t skip = skip_mask(lane, T, 4);
  int key[kT];
  lane_keys(cs, m, lane, key);
  const int before = side_sum(key, m, rowT, colT, 4, skip, lutf, hist, lane);
  // the 12 candidate positions: target i with the column of source j != i (index 3 i + (j > i ? j - 1 : j))
  for (int a = 0; a < 12; ++a) {
    const int i = a / 3, jj = a % 3, j = jj >= i ? jj + 1 : jj;
    const int rx = rowT[i], cx = colT[j];
    int ids[kT];
    const int part = hist_build_excl(key, m, rx, cx, skip, lutf, hist, lane, ids);
    __syncwarp();
    if (lane < 12) {
      const int b = lane, ib = b / 3, jb = b % 3 >= ib ? b % 3 + 1 : b % 3;
      jt[a][b] = ib != i ? hist_get(hist, dir_id_full(lutf, rowT[ib] - rx, colT[jb] - cx)) : 0;
    }
    __syncwarp();
    hist_release(hist, ids);
    const int t = warp_sum(part);
    if (lane == 0) tn[a] = t;
    __syncwarp();
  }
  // the moves: sigma[i] = source of target i
  if (lane < 9) {
    int sigma[4];
    unsigned int idx;
    if (lane < 6) {  // four-cycle with ordering number `lane` of (T1, T2, T3)
      const int perm[6][3] = {{1, 2, 3}, {1, 3, 2}, {2, 1, 3}, {2, 3, 1}, {3, 1, 2}, {3, 2, 1}};
      const int o0 = perm[lane][0], o1 = perm[lane][1], o2 = perm[lane][2];
      sigma[0] = o0;
      sigma[o0] = o1;
      sigma[o1] = o2;
      sigma[o2] = 0;
      idx = (unsigned)((combo * 8 + layers) * 6 + lane);
    } else {  // double switch pairing lane - 6: (a, anchor, c, b), (b, c, anchor, a), (c, b, a, anchor)
      const int pairs[3][4] = {{1, 0, 3, 2}, {2, 3, 0, 1}, {3, 2, 1, 0}};
      for (int i = 0; i < 4; ++i) sigma[i] = pairs[lane - 6][i];
      idx = (unsigned)((combo * 8 + layers) * 3 + (lane - 6));
    }
    bool legal = true;
    int after = 0, pos[4], nr[4], nc[4];
    for (int i = 0; i < 4; ++i) {
      const int j = sigma[i];
      legal = legal && colT[j] != partner[i];
      pos[i] = 3 * i + (j > i ? j - 1 : j);
      nr[i] = rowT[i];
      nc[i] = colT[j];
      after += tn[pos[i]];
    }
    for (int i = 0; i < 4; ++i)
      for (int k = i + 1; k < 4; ++k) after += jt[pos[i]][pos[k]];
    for (int i = 0; i < 4; ++i)
      for (int j = i + 1; j < 4; ++j)
        for (int k = j + 1; k < 4; ++k) after += collinear(nr[i], nc[i], nr[j], nc[j], nr[k], nc[k]);
    if (legal) {
      const int64_t score = A.base + after - before;
      const unsigned long long key = ((unsigned long long)score << 32) | idx;
      const int which = lane < 6 ? 0 : 1;
      atomicMin(A.best + which, key);
      atomicAdd(A.legal + which, 1ull);
    }
  }
}

}  // namespace multi
}  // namespace n3

extern "C" {

int n3_three_cycle_scores(const int32_t* p, const int32_t* q, int n, const int32_t* candidates, int count,
                          int64_t current, int64_t* scores, void* stream) {
  if (n < 3 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "three cycles: n=%d outside [3, %d]", n, N3_MAX_N);
  if (count < 0) return n3host::set_error(N3_ERR_ARG, "three cycles: negative count");
  if (count == 0) return N3_OK;
  if (!p || !q || !candidates || !scores) return n3host::set_error(N3_ERR_ARG, "three cycles: null buffer");
  N3_TRY(n3host::ensure_device_tables());
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(n3::multi::three_cycle_kernel), n3::multi::kSmem));
  const int want = (count + n3::multi::kWarps - 1) / n3::multi::kWarps;
  const int grid = want < 2 * n3host::sm_count() ? want : 2 * n3host::sm_count();
  n3::multi::three_cycle_kernel<<<grid, n3::multi::kWarps * 32, n3::multi::kSmem, (cudaStream_t)stream>>>(
      p, q, n, candidates, count, current, n3host::dir_lut_full_device_ptr(), scores);
  return n3host::check_launch("three_cycle_kernel");
}

int n3_neighborhood_scan(const int32_t* p, const int32_t* q, int n, int anchor, int64_t current,
                         unsigned long long* best, unsigned long long* legal, void* stream) {
  if (n < 5 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "neighbourhood scan: n=%d outside [5, %d]", n,
                                                      N3_MAX_N);
  if (anchor < 0 || anchor >= 2 * n) return n3host::set_error(N3_ERR_RANGE, "anchor index outside point slots");
  if (!p || !q || !best || !legal) return n3host::set_error(N3_ERR_ARG, "neighbourhood scan: null buffer");
  N3_TRY(n3host::ensure_device_tables());
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(n3::multi::scan_kernel), n3::multi::kSmem));
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(best, 0xFF, 2 * sizeof(unsigned long long), st) != cudaSuccess ||
      cudaMemsetAsync(legal, 0, 2 * sizeof(unsigned long long), st) != cudaSuccess)
    return n3host::set_error(N3_ERR_CUDA, "neighbourhood scan: memset failed");
  n3::multi::ScanArgs A;
  A.p = p;
  A.q = q;
  A.n = n;
  A.anchor = anchor;
  A.base = current;
  A.combos = (n - 1) * (n - 2) * (n - 3) / 6;
  A.lut = n3host::dir_lut_full_device_ptr();
  A.best = best;
  A.legal = legal;
  const int warps = A.combos * 8;
  n3::multi::scan_kernel<<<(warps + n3::multi::kWarps - 1) / n3::multi::kWarps, n3::multi::kWarps * 32,
                           n3::multi::kSmem, st>>>(A);
  return n3host::check_launch("scan_kernel");
}

}  // extern "C"
