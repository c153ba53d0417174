// Line-by-line conflict analysis of point sets: every line holding three or
// more of the points, with its canonical (A, B, C), its occupancy and its
// members, plus each point's badness.
//
// Reference: conflicts.analyze_points (src/no_three_75/conflicts.py:36-72),
// which calls geometry.canonical_line (src/no_three_75/geometry.py:14-28) on
// every pair and groups the pairs by line in a dict.  Here, one warp per point
// set, with no pair loop and no hash:
//
// * For each anchor point i, the other points are inserted into the anchor's
//   direction histogram (gcd-reduced directions, the full signed table of
//   dirs.cuh) in index order, 32 at a time: __match_any_sync ranks the lanes of
//   one batch that share a direction, so every point j learns ord(j), the
//   number of earlier points (j' < j, j' != i) on the line through i and j.
// * badness[i] = sum_j ord(j) = sum over lines through i of C(k - 1, 2), the
//   reference's per-point badness.
// * A line is emitted once, by its first member i and its second member j:
//   ord(j) == 0 and j > i.  Its members are the lanes whose direction matches
//   (one ballot per batch of 32 points: a 160-bit member mask), its occupancy
//   k = 1 + count, and (A, B, C) follows the reference's normalisation
//   (A = c_j - c_i, B = r_i - r_j, C = -(A r_i + B c_i), divided by their gcd,
//   A > 0 or A = 0 and B > 0).
//
// Output per line: int32 {A, B, C, k, mask0 .. mask4} (bit t of mask w is
// point 32 w + t).  The host sorts lines and builds the slope histogram and
// the weighted score from them (conflicts.py:60-72).
#include "dirs.cuh"
#include "n3_common.cuh"

namespace n3 {

constexpr int kAnaWarps = 4;
constexpr int kLineWords = 9;                 // A, B, C, k, 5 mask words
constexpr int kAnaMaxM = 32 * kSlotsPerLane;  // 160 points
constexpr size_t kAnaSmem = kFullLutBytes + kAnaWarps * (sizeof(uint32_t) * kDirWords + 3 * sizeof(int) * kAnaMaxM);

__device__ __forceinline__ int igcd(int a, int b) {
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b) {
    const int t = a % b;
    a = b;
    b = t;
  }
  return a;
}

__global__ void __launch_bounds__(kAnaWarps * 32) analyze_kernel(const int16_t* __restrict__ pts, int B, int m,
                                                                 const uint16_t* __restrict__ g_lut,
                                                                 int32_t* __restrict__ badness,
                                                                 int32_t* __restrict__ line_count,
                                                                 int32_t* __restrict__ lines, int cap,
                                                                 uint32_t* __restrict__ error_word) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t* lutf = reinterpret_cast<uint16_t*>(smem);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + kFullLutBytes);
  int* key_all = reinterpret_cast<int*>(hist_all + kAnaWarps * kDirWords);
  full_lut_copy(lutf, g_lut);
  for (int i = threadIdx.x; i < kAnaWarps * kDirWords; i += blockDim.x) hist_all[i] = 0u;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  int* key = key_all + warp * 3 * kAnaMaxM;  // key[s] = r * kLutW + c, then the rows, then the columns
  int* row = key + kAnaMaxM;
  int* col = row + kAnaMaxM;
  uint32_t* hist = hist_all + warp * kDirWords;
  for (int b = blockIdx.x * kAnaWarps + warp; b < B; b += gridDim.x * kAnaWarps) {
    int bad_range = 0;
    for (int s = lane; s < m; s += 32) {
      const int r = pts[((size_t)b * m + s) * 2], c = pts[((size_t)b * m + s) * 2 + 1];
      bad_range |= r < 0 || r >= kMaxN || c < 0 || c >= kMaxN;
      key[s] = r * kLutW + c;
      row[s] = r;
      col[s] = c;
    }
    __syncwarp();
    uint32_t err = __any_sync(0xffffffffu, bad_range) ? kErrColumnRange : 0u;
    int count = 0;
    for (int i = 0; i < m && !err; ++i) {
      const int ki = key[i];
      int ord[kSlotsPerLane], dir[kSlotsPerLane];
      int dup = 0, pairs = 0;
#pragma unroll
      for (int t = 0; t < kSlotsPerLane; ++t) {
        const int j = lane + 32 * t;
        const bool valid = j < m && j != i;
        const int kj = valid ? key[j] : 0;
        dup |= valid && kj == ki;
        // lanes without a point get a value no direction id can take
        const int d = valid && kj != ki ? (int)lutf[kFullLutCentre + kj - ki] : -1 - lane;
        dir[t] = valid ? d : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt_mask);
        const int before = d >= 0 ? hist_get(hist, d) : 0;
        __syncwarp();
        if (d >= 0 && rank == 0) atomicAdd(hist + (d >> 2), (uint32_t)__popc(peers) << ((d & 3) << 3));
        ord[t] = before + rank;
        pairs += d >= 0 ? ord[t] : 0;
        __syncwarp();
      }
      if (__any_sync(0xffffffffu, dup)) {
        err |= kErrDuplicate;
      } else {
        pairs = warp_sum(pairs);
        if (lane == 0) badness[(size_t)b * m + i] = pairs;
        // emit the lines whose first member is i, one per second member j
#pragma unroll
        for (int t = 0; t < kSlotsPerLane; ++t) {
          const int j = lane + 32 * t;
          const bool emit = dir[t] >= 0 && ord[t] == 0 && j > i && hist_get(hist, dir[t]) >= 2;
          unsigned todo = __ballot_sync(0xffffffffu, emit);
          while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const int d = __shfl_sync(0xffffffffu, dir[t], src);
            const int js = 32 * t + src;
            uint32_t mask[kSlotsPerLane];
#pragma unroll
            for (int w = 0; w < kSlotsPerLane; ++w) mask[w] = __ballot_sync(0xffffffffu, dir[w] == d);
#pragma unroll
            for (int w = 0; w < kSlotsPerLane; ++w)
              if (w == (i >> 5)) mask[w] |= 1u << (i & 31);
            if (lane == 0) {
              if (count < cap) {
                const int ri = row[i], ci = col[i], rj = row[js], cj = col[js];
                int A = cj - ci, Bc = ri - rj;
                int C = -(A * ri + Bc * ci);
                const int g = igcd(igcd(A, Bc), C);
                A /= g;
                Bc /= g;
                C /= g;
                if (A < 0 || (A == 0 && Bc < 0)) {
                  A = -A;
                  Bc = -Bc;
                  C = -C;
                }
                int32_t* rec = lines + ((size_t)b * cap + count) * kLineWords;
                rec[0] = A;
                rec[1] = Bc;
                rec[2] = C;
                rec[3] = 1 + hist_get(hist, d);
#pragma unroll
                for (int w = 0; w < kSlotsPerLane; ++w) rec[4 + w] = (int32_t)mask[w];
              }
              ++count;
            }
          }
        }
      }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < kSlotsPerLane; ++t)
        if (dir[t] >= 0) hist_clear(hist, dir[t]);
      __syncwarp();
    }
    if (lane == 0) {
      if (count > cap) err |= kErrCapacity;
      line_count[b] = err ? -1 : count;
      if (err && error_word) atomicOr(error_word, err);
    }
    __syncwarp();
  }
}

}  // namespace n3

extern "C" int n3_analyze_lines(const int16_t* points, int B, int m, int32_t* badness, int32_t* line_count,
                                int32_t* lines, int capacity, uint32_t* error_word, void* stream) {
  if (B < 0 || m < 0 || capacity < 0) return n3host::set_error(N3_ERR_ARG, "negative size");
  if (m > n3::kAnaMaxM) return n3host::set_error(N3_ERR_RANGE, "point sets of %d points exceed %d", m, n3::kAnaMaxM);
  if (B == 0) return N3_OK;
  if (!line_count || (m > 0 && (!points || !badness)) || (!lines && capacity > 0))
    return n3host::set_error(N3_ERR_ARG, "null device pointer");
  N3_TRY(n3host::ensure_device_tables());
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(n3::analyze_kernel), n3::kAnaSmem));
  const int want = (B + n3::kAnaWarps - 1) / n3::kAnaWarps;
  const int grid = want < n3host::sm_count() * 4 ? want : n3host::sm_count() * 4;
  n3::analyze_kernel<<<grid, n3::kAnaWarps * 32, n3::kAnaSmem, (cudaStream_t)stream>>>(
      points, B, m, n3host::dir_lut_full_device_ptr(), badness, line_count, lines, capacity, error_word);
  return n3host::check_launch("analyze_kernel");
}
