// Line tables of the n x n grid and the two table scorers
// (src/no_three_75/precompute.py:18-89 over src/no_three_75/cp_sat.py:109-157).
//
// The tables list every line with three or more grid points that is neither a
// row nor a column (_multi_point_lines skips pairs that share a row or a
// column).  A line enters the reference's dict at its second pair in the
// row-major pair loop, (first member, third member), so line ids follow
// (first member, third member).  For one first member (r, c) the third member
// is (r + 2a, c + 2b) for the line's primitive step (a >= 1, b != 0), so that
// order is the (a, b) order: no sort is needed.
//   count_kernel   CTA per first member: its lines and their grid points
//   scan_kernel    exclusive scans of both over the first members (one CTA)
//   emit_kernel    CTA per first member: line ids and CSR offsets by block
//                  scans in (a, b) order, members in row-major order
//   pairs_kernel   warp per line: pair_to_line of every pair on it
//   pair_score_kernel  score_pair_table: CTA per point list, warp per anchor
//                  point; the line ids of the anchor's pairs with the later
//                  points go into a shared hash; an id met c times before adds
//                  c, so an anchor adds C(m, 2) for m later points on a line and
//                  the anchors of a k-point line add C(k, 3)
//   csr_score_kernel   score_csr over 32 point lists at once: a word per grid
//                  point holds the lists' occupancy bits; a line's members are
//                  added into a 7-plane bit-sliced counter (at most 75 points a
//                  line), and the lists with three or more points on the line
//                  add C(count, 3)
#include <stdint.h>

#include "n3_common.cuh"

namespace n3 {
namespace lines {

constexpr int kThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kPairWarps = 8;
constexpr int kHashSlots = 512;       // per warp; an anchor inserts at most kMaxPairPoints - 1 ids
constexpr int kMaxPairPoints = 512;   // points per list for score_pair_table
constexpr int kCsrLists = 32;         // point lists per occupancy word

enum : uint32_t {
  kErrPointRange = 1u << 0,  // a point id outside [0, n * n)
  kErrPointTwice = 1u << 1,  // a point listed twice
  kErrHashFull = 1u << 2,    // cannot happen within kMaxPairPoints; checked all the same
};

// Candidate d in [0, (n - 1)(2n - 2)) -> step (a, b), in (a, b) order:
// a = 1 .. n - 1, then b = -(n - 1) .. -1, 1 .. n - 1.
__device__ __forceinline__ void step_of(int d, int n, int& a, int& b) {
  const int w = 2 * n - 2;
  a = 1 + d / w;
  const int j = d - (a - 1) * w;
  b = j < n - 1 ? j - (n - 1) : j - (n - 2);
}

__device__ __forceinline__ int gcd_small(int x, int y) {
  while (y != 0) {
    const int t = x % y;
    x = y;
    y = t;
  }
  return x;
}

// Grid points on the line from (r, c) with step (a, b), or 0 unless (a, b) is
// primitive, (r, c) is the line's first grid point and the line has three or
// more grid points.
__device__ __forceinline__ int line_length(int r, int c, int a, int b, int n) {
  if (r + 2 * a >= n || c + 2 * b < 0 || c + 2 * b >= n) return 0;  // no third point
  if (r - a >= 0 && c - b >= 0 && c - b < n) return 0;              // a grid point before (r, c)
  const int ab = b < 0 ? -b : b;
  if (gcd_small(a, ab) != 1) return 0;
  const int sr = (n - 1 - r) / a;
  const int sc = b > 0 ? (n - 1 - c) / b : c / ab;
  return 1 + min(sr, sc);
}

// Exclusive block scan of two values per thread; totals to *t0, *t1.
// `sm`: shared int64[2 * 32].
__device__ __forceinline__ void block_scan2(int64_t v0, int64_t v1, int64_t& e0, int64_t& e1, int64_t& t0,
                                            int64_t& t1, int64_t* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  int64_t x0 = v0, x1 = v1;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y0 = __shfl_up_sync(0xffffffffu, x0, o), y1 = __shfl_up_sync(0xffffffffu, x1, o);
    if (lane >= o) {
      x0 += y0;
      x1 += y1;
    }
  }
  if (lane == 31) {
    sm[warp] = x0;
    sm[32 + warp] = x1;
  }
  __syncthreads();
  if (warp == 0) {
    int64_t w0 = lane < warps ? sm[lane] : 0, w1 = lane < warps ? sm[32 + lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y0 = __shfl_up_sync(0xffffffffu, w0, o), y1 = __shfl_up_sync(0xffffffffu, w1, o);
      if (lane >= o) {
        w0 += y0;
        w1 += y1;
      }
    }
    if (lane < warps) {
      sm[lane] = w0;
      sm[32 + lane] = w1;
    }
  }
  __syncthreads();
  const int64_t b0 = warp > 0 ? sm[warp - 1] : 0, b1 = warp > 0 ? sm[32 + warp - 1] : 0;
  e0 = b0 + x0 - v0;
  e1 = b1 + x1 - v1;
  t0 = sm[warps - 1];
  t1 = sm[32 + warps - 1];
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads) count_kernel(int n, int64_t* __restrict__ line_at,
                                                         int64_t* __restrict__ incidence_at) {
  __shared__ int64_t sm[64];
  const int m0 = blockIdx.x, r = m0 / n, c = m0 - r * n;
  const int D = (n - 1) * (2 * n - 2);
  int64_t lines = 0, points = 0;
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    int a, b;
    step_of(d, n, a, b);
    const int k = line_length(r, c, a, b, n);
    lines += k > 0;
    points += k;
  }
  int64_t e0, e1, t0, t1;
  block_scan2(lines, points, e0, e1, t0, t1, sm);
  if (threadIdx.x == 0) {
    line_at[m0] = t0;
    incidence_at[m0] = t1;
  }
}

// In place, exclusive, over count + 1 entries of two int64 arrays (the last
// entry becomes the total).  One CTA of kScanThreads; each thread a run.
__global__ void __launch_bounds__(kScanThreads) scan_kernel(int count, int64_t* __restrict__ x0,
                                                            int64_t* __restrict__ x1) {
  __shared__ int64_t sm[64];
  const int per = (count + kScanThreads - 1) / kScanThreads;
  const int lo = min(count, (int)threadIdx.x * per), hi = min(count, lo + per);
  int64_t s0 = 0, s1 = 0;
  for (int i = lo; i < hi; ++i) {
    s0 += x0[i];
    s1 += x1[i];
  }
  int64_t e0, e1, t0, t1;
  block_scan2(s0, s1, e0, e1, t0, t1, sm);
  for (int i = lo; i < hi; ++i) {
    const int64_t v0 = x0[i], v1 = x1[i];
    x0[i] = e0;
    x1[i] = e1;
    e0 += v0;
    e1 += v1;
  }
  if (threadIdx.x == 0) {
    x0[count] = t0;
    x1[count] = t1;
  }
}

__global__ void __launch_bounds__(kThreads) emit_kernel(int n, const int64_t* __restrict__ line_at,
                                                        const int64_t* __restrict__ incidence_at,
                                                        int64_t* __restrict__ offsets, int32_t* __restrict__ indices) {
  __shared__ int64_t sm[64];
  const int N = n * n, m0 = blockIdx.x, r = m0 / n, c = m0 - r * n;
  const int D = (n - 1) * (2 * n - 2);
  int64_t line = line_at[m0], point = incidence_at[m0];
  for (int base = 0; base < D; base += blockDim.x) {  // uniform trip count
    const int d = base + (int)threadIdx.x;
    int a = 0, b = 0, k = 0;
    if (d < D) {
      step_of(d, n, a, b);
      k = line_length(r, c, a, b, n);
    }
    int64_t e0, e1, t0, t1;
    block_scan2(k > 0, k, e0, e1, t0, t1, sm);
    if (k > 0) {
      const int64_t at = point + e1;
      offsets[line + e0] = at;
      for (int t = 0; t < k; ++t) indices[at + t] = (r + t * a) * n + (c + t * b);
    }
    line += t0;
    point += t1;
  }
  if (m0 == N - 1 && threadIdx.x == 0) offsets[line_at[N]] = incidence_at[N];
}

__global__ void __launch_bounds__(kThreads) pairs_kernel(int n, int64_t line_count, const int64_t* __restrict__ offsets,
                                                         const int32_t* __restrict__ indices,
                                                         int32_t* __restrict__ pair_to_line) {
  const int64_t id = (int64_t)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (id >= line_count) return;
  const int lane = threadIdx.x & 31;
  const int64_t N = (int64_t)n * n, o = offsets[id];
  const int k = (int)(offsets[id + 1] - o);
  for (int i = 0; i + 1 < k; ++i) {
    const int64_t left = indices[o + i];
    for (int j = i + 1 + lane; j < k; j += 32) {
      const int64_t right = indices[o + j];  // > left: members ascend along the line
      pair_to_line[left * (2 * N - left - 1) / 2 + right - left - 1] = (int32_t)id;
    }
  }
}

// --------------------------------------------------------------------------
// score_pair_table: CTA per point list (at most kMaxPairPoints points).
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(kPairWarps * 32) pair_score_kernel(const int32_t* __restrict__ ids,
                                                                     const int64_t* __restrict__ starts, int n,
                                                                     const int32_t* __restrict__ pair_to_line,
                                                                     int64_t* __restrict__ scores,
                                                                     uint32_t* __restrict__ error_word) {
  __shared__ int32_t pts[kMaxPairPoints];
  __shared__ int32_t keys[kPairWarps][kHashSlots];
  __shared__ int32_t counts[kPairWarps][kHashSlots];
  __shared__ unsigned long long total;
  const int list = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t first = starts[list];
  const int64_t listed = starts[list + 1] - first;
  const int count = listed < kMaxPairPoints ? (int)listed : kMaxPairPoints;  // the host checks the size
  const int N = n * n;
  uint32_t err = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    const int v = ids[first + i];
    if (v < 0 || v >= N) err |= kErrPointRange;
    pts[i] = v;
  }
  for (int s = lane; s < kHashSlots; s += 32) {
    keys[warp][s] = -1;
    counts[warp][s] = 0;
  }
  if (threadIdx.x == 0) total = 0ull;
  __syncthreads();
  const int64_t NN = N;
  unsigned long long pairs = 0ull;
  for (int i = warp; i + 1 < count; i += kPairWarps) {  // anchor i, the points after it
    const int a = pts[i];
    for (int l = i + 1 + lane; l < count; l += 32) {
      const int b = pts[l];
      const int64_t lo = min(a, b), hi = max(a, b);
      if (lo == hi) {
        err |= kErrPointTwice;
        continue;
      }
      if (lo < 0 || hi >= NN) continue;  // reported above
      const int L = pair_to_line[lo * (2 * NN - lo - 1) / 2 + hi - lo - 1];
      if (L < 0) continue;
      unsigned h = ((unsigned)L * 2654435761u) >> (32 - 9);  // kHashSlots = 2^9
      bool placed = false;
      for (int probe = 0; probe < kHashSlots; ++probe) {
        const int prev = atomicCAS(&keys[warp][h], -1, L);
        if (prev == -1 || prev == L) {
          pairs += (unsigned long long)atomicAdd(&counts[warp][h], 1);
          placed = true;
          break;
        }
        h = (h + 1) & (kHashSlots - 1);
      }
      if (!placed) err |= kErrHashFull;
    }
    __syncwarp();
    for (int s = lane; s < kHashSlots; s += 32) {
      keys[warp][s] = -1;
      counts[warp][s] = 0;
    }
    __syncwarp();
  }
  if (pairs != 0ull) atomicAdd(&total, pairs);
  err = __reduce_or_sync(0xffffffffu, err);
  if (lane == 0 && err) atomicOr(error_word, err);
  __syncthreads();
  if (threadIdx.x == 0) scores[list] = (int64_t)total;
}

// --------------------------------------------------------------------------
// score_csr over 32 lists per occupancy word.
// --------------------------------------------------------------------------
// occupancy[g * N + id] bit s: list 32 g + s holds point id.
__global__ void occupancy_kernel(const int32_t* __restrict__ ids, const int64_t* __restrict__ starts, int lists,
                                 int n, uint32_t* __restrict__ occupancy, uint32_t* __restrict__ error_word) {
  const int list = blockIdx.x;
  if (list >= lists) return;
  const int N = n * n;
  const int64_t first = starts[list], last = starts[list + 1];
  uint32_t* occ = occupancy + (size_t)(list / kCsrLists) * N;
  const uint32_t bit = 1u << (list % kCsrLists);
  for (int64_t i = first + threadIdx.x; i < last; i += blockDim.x) {
    const int v = ids[i];
    if (v < 0 || v >= N) {
      atomicOr(error_word, kErrPointRange);
      continue;
    }
    atomicOr(&occ[v], bit);
  }
}

__device__ __forceinline__ int64_t c3(int64_t k) { return k * (k - 1) * (k - 2) / 6; }

// Grid: (line blocks, groups of 32 lists).  smem: the group's N occupancy words.
__global__ void __launch_bounds__(kThreads) csr_score_kernel(int n, int64_t line_count,
                                                             const int64_t* __restrict__ offsets,
                                                             const int32_t* __restrict__ indices,
                                                             const uint32_t* __restrict__ occupancy,
                                                             int64_t* __restrict__ scores) {
  extern __shared__ uint32_t occ[];  // [N]
  __shared__ unsigned long long part[kCsrLists];
  const int N = n * n, g = blockIdx.y;
  for (int i = threadIdx.x; i < N; i += blockDim.x) occ[i] = occupancy[(size_t)g * N + i];
  if (threadIdx.x < kCsrLists) part[threadIdx.x] = 0ull;
  __syncthreads();
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < line_count;
       id += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = offsets[id];
    const int k = (int)(offsets[id + 1] - o);
    uint32_t c0 = 0u, c1 = 0u, c2 = 0u, c3p = 0u, c4 = 0u, c5 = 0u, c6 = 0u;  // bit planes of 32 counts
    for (int t = 0; t < k; ++t) {
      uint32_t carry = occ[indices[o + t]], x;
      x = c0 & carry; c0 ^= carry; carry = x;
      x = c1 & carry; c1 ^= carry; carry = x;
      x = c2 & carry; c2 ^= carry; carry = x;
      x = c3p & carry; c3p ^= carry; carry = x;
      x = c4 & carry; c4 ^= carry; carry = x;
      x = c5 & carry; c5 ^= carry; carry = x;
      c6 ^= carry;  // counts stay below 128
    }
    uint32_t ge3 = c2 | c3p | c4 | c5 | c6 | (c1 & c0);
    while (ge3) {
      const int s = __ffs(ge3) - 1;
      ge3 &= ge3 - 1u;
      const int64_t cnt = ((c0 >> s) & 1u) | (((c1 >> s) & 1u) << 1) | (((c2 >> s) & 1u) << 2) |
                          (((c3p >> s) & 1u) << 3) | (((c4 >> s) & 1u) << 4) | (((c5 >> s) & 1u) << 5) |
                          (((c6 >> s) & 1u) << 6);
      atomicAdd(&part[s], (unsigned long long)c3(cnt));
    }
  }
  __syncthreads();
  if (threadIdx.x < kCsrLists && part[threadIdx.x] != 0ull)
    atomicAdd(reinterpret_cast<unsigned long long*>(&scores[(size_t)g * kCsrLists + threadIdx.x]),
              part[threadIdx.x]);
}

}  // namespace lines
}  // namespace n3

extern "C" {

int n3_line_tables_count(int n, int64_t* line_at, int64_t* incidence_at, int64_t* totals, void* stream) {
  if (n < 1 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "line tables: n=%d outside [1, %d]", n, N3_MAX_N);
  if (!line_at || !incidence_at || !totals) return n3host::set_error(N3_ERR_ARG, "line tables: null buffer");
  cudaStream_t st = (cudaStream_t)stream;
  const int N = n * n;
  if (n >= 3) {
    n3::lines::count_kernel<<<N, n3::lines::kThreads, 0, st>>>(n, line_at, incidence_at);
    N3_TRY(n3host::check_launch("line count_kernel"));
  } else if (cudaMemsetAsync(line_at, 0, sizeof(int64_t) * N, st) != cudaSuccess ||
             cudaMemsetAsync(incidence_at, 0, sizeof(int64_t) * N, st) != cudaSuccess) {
    return n3host::set_error(N3_ERR_CUDA, "line tables: memset failed");
  }
  n3::lines::scan_kernel<<<1, n3::lines::kScanThreads, 0, st>>>(N, line_at, incidence_at);
  N3_TRY(n3host::check_launch("line scan_kernel"));
  if (cudaMemcpyAsync(&totals[0], line_at + N, sizeof(int64_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(&totals[1], incidence_at + N, sizeof(int64_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return n3host::set_error(N3_ERR_CUDA, "line tables: reading the totals failed");
  return N3_OK;
}

int n3_line_tables_build(int n, const int64_t* line_at, const int64_t* incidence_at, int64_t line_count,
                         int64_t* offsets, int32_t* indices, int32_t* pair_to_line, void* stream) {
  if (n < 1 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "line tables: n=%d outside [1, %d]", n, N3_MAX_N);
  if (line_count < 0) return n3host::set_error(N3_ERR_ARG, "line tables: negative line count");
  const int64_t N = (int64_t)n * n, pairs = N * (N - 1) / 2;
  if (!line_at || !incidence_at || !offsets || (line_count > 0 && !indices) || (pairs > 0 && !pair_to_line))
    return n3host::set_error(N3_ERR_ARG, "line tables: null buffer");
  cudaStream_t st = (cudaStream_t)stream;
  if (pairs > 0 && cudaMemsetAsync(pair_to_line, 0xff, sizeof(int32_t) * pairs, st) != cudaSuccess)
    return n3host::set_error(N3_ERR_CUDA, "line tables: memset failed");
  if (line_count == 0) {
    if (cudaMemsetAsync(offsets, 0, sizeof(int64_t), st) != cudaSuccess)
      return n3host::set_error(N3_ERR_CUDA, "line tables: memset failed");
    return N3_OK;
  }
  n3::lines::emit_kernel<<<(int)N, n3::lines::kThreads, 0, st>>>(n, line_at, incidence_at, offsets, indices);
  N3_TRY(n3host::check_launch("line emit_kernel"));
  const int64_t blocks = (line_count + n3::lines::kThreads / 32 - 1) / (n3::lines::kThreads / 32);
  n3::lines::pairs_kernel<<<(unsigned)blocks, n3::lines::kThreads, 0, st>>>(n, line_count, offsets, indices,
                                                                           pair_to_line);
  return n3host::check_launch("line pairs_kernel");
}

int n3_lines_score_pairs(const int32_t* ids, const int64_t* starts, int lists, int n, const int32_t* pair_to_line,
                         int64_t* scores, uint32_t* error_word, void* stream) {
  if (n < 1 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "pair-table scores: n=%d outside [1, %d]", n,
                                                      N3_MAX_N);
  if (lists < 0) return n3host::set_error(N3_ERR_ARG, "pair-table scores: negative list count");
  if (lists == 0) return N3_OK;
  if (!ids || !starts || !scores || !error_word || (n > 1 && !pair_to_line))
    return n3host::set_error(N3_ERR_ARG, "pair-table scores: null buffer");
  n3::lines::pair_score_kernel<<<lists, n3::lines::kPairWarps * 32, 0, (cudaStream_t)stream>>>(
      ids, starts, n, pair_to_line, scores, error_word);
  return n3host::check_launch("pair_score_kernel");
}

int n3_lines_score_csr(const int32_t* ids, const int64_t* starts, int lists, int n, int64_t line_count,
                       const int64_t* offsets, const int32_t* indices, uint32_t* occupancy, int64_t* scores,
                       uint32_t* error_word, void* stream) {
  if (n < 1 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "CSR scores: n=%d outside [1, %d]", n, N3_MAX_N);
  if (lists < 0 || line_count < 0) return n3host::set_error(N3_ERR_ARG, "CSR scores: negative count");
  if (lists == 0) return N3_OK;
  if (!ids || !starts || !occupancy || !scores || !error_word || !offsets || (line_count > 0 && !indices))
    return n3host::set_error(N3_ERR_ARG, "CSR scores: null buffer");
  cudaStream_t st = (cudaStream_t)stream;
  const int N = n * n, groups = (lists + n3::lines::kCsrLists - 1) / n3::lines::kCsrLists;
  if (cudaMemsetAsync(occupancy, 0, sizeof(uint32_t) * (size_t)groups * N, st) != cudaSuccess ||
      cudaMemsetAsync(scores, 0, sizeof(int64_t) * (size_t)lists, st) != cudaSuccess)
    return n3host::set_error(N3_ERR_CUDA, "CSR scores: memset failed");
  n3::lines::occupancy_kernel<<<lists, 128, 0, st>>>(ids, starts, lists, n, occupancy, error_word);
  N3_TRY(n3host::check_launch("occupancy_kernel"));
  if (line_count == 0) return N3_OK;
  // a partial last group adds nothing past `lists`: its missing lists hold no points
  const int64_t want = (line_count + n3::lines::kThreads - 1) / n3::lines::kThreads;
  const int blocks = (int)(want < 4 * (int64_t)n3host::sm_count() ? want : 4 * (int64_t)n3host::sm_count());
  const size_t smem = sizeof(uint32_t) * N;
  n3::lines::csr_score_kernel<<<dim3(blocks, groups), n3::lines::kThreads, smem, st>>>(n, line_count, offsets,
                                                                                     indices, occupancy, scores);
  return n3host::check_launch("csr_score_kernel");
}

}  // extern "C"
