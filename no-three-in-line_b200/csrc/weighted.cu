// Line-weighted energies of breakout search (src/no_three_75/breakout.py:39-81):
// a weighted line L = (a, b, c) (points with a*row + b*col + c == 0) of weight
// w > 1 adds (w - 1) * C(occupancy, 3) to the triple count E.
//   weighted_switch_kernel  weighted_candidate_scores: for a selected slot u and
//                           every partner v, the weighted score after swapping
//                           the columns of u and v, from the raw score of that
//                           move (breakout.py:39-75)
//   weighted_state_kernel   weighted_state_score over a population (:78-86)
// Occupancies are counted exactly in 64-bit arithmetic (the line keys are
// caller data and may be large).
#include <stdint.h>

#include "n3_common.cuh"

namespace n3 {
namespace weighted {

constexpr int kThreads = 256;

__device__ __forceinline__ int64_t c3(int64_t k) { return k >= 3 ? k * (k - 1) * (k - 2) / 6 : 0; }

__device__ __forceinline__ bool on_line(const int32_t* L, int row, int col) {
  return (int64_t)L[0] * row + (int64_t)L[1] * col + (int64_t)L[2] == 0;
}

// One CTA.  smem: rows/cols of the 2n slots, per line its occupancy and whether
// slot u lies on it.
__global__ void __launch_bounds__(kThreads) weighted_switch_kernel(const int32_t* __restrict__ p,
                                                                   const int32_t* __restrict__ q, int n, int u,
                                                                   const int64_t* __restrict__ raw,
                                                                   const int32_t* __restrict__ lines,
                                                                   const int32_t* __restrict__ weights, int nl,
                                                                   int64_t* __restrict__ out) {
  extern __shared__ int32_t sm[];
  int32_t* col = sm;            // [2n]
  int32_t* occ = col + 2 * n;   // [nl]
  int32_t* on_u = occ + nl;     // [nl]
  const int m = 2 * n;
  for (int s = threadIdx.x; s < m; s += blockDim.x) col[s] = (s & 1) ? q[s >> 1] : p[s >> 1];
  __syncthreads();
  for (int l = threadIdx.x; l < nl; l += blockDim.x) {
    const int32_t* L = lines + 3 * l;
    int k = 0;
    for (int s = 0; s < m; ++s) k += on_line(L, s >> 1, col[s]);
    occ[l] = k;
    on_u[l] = on_line(L, u >> 1, col[u]);
  }
  __syncthreads();
  const int ru = u >> 1, cu = col[u];
  for (int v = threadIdx.x; v < m; v += blockDim.x) {
    const int rv = v >> 1, cv = col[v];
    int64_t extra = 0;
    for (int l = 0; l < nl; ++l) {
      const int w = weights[l];
      if (w <= 1) continue;
      const int32_t* L = lines + 3 * l;
      // occupancy after u -> (ru, cv) and v -> (rv, cu), counted as the reference does
      const int64_t k = (int64_t)occ[l] - on_u[l] - on_line(L, rv, cv) + on_line(L, ru, cv) + on_line(L, rv, cu);
      extra += (int64_t)(w - 1) * c3(k);
    }
    out[v] = raw[v] + extra;
  }
}

// Warp per state.
__global__ void __launch_bounds__(kThreads) weighted_state_kernel(const int32_t* __restrict__ p,
                                                                  const int32_t* __restrict__ q, int B, int n,
                                                                  const int64_t* __restrict__ raw,
                                                                  const int32_t* __restrict__ lines,
                                                                  const int32_t* __restrict__ weights, int nl,
                                                                  int64_t* __restrict__ out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= B) return;
  const int32_t* P = p + (size_t)warp * n;
  const int32_t* Q = q + (size_t)warp * n;
  int64_t extra = 0;
  for (int l = lane; l < nl; l += 32) {
    const int w = weights[l];
    if (w <= 1) continue;
    const int32_t* L = lines + 3 * l;
    int k = 0;
    for (int r = 0; r < n; ++r) k += on_line(L, r, P[r]) + on_line(L, r, Q[r]);
    extra += (int64_t)(w - 1) * c3(k);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) extra += __shfl_xor_sync(0xffffffffu, extra, o);
  if (lane == 0) out[warp] = raw[warp] + extra;
}

}  // namespace weighted
}  // namespace n3

extern "C" {

int n3_weighted_switch_scores(const int32_t* p, const int32_t* q, int n, int u, const int64_t* raw,
                              const int32_t* lines, const int32_t* weights, int n_lines, int64_t* scores,
                              void* stream) {
  if (n < 2 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "weighted scores: n=%d outside [2, %d]", n,
                                                      N3_MAX_N);
  if (u < 0 || u >= 2 * n) return n3host::set_error(N3_ERR_RANGE, "weighted scores: slot %d outside [0, %d)", u,
                                                    2 * n);
  if (n_lines < 0 || n_lines > 4096) return n3host::set_error(N3_ERR_RANGE, "weighted scores: 0..4096 lines");
  if (!p || !q || !raw || !scores || (n_lines > 0 && (!lines || !weights)))
    return n3host::set_error(N3_ERR_ARG, "weighted scores: null buffer");
  const size_t smem = sizeof(int32_t) * (2 * n + 2 * (size_t)n_lines);
  n3::weighted::weighted_switch_kernel<<<1, n3::weighted::kThreads, smem, (cudaStream_t)stream>>>(
      p, q, n, u, raw, lines, weights, n_lines, scores);
  return n3host::check_launch("weighted_switch_kernel");
}

int n3_weighted_state_scores(const int32_t* p, const int32_t* q, int B, int n, const int64_t* raw,
                             const int32_t* lines, const int32_t* weights, int n_lines, int64_t* scores,
                             void* stream) {
  if (n < 2 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "weighted scores: n=%d outside [2, %d]", n,
                                                      N3_MAX_N);
  if (B < 0 || n_lines < 0) return n3host::set_error(N3_ERR_ARG, "weighted scores: negative count");
  if (B == 0) return N3_OK;
  if (!p || !q || !raw || !scores || (n_lines > 0 && (!lines || !weights)))
    return n3host::set_error(N3_ERR_ARG, "weighted scores: null buffer");
  const int warps_per_block = n3::weighted::kThreads / 32;
  n3::weighted::weighted_state_kernel<<<(B + warps_per_block - 1) / warps_per_block, n3::weighted::kThreads, 0,
                                        (cudaStream_t)stream>>>(p, q, B, n, raw, lines, weights, n_lines, scores);
  return n3host::check_launch("weighted_state_kernel");
}

}  // extern "C"
