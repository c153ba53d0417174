// (a) Population scoring: exact collinear-triple counts, one warp per state.
//
// Two independent kernels and a fused, cross-checked one:
//
// * Determinant count (replaces src/no_three_75/gpu.py:13-42 and
//   src/no_three_75/gpu_device_search.py:118-161).  Every triple i<j<k is
//   tested once with an exact int32 cross product, at its middle slot j.  The
//   two slots of j's row are pivots together; the triple's other two points
//   lie in rows above and below that row.  The larger side sits in lane
//   registers, the smaller side is broadcast from shared memory one row (two
//   slots) at a time, so one pair of products serves four tests.  Triples
//   holding j's row partner are skipped: two points of a row and a third point
//   in another row are never collinear.
//
// * Normalised-slope line count (the counting form of
//   src/no_three_75/verifier_b.py:8-33).  For every anchor a, the other points
//   are binned by gcd-reduced undirected direction in an 8-bit shared-memory
//   histogram; sum over bins of C(c,2) is the anchor's badness and
//   E = sum(badness) / 3 (a line of k points gives each member C(k-1,2) pairs,
//   src/no_three_75/conflicts.py:373-378).  The gcd reduction is tabulated once
//   per device by build_dir_lut_kernel.
//
// * Checked scoring runs both per state and flags disagreement on device.
#include <cstdio>

#include "score_impl.cuh"

namespace n3 {

__device__ uint16_t g_dir_lut[kLutSize];
__device__ __align__(16) uint16_t g_dir_lut_full[kFullLutBytes / 2];
__device__ int g_dir_count;

__device__ __forceinline__ int gcd_dev(int a, int b) {
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b) {
    const int t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// Entry e = p * kLutW + (q + kMaxN - 1) names a primitive direction iff
// gcd(p, |q|) == 1 with p > 0, or (p, q) == (0, 1).
__device__ __forceinline__ bool is_primitive(int e) {
  const int p = e / kLutW, q = e % kLutW - (kMaxN - 1);
  return p == 0 ? q == 1 : gcd_dev(p, q) == 1;
}

// One block: numbers the primitive directions in (p, q) order, then maps every
// difference vector to the id of its gcd-reduced direction.
__global__ void __launch_bounds__(1024) build_dir_lut_kernel() {
  __shared__ uint16_t prim[kLutSize];
  __shared__ int scan[1024];
  const int tid = threadIdx.x;
  constexpr int per = (kLutSize + 1023) / 1024;
  const int lo = tid * per, hi = min(lo + per, kLutSize);
  int c = 0;
  for (int e = lo; e < hi; ++e) c += is_primitive(e);
  scan[tid] = c;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {  // inclusive Hillis-Steele scan
    const int v = tid >= off ? scan[tid - off] : 0;
    __syncthreads();
    scan[tid] += v;
    __syncthreads();
  }
  int id = scan[tid] - c;
  for (int e = lo; e < hi; ++e) prim[e] = is_primitive(e) ? (uint16_t)id++ : (uint16_t)0xFFFFu;
  if (tid == 1023) g_dir_count = scan[1023];
  __syncthreads();
  for (int e = tid; e < kLutSize; e += 1024) {
    const int dx = e / kLutW, dy = e % kLutW - (kMaxN - 1);
    const int g = gcd_dev(dx, dy);
    uint16_t v = 0xFFFFu;  // (0, 0) has no direction
    if (g) {
      const int p = dx / g;
      const int q = p == 0 ? 1 : dy / g;  // (0, -1) ~ (0, 1)
      v = prim[p * kLutW + q + (kMaxN - 1)];
    }
    g_dir_lut[e] = v;
  }
}

// The full signed table from the compact one (one entry per thread).
__global__ void build_full_lut_kernel() {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kFullLutSize) return;
  const int dx = e / kLutW - (kMaxN - 1), dy = e % kLutW - (kMaxN - 1);
  g_dir_lut_full[e] = (dx == 0 && dy == 0) ? (uint16_t)0 : (uint16_t)dir_id(g_dir_lut, dx, dy);
}

struct PQSource {
  const int32_t* p;
  const int32_t* q;
  __device__ __forceinline__ int col(int b, int n, int s) const {
    const size_t base = (size_t)b * n + (s >> 1);
    return (s & 1) ? q[base] : p[base];
  }
};

struct ColSource {
  const int16_t* c;
  __device__ __forceinline__ int col(int b, int n, int s) const { return c[(size_t)b * 2 * n + s]; }
};

constexpr int kDetWarps = 4;  // small CTAs: 4096 states spread evenly over 148 SMs

template <class Src, bool BAD>
__global__ void __launch_bounds__(kDetWarps * 32) det_kernel(Src src, int B, int n, int32_t* __restrict__ scores,
                                                               int32_t* __restrict__ badness) {
  __shared__ __align__(16) int cs_all[kDetWarps][kMaxM];
  __shared__ int bad_all[BAD ? kDetWarps : 1][BAD ? kMaxM : 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * kDetWarps + warp;
  if (b >= B) return;
  const int m = 2 * n;
  int* cs = cs_all[warp];
  int* bad = BAD ? bad_all[warp] : nullptr;
  for (int s = lane; s < m; s += 32) {
    cs[s] = src.col(b, n, s);
    if (BAD) bad[s] = 0;
  }
  __syncwarp();
  const int cnt = warp_sum(det_state<BAD>(cs, n, lane, bad));
  if (lane == 0) scores[b] = cnt;
  if (BAD) {
    __syncwarp();
    for (int s = lane; s < m; s += 32) badness[(size_t)b * m + s] = bad[s];
  }
}

// Loads one state, validating columns (range, row duplicates).  Returns the
// device error bits for this state (warp-uniform).
template <class Src>
__device__ __forceinline__ uint32_t load_checked(const Src& src, int b, int n, int* cs, int lane) {
  const int m = 2 * n;
  uint32_t err = 0;
  for (int s = lane; s < m; s += 32) {
    const int c = src.col(b, n, s);
    if (c < 0 || c >= n) err |= kErrColumnRange;
    cs[s] = min(max(c, 0), n - 1);
  }
  __syncwarp();
  for (int r = lane; r < n; r += 32)
    if (cs[2 * r] == cs[2 * r + 1]) err |= kErrDuplicate;
  err = __reduce_or_sync(0xffffffffu, err);
  return err;
}

// The slope count of every state with 4-bit histograms: W = blockDim.x / 32
// <= 32 warps share one direction table, a warp per state, each state loaded
// and validated (column range, row duplicates).  MODE 0: slope count only
// (scores, badness).  MODE 2: slope count and badness, checked against the
// determinant counts already in `scores` (written by det_kernel on the same
// stream).  MODE 3: the forward slope count of E only (slope_forward_state4),
// checked the same way (and, if `badness` is given, that badness checked to
// sum to 3E).  A state that may have overflowed a 4-bit counter is recounted
// by slope_state_halves in the same shared memory.
constexpr int kSlope4MaxWarps = 32;
__host__ __device__ constexpr size_t slope4_smem(int warps) {
  return kFullLutBytes + (size_t)warps * (sizeof(uint32_t) * kHist4Words + sizeof(int) * kMaxM * 2);
}

template <int MODE>
__global__ void __launch_bounds__(kSlope4MaxWarps * 32, 1) slope4_kernel(ColSource src, int B, int n,
                                                                          int32_t* __restrict__ scores,
                                                                          int32_t* __restrict__ badness,
                                                                          int32_t* __restrict__ mismatch,
                                                                          uint32_t* __restrict__ error_word) {
  static_assert(MODE == 0 || MODE == 2 || MODE == 3, "slope count only, or checked against determinant counts");
  extern __shared__ __align__(16) unsigned char smem[];
  const int W = blockDim.x >> 5;
  uint16_t* lut = reinterpret_cast<uint16_t*>(smem);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + kFullLutBytes);
  int* cs_all = reinterpret_cast<int*>(hist_all + kHist4Words * W);
  int* bad_all = cs_all + kMaxM * W;
  full_lut_copy(lut, g_dir_lut_full);
  for (int i = threadIdx.x; i < kHist4Words * W; i += blockDim.x) hist_all[i] = 0u;
  __syncthreads();
  if (threadIdx.x == 0) lut[kFullLutCentre] = (uint16_t)kDirCount;  // (0, 0): the centre's own counter
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m = 2 * n;
  int* cs = cs_all + warp * kMaxM;
  int* bad = bad_all + warp * kMaxM;
  uint32_t* hist = hist_all + warp * kHist4Words;
  for (int b = blockIdx.x * W + warp; b < B; b += gridDim.x * W) {
    const uint32_t err = load_checked(src, b, n, cs, lane);
    if (err) {  // invalid state: no count is meaningful
      if (lane == 0) {
        scores[b] = -1;
        if (error_word) atomicOr(error_word, err);
        if (MODE != 0) atomicAdd(mismatch, 1);
      }
      if (badness)
        for (int s = lane; s < m; s += 32) badness[(size_t)b * m + s] = -1;
      __syncwarp();
      continue;
    }
    bool overflow;
    if (MODE == 3) {  // forward count of E, compared with the determinant count (and badness, if given)
      int e_slope = slope_forward_state4(cs, n, lut, hist, lane, &overflow);
      if (overflow) {  // uniform
        __syncwarp();
        e_slope = slope_state_halves(cs, n, lut, hist, lane, nullptr) / 3;
      }
      int bad_sum = 0;
      if (badness)
        for (int s = lane; s < m; s += 32) bad_sum += badness[(size_t)b * m + s];
      bad_sum = warp_sum(bad_sum);
      const int e_det = scores[b];
      if (lane == 0 && (e_slope != e_det || (badness && bad_sum != 3 * e_det))) {
        atomicAdd(mismatch, 1);
        if (error_word) atomicOr(error_word, kErrMismatch);
      }
      __syncwarp();
      continue;
    }
    int total = slope_state4(cs, n, lut, hist, lane, bad, &overflow);
    if (overflow) {  // uniform
      __syncwarp();
      total = slope_state_halves(cs, n, lut, hist, lane, bad);
    }
    __syncwarp();
    if (MODE == 0) {
      if (lane == 0) scores[b] = total / 3;
    } else {  // scores[b] holds the determinant count of this state
      if (lane == 0 && total != 3 * scores[b]) {
        atomicAdd(mismatch, 1);
        if (error_word) atomicOr(error_word, kErrMismatch);
      }
    }
    if (badness)
      for (int s = lane; s < m; s += 32) badness[(size_t)b * m + s] = bad[s];
    __syncwarp();
  }
}

}  // namespace n3

namespace n3host {

int build_dir_lut(cudaStream_t st) {
  n3::build_dir_lut_kernel<<<1, 1024, 0, st>>>();
  N3_TRY(check_launch("build_dir_lut_kernel"));
  n3::build_full_lut_kernel<<<(n3::kFullLutSize + 255) / 256, 256, 0, st>>>();
  N3_TRY(check_launch("build_full_lut_kernel"));
  int count = 0;
  if (cudaMemcpyFromSymbolAsync(&count, n3::g_dir_count, sizeof(int), 0, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return check_launch("direction table read-back");
  if (count != n3::kDirCount)
    return set_error(N3_ERR_CUDA, "direction table has %d ids, expected %d", count, n3::kDirCount);
  return N3_OK;
}

const uint16_t* dir_lut_device_ptr() {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, n3::g_dir_lut) != cudaSuccess) return nullptr;
  return static_cast<const uint16_t*>(p);
}

const uint16_t* dir_lut_full_device_ptr() {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, n3::g_dir_lut_full) != cudaSuccess) return nullptr;
  return static_cast<const uint16_t*>(p);
}

static int check_common(int B, int n, const void* a, const void* out) {
  if (n < 2 || n > N3_MAX_N) return set_error(N3_ERR_RANGE, "n=%d outside [2, %d]", n, N3_MAX_N);
  if (B < 0) return set_error(N3_ERR_ARG, "negative batch size %d", B);
  if (B > 0 && (a == nullptr || out == nullptr)) return set_error(N3_ERR_ARG, "null device pointer");
  return N3_OK;
}

int prepare_score() {
  N3_TRY(allow_smem(reinterpret_cast<const void*>(n3::slope4_kernel<0>), n3::slope4_smem(n3::kSlope4MaxWarps)));
  N3_TRY(allow_smem(reinterpret_cast<const void*>(n3::slope4_kernel<2>), n3::slope4_smem(n3::kSlope4MaxWarps)));
  return allow_smem(reinterpret_cast<const void*>(n3::slope4_kernel<3>), n3::slope4_smem(n3::kSlope4MaxWarps));
}

template <class Src>
static int launch_det(Src src, int B, int n, int32_t* scores, int32_t* badness, cudaStream_t st) {
  if (B == 0) return N3_OK;
  const int grid = (B + n3::kDetWarps - 1) / n3::kDetWarps;
  if (badness)
    n3::det_kernel<Src, true><<<grid, n3::kDetWarps * 32, 0, st>>>(src, B, n, scores, badness);
  else
    n3::det_kernel<Src, false><<<grid, n3::kDetWarps * 32, 0, st>>>(src, B, n, scores, nullptr);
  return check_launch("det_kernel");
}

// The 4-bit slope kernel: one CTA per SM of W warps, W = ceil(B / SMs) up to
// 32, so that 4096 states are one state per warp on 147 SMs.
template <int MODE>
static int launch_slope4(const int16_t* cols, int B, int n, int32_t* scores, int32_t* badness, int32_t* mismatch,
                         uint32_t* error_word, cudaStream_t st) {
  if (B == 0) return N3_OK;
  N3_TRY(ensure_device_tables());
  N3_TRY(allow_smem(reinterpret_cast<const void*>(n3::slope4_kernel<MODE>), n3::slope4_smem(n3::kSlope4MaxWarps)));
  const int sms = sm_count();
  int W = (B + sms - 1) / sms;
  W = W < 1 ? 1 : (W > n3::kSlope4MaxWarps ? n3::kSlope4MaxWarps : W);
  const int blocks_needed = (B + W - 1) / W;
  const int grid = blocks_needed < sms ? blocks_needed : sms;
  n3::slope4_kernel<MODE><<<grid, W * 32, n3::slope4_smem(W), st>>>(n3::ColSource{cols}, B, n, scores, badness,
                                                                    mismatch, error_word);
  return check_launch("slope4_kernel");
}

}  // namespace n3host

extern "C" {

int n3_score_population(const int32_t* p, const int32_t* q, int B, int n, int32_t* scores, int32_t* badness,
                        void* stream) {
  N3_TRY(n3host::check_common(B, n, p, scores));
  if (B > 0 && q == nullptr) return n3host::set_error(N3_ERR_ARG, "null Q pointer");
  return n3host::launch_det(n3::PQSource{p, q}, B, n, scores, badness, (cudaStream_t)stream);
}

int n3_score_columns(const int16_t* cols, int B, int n, int32_t* scores, int32_t* badness, void* stream) {
  N3_TRY(n3host::check_common(B, n, cols, scores));
  return n3host::launch_det(n3::ColSource{cols}, B, n, scores, badness, (cudaStream_t)stream);
}

int n3_score_slope(const int16_t* cols, int B, int n, int32_t* scores, int32_t* badness, void* stream) {
  N3_TRY(n3host::check_common(B, n, cols, scores));
  return n3host::launch_slope4<0>(cols, B, n, scores, badness, nullptr, nullptr, (cudaStream_t)stream);
}

int n3_score_checked(const int16_t* cols, int B, int n, int32_t* scores, int32_t* badness, int32_t* mismatch,
                     uint32_t* error_word, void* stream) {
  N3_TRY(n3host::check_common(B, n, cols, scores));
  if (B > 0 && mismatch == nullptr) return n3host::set_error(N3_ERR_ARG, "null mismatch counter");
  // Two launches on one stream: the determinant count at full occupancy, then
  // the independent slope count, which validates each state and compares.  With
  // badness wanted, the full slope count provides it (the determinant kernel's
  // own badness output costs it 70 % more time than the whole slope pass);
  // without, the forward slope count checks E at 3/4 of the cost.
  N3_TRY(n3host::launch_det(n3::ColSource{cols}, B, n, scores, nullptr, (cudaStream_t)stream));
  if (badness)
    return n3host::launch_slope4<2>(cols, B, n, scores, badness, mismatch, error_word, (cudaStream_t)stream);
  return n3host::launch_slope4<3>(cols, B, n, scores, nullptr, mismatch, error_word, (cudaStream_t)stream);
}

}  // extern "C"
