// (d) Learned move proposal: a 192 -> 256 -> 256 -> 1 MLP (bf16 weights,
// fp32 accumulation) that ranks candidate swaps by predicted dE, trained online
// on (features, exact dE) tuples emitted by the run.  No reference counterpart
// (the reference proposes uniformly, src/no_three_75/tempering.py:50-56).
//
// Features of a candidate (u, v) of a chain, all float, 192 wide:
//   [0..3]    badness of u, v, u^1, v^1, / 16
//   [4..7]    rows of u, v, u^1, v^1, / n
//   [8..11]   columns of u, v, u^1, v^1, / n
//   [12..161] the chain's per-slot badness (150 slots, zero beyond 2n), / 16
//   [162..191] zero
// Layer 1 is split accordingly: W1 = [W1a | W1b].  The 150 chain features are
// shared by all 128 candidates of a chain, so the chain part c1 = W1b x + b1 is
// computed once per chain (a tcgen05 GEMM after candidates_kernel, bf16
// operands as in the training forward) and enters the
// per-candidate K = 16 tensor-core product through two constant-1 columns of
// A1 (k = 12, 13) against c1 split into bf16 high and low parts (B columns
// 12, 13; c1 = hi + lo to about 2^-17 relative).  Inference per chain is one
// M = 128 tile:
//   D1 = A1 (128 x 16) [W1a | hi | lo]^T  -> ReLU, bf16 -> A2 (shared memory)
//   D2 = A2 (128 x 256) W2^T              -> + b2, ReLU, . w3 + b3 -> predicted dE
// both on tcgen05 with fp32 accumulators in tensor memory.
// Training uses MSE on dE / kTargetScale with Adam: the five GEMMs of a step
// (two forward layers, two weight gradients, the backward through layer 2) run
// on tcgen05 with bf16 operands and fp32 accumulators (tc_gemm_kernel), the
// head, bias gradients and Adam in fp32 SIMT; the packed bf16 images are
// rebuilt after each update.  fp32 master weights.
#include <cuda.h>
#include <cuda_bf16.h>
#include <mutex>
#include <math.h>

#include "chain_move.cuh"
#include "dirs.cuh"
#include "n3_common.cuh"
#include "philox.cuh"
#include "umma.cuh"

namespace n3 {
namespace mlp {

constexpr int kCand = 128;    // candidates per chain per step (one M tile)
constexpr int kIn = 192;      // input width
constexpr int kCandFeat = 12; // per-candidate features (A1 columns 12 and 13 hold 1.0)
constexpr int kChainFeat = 150;
constexpr int kH = 256;
constexpr float kTargetScale = 16.0f;
// Parameter buffer layout (fp32): W1 [256][192], b1, W2 [256][256], b2, w3, b3.
constexpr int oW1 = 0;
constexpr int oB1 = oW1 + kH * kIn;
constexpr int oW2 = oB1 + kH;
constexpr int oB2 = oW2 + kH * kH;
constexpr int oW3 = oB2 + kH;
constexpr int oB3 = oW3 + kH;
constexpr int kParams = oB3 + 4;  // padded to a multiple of 4

// Inference shared-memory map (offsets from a 1024-aligned base).  A1 and the
// chain part have three buffers: tile i + 2 loads while tile i is processed.
constexpr uint32_t sW2 = 0;                        // SW128 image, 4 x [256 x 128 B]
constexpr uint32_t sA2 = sW2 + 4 * kH * 128;       // SW128, 4 x [128 x 128 B]
constexpr uint32_t sW1a = sA2 + 4 * kCand * 128;   // INTERLEAVE K=16, 256 rows: W1a | c1 hi | c1 lo | 0
constexpr int kStages = 3;
constexpr uint32_t sA1 = sW1a + kH * 32;           // 3 x INTERLEAVE K=16, 128 rows
constexpr uint32_t sC1 = sA1 + kStages * kCand * 32;  // 3 x fp32[256] chain part of layer 1
constexpr uint32_t sB2 = sC1 + kStages * kH * 4;
constexpr uint32_t sW3 = sB2 + kH * 4;
constexpr uint32_t sPart = sW3 + kH * 4;           // fp32[2][2][128] half dot products
constexpr uint32_t sBar = sPart + 4 * kCand * 4;   // 9 mbarriers, TMEM address, abort flag
constexpr uint32_t kInferSmem = sBar + 128 + 1024; // + alignment slack
constexpr int kGroupThreads = 256;                 // a warp group: 2 warps per tensor-memory lane quarter
constexpr int kInferThreads = 2 * kGroupThreads;
constexpr uint32_t kWaitTries = 1u << 24;

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<const uint16_t*>(&h);
}

// ReLU of two floats rounded to bf16 (round-to-nearest-even) and packed, a in
// bits 0-15, b in 16-31: one paired conversion, then a paired bf16 max with 0
// (rounding keeps the sign, so ReLU after rounding equals rounding after ReLU).
__device__ __forceinline__ uint32_t relu_bf16x2_bits(float a, float b) {
  const __nv_bfloat162 h = __hmax2(__floats2bfloat162_rn(a, b), __float2bfloat162_rn(0.f));
  return *reinterpret_cast<const uint32_t*>(&h);
}

// Two floats rounded to bf16 in one conversion: lo in bits 0-15, hi in 16-31.
__device__ __forceinline__ uint32_t bf16x2_bits(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// ---------------------------------------------------------------------------
// Packing: fp32 parameters -> bf16 tensor-core images + transposed W1b.
// ---------------------------------------------------------------------------
__global__ void pack_kernel(const float* __restrict__ P, uint8_t* __restrict__ w2_img, uint8_t* __restrict__ w1a_img) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  for (int i = tid; i < kH * kH; i += stride) {  // W2[n][k]: row n of the B operand, K index k
    const int n = i / kH, k = i % kH;
    *reinterpret_cast<uint16_t*>(w2_img + umma::sw128_offset(n, k, kH)) = bf16_bits(P[oW2 + n * kH + k]);
  }
  for (int i = tid; i < kH * 16; i += stride) {
    const int n = i / 16, k = i % 16;
    const float w = k < kCandFeat ? P[oW1 + n * kIn + k] : 0.0f;
    *reinterpret_cast<uint16_t*>(w1a_img + umma::inter16_offset(n, k)) = bf16_bits(w);
  }
}

// ---------------------------------------------------------------------------
// Candidates: per chain, 128 Philox-drawn (u, v) slot pairs and their features
// as the INTERLEAVE A1 image, plus the chain's scaled badness row (the input
// of the chain part of layer 1, computed for all chains by one GEMM).
// ---------------------------------------------------------------------------
struct CandArgs {
  const int16_t* cols;     // [C][150]
  const int32_t* badness;  // [C][150]
  const int32_t* ladder_n; // [C/L]
  int ladder_size, n_chains;
  uint8_t* a1_img;         // [C][128 rows x 32 B]
  float* badn;             // [C][150] badness / 16
  int32_t* cand;           // [C][128]: u | v << 8 | legal << 31
  const uint64_t* step;    // device step counter
  uint32_t k0, k1;
  int bad_bias;            // percent of candidates with a badness-weighted slot u
};

template <class ColT, class BadT>
__device__ __forceinline__ void candidate_features(const ColT* cols, const BadT* bad, int n, int u, int v,
                                                   float (&f)[kCandFeat]) {
  const float inv_n = 1.0f / (float)n;
  const int s[4] = {u, v, u ^ 1, v ^ 1};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    f[i] = (float)bad[s[i]] * (1.0f / 16.0f);
    f[4 + i] = (float)(s[i] >> 1) * inv_n;
    f[8 + i] = (float)cols[s[i]] * inv_n;
  }
}

__global__ void __launch_bounds__(kCand) candidates_kernel(const CandArgs A) {
  __shared__ int s_cols[kChainFeat], s_bad[kChainFeat], s_pre[kChainFeat];
  const int c = blockIdx.x;
  const int n = A.ladder_n[c / A.ladder_size], m = 2 * n;
  for (int s = threadIdx.x; s < kChainFeat; s += blockDim.x) {
    const int b = A.badness[(size_t)c * kChainFeat + s];
    s_cols[s] = A.cols[(size_t)c * kChainFeat + s];
    s_bad[s] = b;
    A.badn[(size_t)c * kChainFeat + s] = s < m ? (float)b * (1.0f / 16.0f) : 0.f;
  }
  __syncthreads();
  if (A.bad_bias > 0 && threadIdx.x < 32) {  // running badness sums (warp 0, five slots a lane)
    const int lane = threadIdx.x, s0 = lane * kSlotsPerLane;
    int val[kSlotsPerLane], local = 0;
#pragma unroll
    for (int t = 0; t < kSlotsPerLane; ++t) {
      val[t] = s0 + t < m ? s_bad[s0 + t] : 0;
      local += val[t];
    }
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    int run = incl - local;
#pragma unroll
    for (int t = 0; t < kSlotsPerLane; ++t) {
      run += val[t];
      if (s0 + t < m) s_pre[s0 + t] = run;
    }
  }
  __syncthreads();
  const int j = threadIdx.x;
  const uint64_t step = *A.step;
  const U4 r = philox4x32_10(U4{(uint32_t)step, (uint32_t)(step >> 32), (uint32_t)c, kTagCandidate | (uint32_t)j},
                             A.k0, A.k1);
  int u = (int)__umulhi(r.x, (unsigned)m);
  const int v = (int)__umulhi(r.y, (unsigned)m);
  if (A.bad_bias > 0) {
    // the reference walk's badness-weighted u (tempering.py:51-55): the first
    // slot whose running badness sum exceeds a uniform integer below 3E
    const int total = s_pre[m - 1];
    if (total > 0 && __umulhi(r.z, 100u) < (unsigned)A.bad_bias) {
      const int target = (int)__umulhi(r.w, (unsigned)total);
      int lo = 0, hi = m - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (s_pre[mid] > target)
          hi = mid;
        else
          lo = mid + 1;
      }
      u = lo;
    }
  }
  const int cu = s_cols[u], cv = s_cols[v];
  const bool legal = (u >> 1) != (v >> 1) && cu != cv && s_cols[u ^ 1] != cv && s_cols[v ^ 1] != cu;
  float f[kCandFeat];
  candidate_features(s_cols, s_bad, n, u, v, f);
  // row j of the INTERLEAVE image: K 0-7 and K 8-15 are two 16-byte core-matrix rows
  uint8_t* img = A.a1_img + (size_t)c * (kCand * 32);
  const uint4 lo = make_uint4(bf16x2_bits(f[0], f[1]), bf16x2_bits(f[2], f[3]), bf16x2_bits(f[4], f[5]),
                              bf16x2_bits(f[6], f[7]));
  const uint4 hi = make_uint4(bf16x2_bits(f[8], f[9]), bf16x2_bits(f[10], f[11]), bf16x2_bits(1.0f, 1.0f), 0u);
  *reinterpret_cast<uint4*>(img + umma::inter16_offset(j, 0)) = lo;
  *reinterpret_cast<uint4*>(img + umma::inter16_offset(j, 8)) = hi;
  A.cand[(size_t)c * kCand + j] = u | (v << 8) | (legal ? (1 << 31) : 0);
}

// ---------------------------------------------------------------------------
// Tensor-core inference: one persistent CTA per SM, 4 warps, one chain tile
// (128 candidates) per iteration.
// ---------------------------------------------------------------------------
struct InferArgs {
  const uint8_t* a1_img;  // [T][4096 B]
  const float* c1;        // [T][256]
  const uint8_t* w2_img;  // 128 KB
  const uint8_t* w1a_img; // 8 KB
  const float* P;         // b2, w3, b3
  float* pred;            // [T][128]
  int tiles;
  uint32_t* error_word;
};

__device__ __forceinline__ void copy16(uint8_t* dst, const uint8_t* src, int bytes, int tid, int nthreads) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(dst);
  for (int i = tid; i < bytes / 16; i += nthreads) d[i] = s[i];
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t saddr, const void* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// All but the most recent group have landed.
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Prefetch of tile t's candidate features (4 KB) and chain part (1 KB) by
// `nthreads` >= 256 threads, as one cp.async group (committed, empty when t is
// past the last tile, so that every thread's group count stays in step).
// Thread j < 256 copies chain-part float j itself.
__device__ __forceinline__ void load_tile_async(uint32_t base, int buf, const InferArgs& A, int t, int tid,
                                                int nthreads) {
  if (t < A.tiles) {
    const uint8_t* a1 = A.a1_img + (size_t)t * (kCand * 32);
    const uint32_t sa = base + sA1 + (uint32_t)buf * (kCand * 32);
    for (int i = tid; i < kCand * 32 / 16; i += nthreads) cp_async16(sa + 16 * i, a1 + 16 * i);
    if (tid < kH) cp_async4(base + sC1 + (uint32_t)buf * (kH * 4) + 4 * tid, A.c1 + (size_t)t * kH + tid);
  }
  cp_async_commit();
}

// Writes chain part value c of B row n into columns 12 (bf16 high part) and 13
// (bf16 low part) of the layer-1 B operand.
__device__ __forceinline__ void put_chain_part(uint8_t* sm, int n, float c) {
  const float hi = __bfloat162float(__float2bfloat16_rn(c));
  *reinterpret_cast<uint32_t*>(sm + sW1a + umma::inter16_offset(n, kCandFeat)) = bf16x2_bits(hi, c - hi);
}

// Barrier of one warp group (named barrier ID, kGroupThreads threads) that
// also ORs a flag over the group, so that the group leaves its loop together.
template <int ID>
__device__ __forceinline__ bool group_sync_or(bool v) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "barrier.cta.red.or.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(out)
      : "r"((uint32_t)v), "n"(ID), "n"(kGroupThreads)
      : "memory");
  return out != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t saddr) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(saddr) : "memory");
}

// Layer-2 product of one tile: D (+)= A2 (128 x 256) W2^T, sixteen K = 16 steps.
__device__ __forceinline__ void issue_layer2(uint32_t base, uint32_t d, uint32_t idesc) {
#pragma unroll
  for (int s = 0; s < kH / 16; ++s) {
    const uint32_t koff = (uint32_t)(s & 3) * 32u;  // K = 16 step inside a 64-wide slice
    const uint64_t ad = umma::desc_sw128(base + sA2 + (uint32_t)(s >> 2) * (kCand * 128) + koff);
    const uint64_t bd = umma::desc_sw128(base + sW2 + (uint32_t)(s >> 2) * (kH * 128) + koff);
    umma::mma_bf16(d, ad, bd, idesc, s > 0 ? 1u : 0u);
  }
}

__device__ __forceinline__ void issue_layer1(uint32_t base, int a1buf, uint32_t d, uint32_t idesc) {
  const uint32_t a1 = base + sA1 + (uint32_t)a1buf * (kCand * 32);
  umma::mma_bf16(d, umma::desc_interleave(a1, 128, 256), umma::desc_interleave(base + sW1a, 128, 256), idesc, 0u);
}

// Per CTA: tiles t_i = blockIdx.x + i * gridDim.x.  Tensor memory holds two
// 256-column accumulators; tile i uses buffer i & 1 first for its layer-1
// product D1 and then, once D1 has been read, for its layer-2 product D2.
// Warp group 1 (warps 0-7) runs epilogue 1 (D1 + chain part, ReLU, bf16 into
// the A2 operand); its thread 0 issues the layer-2 MMAs and thread 32 the
// layer-1 MMAs (each tracks its own MMAs with tcgen05.commit).  Warp group 2
// (warps 8-15) runs epilogue 2 (ReLU(D2 + b2) . w3).  Per tile:
//   MMA1(i) done, MMA2(i-1) done (A2 free)  -> group 1: epilogue 1(i) -> MMA2(i)
//   MMA2(i) done                            -> group 2: epilogue 2(i) -> frees buffer i & 1
//   epilogue 2(i-1) done                    -> MMA1(i+1) into buffer (i+1) & 1
//   epilogue 1(i+1) done                    -> group 2 starts epilogue 2(i)
// so epilogue 2 of tile i runs beside the layer-2 MMAs of tile i+1, and
// epilogue 1, which the tensor core waits for, has the SM's issue slots alone.
// In each group, warp w reads tensor-memory lanes 32 (w % 4) .. (its quarter of
// the 128 rows), columns 128 ((w / 4) % 2) ..: each thread owns one row and
// half of the 256 columns.
__global__ void __launch_bounds__(kInferThreads, 1) infer_kernel(const InferArgs A) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = umma::smem_addr(smem_raw);
  uint8_t* sm = smem_raw + ((1024u - (raw & 1023u)) & 1023u);  // 1024-aligned base
  const uint32_t base = umma::smem_addr(sm);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int group = warp >> 3, quarter = warp & 3, colhalf = (warp >> 2) & 1;
  const int gtid = tid & (kGroupThreads - 1);
  float* b2s = reinterpret_cast<float*>(sm + sB2);
  float* w3s = reinterpret_cast<float*>(sm + sW3);
  float* part = reinterpret_cast<float*>(sm + sPart);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + sBar + 80);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + sBar + 88);
  // mbarriers: MMA1 done [2], MMA2 done [2], epilogue 2 done [2], final drain, epilogue 1 done [2]
  const uint32_t barM1 = base + sBar, barM2 = base + sBar + 16, barE2 = base + sBar + 32, barFin = base + sBar + 48;
  const uint32_t barE1 = base + sBar + 56;
  const int G = gridDim.x;

  load_tile_async(base, 0, A, blockIdx.x, tid, kInferThreads);
  load_tile_async(base, 1, A, blockIdx.x + gridDim.x, tid, kInferThreads);
  copy16(sm + sW2, A.w2_img, 4 * kH * 128, tid, kInferThreads);
  copy16(sm + sW1a, A.w1a_img, kH * 32, tid, kInferThreads);
  for (int i = tid; i < kH; i += kInferThreads) {
    b2s[i] = A.P[oB2 + i];
    w3s[i] = A.P[oW3 + i];
  }
  const float b3 = A.P[oB3];
  cp_async_wait_all();
  __syncthreads();  // the W1a image is in place before its chain-part columns are written
  if (tid < kH && blockIdx.x < A.tiles)  // this thread's own copy of tile 0's chain part
    put_chain_part(sm, tid, reinterpret_cast<const float*>(sm + sC1)[tid]);
  if (warp == 0) {
    umma::tmem_alloc(base + sBar + 80, 512);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    for (int k = 0; k < 2; ++k) {
      umma::mbar_init(barM1 + 8 * k, 1);
      umma::mbar_init(barM2 + 8 * k, 1);
      umma::mbar_init(barE2 + 8 * k, kGroupThreads);
      umma::mbar_init(barE1 + 8 * k, 1);
    }
    umma::mbar_init(barFin, 2);  // threads 0 and 32 each commit their MMAs
    umma::mbar_fence_init();
    *abort_flag = 0;
  }
  cp_async_wait_all();
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_off = (uint32_t)(32 * quarter) << 16;
  const uint32_t idesc = umma::idesc_bf16_f32(128, 256);
  const int row = 32 * quarter + lane;
  const int sl0 = 2 * colhalf;  // this thread's two K = 64 slices / column blocks
  if (tid == 0 && blockIdx.x < A.tiles) {
    issue_layer1(base, 0, tmem, idesc);
    umma::commit(barM1);
  }

  if (group == 0) {
    // ---- warp group 1: epilogue 1 and the MMA issue ----
    for (int i = 0, t = blockIdx.x; t < A.tiles; ++i, t += G) {
      const int b = i & 1;
      const uint32_t d = tmem + 256u * (uint32_t)b;
      const bool has_next = t + G < A.tiles;
      const int next_stage = (i + 1) % kStages;
      // tile i + 2 into the stage that tile i - 1 used (its MMA1 is done)
      load_tile_async(base, (i + 2) % kStages, A, t + 2 * G, gtid, kGroupThreads);
      bool ok = umma::mbar_wait(barM1 + 8 * b, (uint32_t)(i >> 1) & 1u, kWaitTries);
      if (i > 0) ok = ok && umma::mbar_wait(barM2 + 8 * (b ^ 1), (uint32_t)((i - 1) >> 1) & 1u, kWaitTries);
      ok = __all_sync(0xffffffffu, ok && !*abort_flag);  // warp-uniform: tcgen05.ld is .sync.aligned
      umma::fence_after_sync();
      if (ok) {
#pragma unroll 1
        for (int h = 2 * sl0; h < 2 * sl0 + 4; ++h) {  // columns 32 h .. 32 h + 31 (K slice h / 2 of A2)
          float r[32];
          umma::tmem_ld32(d + lane_off + 32u * (uint32_t)h, r);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            uint32_t w[4];
#pragma unroll
            for (int e = 0; e < 4; ++e)
              w[e] = relu_bf16x2_bits(r[8 * q + 2 * e], r[8 * q + 2 * e + 1]);
            *reinterpret_cast<uint4*>(sm + sA2 + umma::sw128_offset(row, 32 * h + 8 * q, kCand)) =
                make_uint4(w[0], w[1], w[2], w[3]);
          }
        }
      }
      cp_async_wait_prev();  // tile i + 1's A1 / chain part have landed (this thread's copies)
      if (ok && has_next)  // MMA1(i) has completed: columns 12, 13 are free; one value per thread
        put_chain_part(sm, gtid, reinterpret_cast<const float*>(sm + sC1 + (uint32_t)next_stage * (kH * 4))[gtid]);
      umma::fence_async_smem();
      umma::fence_before_sync();
      if (group_sync_or<1>(!ok)) {
        if (tid == 0) *abort_flag = 1;
        break;
      }
      if (tid == 0) {
        umma::fence_after_sync();
        issue_layer2(base, d, idesc);
        umma::commit(barM2 + 8 * b);
      } else if (tid == 32) {
        mbar_arrive(barE1 + 8 * b);  // epilogue 1(i) is done: group 2 may run epilogue 2(i - 1)
        if (has_next) {  // buffer b ^ 1 is free once epilogue 2 of tile i - 1 has read it
          if (i == 0 || umma::mbar_wait(barE2 + 8 * (b ^ 1), (uint32_t)((i - 1) >> 1) & 1u, kWaitTries)) {
            umma::fence_after_sync();
            issue_layer1(base, next_stage, tmem + 256u * (uint32_t)(b ^ 1), idesc);
            umma::commit(barM1 + 8 * (b ^ 1));
          } else {
            *abort_flag = 1;
          }
        }
      }
    }
  } else {
    // ---- warp group 2: epilogue 2 ----
    const float4* b2v = reinterpret_cast<const float4*>(b2s);
    const float4* w3v = reinterpret_cast<const float4*>(w3s);
    for (int i = 0, t = blockIdx.x; t < A.tiles; ++i, t += G) {
      const int b = i & 1;
      const uint32_t d = tmem + 256u * (uint32_t)b;
      bool ok = umma::mbar_wait(barM2 + 8 * b, (uint32_t)(i >> 1) & 1u, kWaitTries);
      // leave the issue slots to epilogue 1 of the next tile, which the tensor core waits for
      if (t + G < A.tiles) ok = ok && umma::mbar_wait(barE1 + 8 * (b ^ 1), (uint32_t)((i + 1) >> 1) & 1u, kWaitTries);
      ok = __all_sync(0xffffffffu, ok && !*abort_flag);
      umma::fence_after_sync();
      float* pb = part + b * (2 * kCand);
      if (ok) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
        for (int sl = sl0; sl < sl0 + 2; ++sl) {
          uint32_t r[64];
          umma::tmem_ld64(d + lane_off + 64u * (uint32_t)sl, r);
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const float4 bb = b2v[16 * sl + q], ww = w3v[16 * sl + q];
            acc[0] = fmaf(fmaxf(__uint_as_float(r[4 * q + 0]) + bb.x, 0.f), ww.x, acc[0]);
            acc[1] = fmaf(fmaxf(__uint_as_float(r[4 * q + 1]) + bb.y, 0.f), ww.y, acc[1]);
            acc[2] = fmaf(fmaxf(__uint_as_float(r[4 * q + 2]) + bb.z, 0.f), ww.z, acc[2]);
            acc[3] = fmaf(fmaxf(__uint_as_float(r[4 * q + 3]) + bb.w, 0.f), ww.w, acc[3]);
          }
        }
        umma::fence_before_sync();
        mbar_arrive(barE2 + 8 * b);
        pb[colhalf * kCand + row] = (acc[0] + acc[1]) + (acc[2] + acc[3]);
      }
      if (group_sync_or<2>(!ok)) {
        *abort_flag = 1;
        break;
      }
      if (colhalf == 0) A.pred[(size_t)t * kCand + row] = (pb[row] + pb[kCand + row] + b3) * kTargetScale;
    }
  }
  if (tid == 0 || tid == 32) {  // drain: every MMA issued by threads 0 and 32 has completed
    umma::commit(barFin);
    if (!umma::mbar_wait(barFin, 0u, kWaitTries)) *abort_flag = 1;
  }
  cp_async_wait_all();
  umma::fence_before_sync();
  __syncthreads();
  if (tid == 0 && *abort_flag && A.error_word) atomicOr(A.error_word, kErrTimeout);
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, 512);
  }
}

// ---------------------------------------------------------------------------
// Learned step: sample one candidate per chain from softmax(-pred / T), score
// it exactly, Metropolis-accept with the chain's threshold row, update the
// state and badness, and push the (features, exact dE) tuple to the ring.
// One team of WPC warps per chain (1 or 2), state in shared memory (as in the
// tempering kernel).  Every warp of a team runs the same draw on the same
// registers, so the team needs no broadcast; the exact move splits its slots
// over the team.
// ---------------------------------------------------------------------------
struct StepArgs {
  n3_chains ch;
  const uint16_t* lut;
  const float* temps;     // [L] ladder temperatures
  const int32_t* cand;    // [C][128]
  const float* pred;      // [C][128]
  const uint64_t* step;   // device step counter
  uint32_t k0, k1;
  // ring buffer
  uint16_t* rb_feat;      // [cap][12] bf16
  uint8_t* rb_bad;        // [cap][150]
  int16_t* rb_dE;         // [cap]
  int64_t rb_cap;
  float* stats;           // [4]: sum |pred - dE|, count, accepted, sum dE accepted
  int moves;              // moves drawn per step (without replacement)
};

constexpr int kStepChains = 14;  // chains per CTA: 2048 chains -> 147 CTAs, one per SM

template <int WPC>
__global__ void __launch_bounds__(kStepChains * 32 * WPC, 1) learned_step_kernel(const StepArgs A) {
  constexpr int TT = Team<WPC>::kThreads;
  extern __shared__ __align__(16) unsigned char smem[];
  const n3_chains& ch = A.ch;
  uint16_t* lut = reinterpret_cast<uint16_t*>(smem);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + kFullLutBytes);
  int* cs_all = reinterpret_cast<int*>(hist_all + kStepChains * kDirWords);
  int* bs_all = cs_all + kStepChains * kMaxM;
  int* team_red = bs_all + kStepChains * kMaxM;  // 2 WPC ints per chain (WPC > 1)
  int* cand_all = team_red + kStepChains * 4;    // this step's candidate codes and predictions
  float* pred_all = reinterpret_cast<float*>(cand_all + kStepChains * kCand);
  full_lut_copy(lut, A.lut);
  for (int i = threadIdx.x; i < kStepChains * kDirWords / 4; i += blockDim.x)
    reinterpret_cast<uint4*>(hist_all)[i] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  const int team = threadIdx.x / TT;  // this chain's index in the CTA
  Team<WPC> tm{(int)threadIdx.x % TT, 1 + team, team_red + 2 * WPC * team, 0, {}};
  const int lane = tm.t & 31;
  const int c = blockIdx.x * kStepChains + team;
  if (c >= ch.n_chains) return;  // the whole team leaves; no block-level barrier follows
  const int L = ch.ladder_size;
  const int n = ch.ladder_n[c / L], m = 2 * n;
  int* cs = cs_all + team * kMaxM;
  int* bs = bs_all + team * kMaxM;
  uint32_t* hist = hist_all + team * kDirWords;
  for (int s = tm.t; s < m; s += TT) {
    cs[s] = ch.cols[(size_t)c * kMaxM + s];
    bs[s] = ch.badness[(size_t)c * kMaxM + s];
  }
  team_load_keys(tm, cs, m);  // the thread's own slots' table keys, kept in registers across the moves
  const int temp = ch.temp_of[c];
  const float T = A.temps[temp];
  // softmax(-pred / T) over the legal candidates, sampled by inverse CDF;
  // with moves > 1 the step draws again without replacement after each move
  // (candidates are re-checked for legality on the current state).  Lane l
  // holds candidates 4l .. 4l + 3 (weights, codes and predictions in registers),
  // so a draw needs one warp scan of the lane totals.
  constexpr int kPer = kCand / 32;
  static_assert(kPer == 4, "four candidates per lane");
  // The codes and predictions also go to shared memory, where a draw reads the
  // picked one (registers hold only the weights).
  int* cand_c = cand_all + team * kCand;
  float* pred_c = pred_all + team * kCand;
  float w[kPer];
  float mx = -INFINITY;
  {
    const int4 cw4 = reinterpret_cast<const int4*>(A.cand + (size_t)c * kCand)[lane];
    const float4 pr4 = reinterpret_cast<const float4*>(A.pred + (size_t)c * kCand)[lane];
    if (tm.t < 32) {
      reinterpret_cast<int4*>(cand_c)[lane] = cw4;
      reinterpret_cast<float4*>(pred_c)[lane] = pr4;
    }
    const int cwv[kPer] = {cw4.x, cw4.y, cw4.z, cw4.w};
    const float prv[kPer] = {pr4.x, pr4.y, pr4.z, pr4.w};
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      w[q] = cwv[q] < 0 ? -prv[q] / T : -INFINITY;
      mx = fmaxf(mx, w[q]);
    }
  }
  tm.sync();  // the state and the candidates are read by the whole team from here on
#pragma unroll
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
#pragma unroll
  for (int q = 0; q < kPer; ++q) w[q] = w[q] > -INFINITY ? __expf(w[q] - mx) : 0.f;
  const uint64_t step = *A.step;
  int E = ch.energy[c];
  int bestE = ch.best_energy[c];
  uint32_t err = 0, n_acc = 0, n_scored = 0;
  int sum_dE_acc = 0;  // with n_acc, n_scored and st_abs: this chain's statistics (team-uniform)
  float st_abs = 0.f;
  // the moves' Philox blocks 32 at a time: lane l makes move k0 + l's, move k takes lane k % 32's
  U4 batch = {0u, 0u, 0u, 0u};
  // ring slot of move k: tuple (step C + c) moves + k modulo the capacity,
  // from one 64-bit remainder per chain and step
  const int64_t slot0 =
      (int64_t)(((step * (uint64_t)ch.n_chains + (uint64_t)c) * (uint64_t)A.moves) % (uint64_t)A.rb_cap);
  for (int k = 0; k < A.moves; ++k) {
    const int j = k & 31;
    if (j == 0)
      batch = philox4x32_10(U4{(uint32_t)step, (uint32_t)(step >> 32), (uint32_t)c,
                               kTagCandidate | 0xFF00u | (uint32_t)(k + lane)}, A.k0, A.k1);
    const U4 r = {__shfl_sync(0xffffffffu, batch.x, j), __shfl_sync(0xffffffffu, batch.y, j), 0u, 0u};
    // inclusive prefix of the weights in candidate order: within the lane, then across lanes
    float pre[kPer];
    pre[0] = w[0];
#pragma unroll
    for (int q = 1; q < kPer; ++q) pre[q] = pre[q - 1] + w[q];
    float incl = pre[kPer - 1];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const float y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const float acc_w = __shfl_sync(0xffffffffu, incl, 31);
    if (!(acc_w > 0.f)) break;  // no legal candidate left
    const float base = incl - pre[kPer - 1];
    const float target = ((float)(r.x >> 8) + 0.5f) * (1.0f / 16777216.0f) * acc_w;
    int q_hit = -1;
#pragma unroll
    for (int q = kPer - 1; q >= 0; --q)
      if (w[q] > 0.f && base + pre[q] > target) q_hit = q;  // the first such q
    unsigned hit = __ballot_sync(0xffffffffu, q_hit >= 0);
    int owner, q_pick;
    if (hit) {
      owner = __ffs(hit) - 1;
      q_pick = __shfl_sync(0xffffffffu, q_hit, owner);
    } else {  // rounding at the top end: the last candidate with weight
      int q_last = -1;
#pragma unroll
      for (int q = 0; q < kPer; ++q)
        if (w[q] > 0.f) q_last = q;
      hit = __ballot_sync(0xffffffffu, q_last >= 0);
      owner = 31 - __clz(hit);
      q_pick = __shfl_sync(0xffffffffu, q_last, owner);
    }
    const int cw = cand_c[kPer * owner + q_pick];
    const float p = pred_c[kPer * owner + q_pick];
    if (lane == owner) {  // without replacement
#pragma unroll
      for (int q = 0; q < kPer; ++q)
        if (q == q_pick) w[q] = 0.f;
    }
    const int u = cw & 0xFF, v = (cw >> 8) & 0xFF;
    if (k > 0 && !legal_swap(cs, u, v)) continue;  // an earlier move of this step made it illegal
    // tuple: features of the state before the move (thread i writes feature i).
    // These reads of cs and bs come before the move's first team barrier, and
    // the move writes the state only after later ones.
    int64_t slot = slot0 + k;
    if (slot >= A.rb_cap) {
      slot -= A.rb_cap;
      if (slot >= A.rb_cap) slot %= A.rb_cap;
    }
    if (tm.t < kCandFeat) {
      const int which = tm.t & 3;
      const int sidx = which == 0 ? u : which == 1 ? v : which == 2 ? (u ^ 1) : (v ^ 1);
      const float f = tm.t < 4 ? (float)bs[sidx] * (1.0f / 16.0f)
                               : (float)(tm.t < 8 ? (sidx >> 1) : cs[sidx]) * (1.0f / (float)n);
      A.rb_feat[slot * kCandFeat + tm.t] = bf16_bits(f);
    }
    for (int s = tm.t; s < kChainFeat; s += TT)
      A.rb_bad[slot * kChainFeat + s] = (uint8_t)(s < m ? min(bs[s], 255) : 0);
    int dE = 0;
    const uint32_t* thr = ch.acc_thresh + (size_t)temp * ch.acc_width;  // formed here: fewer live registers
    const int acc = team_move<WPC, false, false, false, true>(tm, cs, bs, m, lut, hist, u, v, r.y, thr, ch.acc_width,
                                                              E, err, &dE);
    if (tm.t == 0) A.rb_dE[slot] = (int16_t)max(-32768, min(32767, dE));
    n_acc += acc ? 1u : 0u;
    st_abs += fabsf(p - (float)dE);
    n_scored += 1u;
    if (acc) sum_dE_acc += dE;
    if (acc && E < bestE) {
      bestE = E;
      for (int s = tm.t; s < m; s += TT) ch.best_cols[(size_t)c * kMaxM + s] = (int16_t)cs[s];
    }
  }
  for (int s = tm.t; s < m; s += TT) {
    ch.cols[(size_t)c * kMaxM + s] = (int16_t)cs[s];
    ch.badness[(size_t)c * kMaxM + s] = bs[s];
  }
  if (tm.t == 0) {
    ch.energy[c] = E;
    ch.best_energy[c] = bestE;
    ch.accepted[c] += n_acc;
    if (err && ch.error_word) atomicOr(ch.error_word, err);
    if (ch.global_best) atomicMin(ch.global_best, E);
    // one set of statistics atomics per chain and step, not per move
    atomicAdd(A.stats + 0, st_abs);
    atomicAdd(A.stats + 1, (float)n_scored);
    atomicAdd(A.stats + 2, (float)n_acc);
    atomicAdd(A.stats + 3, (float)sum_dE_acc);
  }
}

// ---------------------------------------------------------------------------
// Training: batch gather, tensor-core GEMMs, fp32 head, bias sums and Adam.
// ---------------------------------------------------------------------------
struct Batch {
  float* X;   // [B][192]
  float* y;   // [B]
};

// Draws batch row b from the first `filled` ring slots, filled =
// min(capacity, steps recorded * chains); the draw is keyed by the training
// step counter.
__global__ void gather_kernel(const uint16_t* __restrict__ rb_feat, const uint8_t* __restrict__ rb_bad,
                              const int16_t* __restrict__ rb_dE, const uint64_t* __restrict__ counters,
                              int64_t capacity, int n_chains, int B, uint32_t k0, uint32_t k1, float* __restrict__ X,
                              float* __restrict__ y) {
  const int b = blockIdx.x;
  __shared__ int64_t slot_s;
  if (threadIdx.x == 0) {
    const uint64_t steps = counters[0], t = counters[1];
    const uint64_t recorded = steps * (uint64_t)n_chains;
    const uint64_t filled = recorded < (uint64_t)capacity ? (recorded ? recorded : 1) : (uint64_t)capacity;
    const U4 r = philox4x32_10(U4{(uint32_t)t, (uint32_t)(t >> 32), (uint32_t)b, 0x7A000000u}, k0, k1);
    const uint64_t x = ((uint64_t)r.x << 32) | r.y;
    slot_s = (int64_t)(x % filled);
    y[b] = (float)rb_dE[slot_s] / kTargetScale;
  }
  __syncthreads();
  const int64_t s = slot_s;
  for (int k = threadIdx.x; k < kIn; k += blockDim.x) {
    float v = 0.f;
    if (k < kCandFeat) {
      const uint16_t h = rb_feat[s * kCandFeat + k];
      v = __uint_as_float((uint32_t)h << 16);
    } else if (k < kCandFeat + kChainFeat) {
      v = (float)rb_bad[s * kChainFeat + (k - kCandFeat)] * (1.0f / 16.0f);
    }
    X[(size_t)b * kIn + k] = v;
  }
}


// out = H2 . w3 + b3, d = 2 (out - y) / B, dZ2 = d w3 (Z2 > 0), loss += (out - y)^2
// GEMMs on the tensor cores (tcgen05, kind::f16): C (M x N, fp32) =
// sum_k A(m, k) B(k, n) for fp32 operands given by element strides (A(m, k) at
// A[m sam + k sak], B(k, n) at Bm[k sbk + n sbn]), with the epilogues of the
// training step: EPI 0 store (or add, with a K split over gridDim.z: the
// weight gradients), EPI 1 Z = acc + bias, H = relu(Z) (the forward layers),
// EPI 2 acc masked by Z > 0 (back through a ReLU); and EPI 3 acc + bias (the
// chain part of layer 1 before inference).
//
// A CTA of 4 warps owns a 128 x kTcN output tile.  Per K slice of 64 it rounds
// the operands to bf16 while staging them into 128B-swizzled K-major shared
// tiles (two buffers: the next slice is staged while the tensor core reads the
// current one), thread 0 issues the slice's four K = 16 MMAs into a 128 x kTcN
// fp32 accumulator in tensor memory and commits them to the buffer's mbarrier,
// and the epilogue reads the accumulator back with tcgen05.ld (warp w: rows
// 32 w .. 32 w + 31).  Every mbarrier wait is bounded; an expired wait sets
// error bit 8 and skips the epilogue.
constexpr int kTcN = 64;                            // output columns per CTA (tensor-memory columns)
constexpr uint32_t kTcA = 128 * 128;                // bytes of one A slice (128 rows x 64 bf16)
constexpr uint32_t kTcB = kTcN * 128;               // bytes of one B slice
constexpr uint32_t kTcBar = 2 * (kTcA + kTcB);      // two mbarriers and the tensor-memory address
constexpr uint32_t kTcSmem = kTcBar + 64 + 1024;    // + alignment slack

// Stages ROWS x 64 elements of an operand, element (r, k) at src[(r0 + r) sr + (k0 + k) sk],
// zero outside r0 + r < R, k0 + k < Ke, into an SW128 K-major bf16 tile.  All
// of a thread's loads are issued before any conversion (a fixed count per
// thread, in registers), so their latencies overlap.
template <int ROWS>
__device__ __forceinline__ void tc_stage(uint8_t* tile, const float* __restrict__ src, int sr, int sk, int r0, int R,
                                         int k0, int Ke, int tid) {
  constexpr int kPer = ROWS * 64 / 128;  // elements per thread
  float v[kPer];
  if (sk == 1) {  // k contiguous: a warp reads 64 consecutive floats (two per lane) of one row
#pragma unroll
    for (int e = 0; e < kPer / 2; ++e) {
      const int i = tid + 128 * e, r = i >> 5, k = 2 * (i & 31);
      const bool rin = r0 + r < R;
      const float* q = src + (size_t)(r0 + r) * sr + (k0 + k);
      v[2 * e] = rin && k0 + k < Ke ? __ldg(q) : 0.f;
      v[2 * e + 1] = rin && k0 + k + 1 < Ke ? __ldg(q + 1) : 0.f;
    }
#pragma unroll
    for (int e = 0; e < kPer / 2; ++e) {
      const int i = tid + 128 * e, r = i >> 5, k = 2 * (i & 31);
      *reinterpret_cast<uint32_t*>(tile + umma::sw128_offset(r, k, ROWS)) = bf16x2_bits(v[2 * e], v[2 * e + 1]);
    }
  } else {  // rows contiguous (or neither): a warp reads 32 consecutive rows of one k
#pragma unroll
    for (int e = 0; e < kPer; ++e) {
      const int i = tid + 128 * e, k = i / ROWS, r = i % ROWS;
      v[e] = r0 + r < R && k0 + k < Ke ? __ldg(src + (size_t)(r0 + r) * sr + (size_t)(k0 + k) * sk) : 0.f;
    }
#pragma unroll
    for (int e = 0; e < kPer; ++e) {
      const int i = tid + 128 * e, k = i / ROWS, r = i % ROWS;
      *reinterpret_cast<uint16_t*>(tile + umma::sw128_offset(r, k, ROWS)) = bf16_bits(v[e]);
    }
  }
}

template <int EPI>
__global__ void __launch_bounds__(128) tc_gemm_kernel(int M, int N, int K, const float* __restrict__ A, int sam,
                                                      int sak, const float* __restrict__ Bm, int sbk, int sbn,
                                                      float* __restrict__ C, int ldc, const float* __restrict__ bias,
                                                      float* __restrict__ aux, uint32_t* error_word) {
  extern __shared__ __align__(16) uint8_t tc_smem[];
  const uint32_t raw = umma::smem_addr(tc_smem);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* sm = tc_smem + (base - raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * 128, n0 = blockIdx.x * kTcN;
  const int kchunk = ((K + (int)gridDim.z - 1) / (int)gridDim.z + 63) / 64 * 64;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  const int slices = kb < ke ? (ke - kb + 63) / 64 : 0;
  if (slices == 0) return;  // a K split with nothing to add (uniform across the CTA)
  const uint32_t bar0 = base + kTcBar, bar1 = bar0 + 8, taddr_slot = bar0 + 16;
  if (warp == 0) {
    umma::tmem_alloc(taddr_slot, kTcN);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    umma::mbar_init(bar0, 1);
    umma::mbar_init(bar1, 1);
    umma::mbar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kTcBar + 16);
  constexpr uint32_t idesc = umma::idesc_bf16_f32(128, kTcN);
  bool ok = true;
  for (int s = 0; s < slices; ++s) {
    const int buf = s & 1;
    const uint32_t bar = buf ? bar1 : bar0;
    // the MMAs of slice s - 2 read this buffer: wait for their commit
    if (s >= 2) ok = ok && umma::mbar_wait(bar, (uint32_t)((s - 2) >> 1) & 1u, kWaitTries);
    uint8_t* ta = sm + buf * (kTcA + kTcB);
    uint8_t* tb = ta + kTcA;
    const int k0 = kb + 64 * s;
    tc_stage<128>(ta, A, sam, sak, m0, M, k0, ke, tid);
    tc_stage<kTcN>(tb, Bm, sbn, sbk, n0, N, k0, ke, tid);
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a_s = base + buf * (kTcA + kTcB), b_s = a_s + kTcA;
#pragma unroll
      for (int k16 = 0; k16 < 4; ++k16)
        umma::mma_bf16(tmem, umma::desc_sw128(a_s + 32 * k16), umma::desc_sw128(b_s + 32 * k16), idesc,
                       (s > 0 || k16 > 0) ? 1u : 0u);
      umma::commit(bar);
    }
  }
  // the last commit covers every MMA issued before it
  const int last = slices - 1;
  ok = ok && umma::mbar_wait((last & 1) ? bar1 : bar0, (uint32_t)(last >> 1) & 1u, kWaitTries);
  ok = __syncthreads_and(ok);
  umma::fence_after_sync();
  if (ok) {
    // Each thread reads its row's 32 columns of a chunk from tensor memory; the
    // warp's 32 x 32 block goes through shared memory (the staging tiles are
    // free now) so that each store instruction writes one row's 32 columns.
    float* blk = reinterpret_cast<float*>(sm) + warp * (32 * 33);
#pragma unroll 1
    for (int c0 = 0; c0 < kTcN; c0 += 32) {
      float v[32];
      umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
#pragma unroll
      for (int j = 0; j < 32; ++j) blk[lane * 33 + j] = v[j];
      __syncwarp();
      const int nn = n0 + c0 + lane;
#pragma unroll 4
      for (int rr = 0; rr < 32; ++rr) {
        const int row = m0 + 32 * warp + rr;
        if (row >= M || nn >= N) continue;
        const float x = blk[rr * 33 + lane];
        const size_t o = (size_t)row * ldc + nn;
        if (EPI == 0) {
          if (gridDim.z > 1)
            atomicAdd(C + o, x);
          else
            C[o] = x;
        } else if (EPI == 1) {
          const float z = x + bias[nn];
          aux[o] = z;
          C[o] = fmaxf(z, 0.f);
        } else if (EPI == 3) {
          C[o] = x + bias[nn];
        } else {
          C[o] = aux[o] > 0.f ? x : 0.f;
        }
      }
      __syncwarp();
    }
  } else if (tid == 0 && error_word) {
    atomicOr(error_word, kErrTimeout);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, kTcN);
}

__global__ void head_kernel(int B, const float* __restrict__ H2, const float* __restrict__ Z2,
                            const float* __restrict__ P, const float* __restrict__ y, float* __restrict__ d,
                            float* __restrict__ dZ2, float* __restrict__ loss) {
  const int b = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (b >= B) return;
  float acc = 0.f;
  for (int k = lane; k < kH; k += 32) acc = fmaf(H2[(size_t)b * kH + k], P[oW3 + k], acc);
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  const float out = acc + P[oB3];
  const float e = out - y[b];
  const float g = 2.f * e / (float)B;
  if (lane == 0) {
    d[b] = g;
    atomicAdd(loss, e * e);
  }
  for (int k = lane; k < kH; k += 32) dZ2[(size_t)b * kH + k] = Z2[(size_t)b * kH + k] > 0.f ? g * P[oW3 + k] : 0.f;
}

// Column sums added into a zeroed `out`: out[n] += sum_b M[b][n] (* scale[b]).
// Block (x, y) sums rows [y * kColRows, ...) of columns x * blockDim.x + t.
constexpr int kColRows = 128;
__global__ void colsum_kernel(int B, int N, const float* __restrict__ Mx, const float* __restrict__ scale,
                              float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int b0 = blockIdx.y * kColRows, b1 = min(B, b0 + kColRows);
  float acc = 0.f;
  for (int b = b0; b < b1; ++b) acc = fmaf(Mx[(size_t)b * N + n], scale ? scale[b] : 1.f, acc);
  atomicAdd(out + n, acc);
}

__global__ void sum_kernel(int B, const float* __restrict__ v, float* __restrict__ out) {
  float acc = 0.f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) acc += v[b];
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x / 32] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int i = 0; i < (int)(blockDim.x / 32); ++i) t += part[i];
    *out = t;
  }
}

// Adam (Kingma & Ba) with bias correction; the step number is counters[1] + 1.
__global__ void adam_kernel(int count, float* __restrict__ P, const float* __restrict__ G, float* __restrict__ Mo,
                            float* __restrict__ V, float lr, float b1, float b2, float eps,
                            const uint64_t* __restrict__ counters) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float t = (float)(counters[1] + 1);
  const float c1 = 1.f - powf(b1, t), c2 = 1.f - powf(b2, t);
  const float g = G[i];
  const float m = b1 * Mo[i] + (1.f - b1) * g;
  const float v = b2 * V[i] + (1.f - b2) * g * g;
  Mo[i] = m;
  V[i] = v;
  P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

__global__ void bump_kernel(uint64_t* counters, int which) { counters[which] += 1; }

}  // namespace mlp
}  // namespace n3

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
namespace n3host {
using namespace n3::mlp;

static int launch_pack(const n3_mlp* M, cudaStream_t st) {
  pack_kernel<<<148, 256, 0, st>>>(M->params, M->w2_img, M->w1a_img);
  return check_launch("mlp pack_kernel");
}

static size_t step_smem() {  // the team scratch is sized for the widest team (2 warps)
  return n3::kFullLutBytes + kStepChains * (sizeof(uint32_t) * n3::kDirWords + 2 * sizeof(int) * n3::kMaxM +
                                            4 * sizeof(int) + kCand * (sizeof(int) + sizeof(float)));
}

// Threads per chain of the learned step when the caller leaves it open: two
// warps for several moves per step (2048 chains x 16 moves: 6.50 against
// 6.68 ms per 50 steps), one for a single move (4.31 against 4.33 ms).
static int default_step_threads(int moves) { return moves > 1 ? 64 : 32; }

int prepare_mlp() {
  N3_TRY(allow_smem(reinterpret_cast<const void*>(infer_kernel), kInferSmem));
  N3_TRY(allow_smem(reinterpret_cast<const void*>(tc_gemm_kernel<3>), kTcSmem));
  N3_TRY(allow_smem(reinterpret_cast<const void*>(learned_step_kernel<1>), step_smem()));
  return allow_smem(reinterpret_cast<const void*>(learned_step_kernel<2>), step_smem());
}

}  // namespace n3host

namespace n3host {

// One training step: gather a batch from the ring buffer, forward, backward,
// Adam, repack the tensor-core weight images.  `scratch` holds the batch
// activations (n3_mlp_scratch_floats(batch) floats), `grads` the gradient
// (kParams floats); both entry points below call this body.
static int train_step(const n3_mlp* M, int n_chains, int B, float lr, uint64_t seed, float* scratch, float* grads,
                      float* adam_m, float* adam_v, cudaStream_t st) {
  using namespace n3::mlp;
  float* X = scratch;
  float* y = X + (size_t)B * kIn;
  float* d = y + B;
  float* Z1 = d + B;
  float* H1 = Z1 + (size_t)B * kH;
  float* Z2 = H1 + (size_t)B * kH;
  float* H2 = Z2 + (size_t)B * kH;
  float* dZ2 = H2 + (size_t)B * kH;
  float* dZ1 = dZ2 + (size_t)B * kH;
  float* loss = dZ1 + (size_t)B * kH;
  float* P = M->params;
  // the gradient and the loss are accumulated: clear them first
  if (cudaMemsetAsync(grads, 0, sizeof(float) * kParams, st) != cudaSuccess ||
      cudaMemsetAsync(loss, 0, sizeof(float), st) != cudaSuccess)
    return check_launch("MLP training: clearing the gradient");
  gather_kernel<<<B, 64, 0, st>>>(M->rb_feat, M->rb_bad, M->rb_dE, M->counters, M->rb_capacity, n_chains, B,
                                  (uint32_t)seed, (uint32_t)(seed >> 32), X, y);
  // tensor-core GEMMs (tc_gemm_kernel): 128-row tiles of kTcN columns; the
  // weight gradients split K = batch over up to 16 CTAs per tile
  N3_TRY(allow_smem(reinterpret_cast<const void*>(tc_gemm_kernel<0>), kTcSmem));
  N3_TRY(allow_smem(reinterpret_cast<const void*>(tc_gemm_kernel<1>), kTcSmem));
  N3_TRY(allow_smem(reinterpret_cast<const void*>(tc_gemm_kernel<2>), kTcSmem));
  const int row_tiles = (B + 127) / 128;
  const int splits = B >= 4096 ? 16 : B >= 512 ? B / 256 : 1;
  uint32_t* ew = M->error_word;
  // Z1 = X W1^T + b1 ; H1 = relu(Z1)     (W1 [256][192]: B(k, n) = W1[n*192 + k])
  tc_gemm_kernel<1><<<dim3(kH / kTcN, row_tiles, 1), 128, kTcSmem, st>>>(B, kH, kIn, X, kIn, 1, P + oW1, 1, kIn,
                                                                          H1, kH, P + oB1, Z1, ew);
  tc_gemm_kernel<1><<<dim3(kH / kTcN, row_tiles, 1), 128, kTcSmem, st>>>(B, kH, kH, H1, kH, 1, P + oW2, 1, kH,
                                                                          H2, kH, P + oB2, Z2, ew);
  head_kernel<<<(B + 7) / 8, 256, 0, st>>>(B, H2, Z2, P, y, d, dZ2, loss);
  // gradients of the head and layer 2
  colsum_kernel<<<dim3((kH + 127) / 128, (B + kColRows - 1) / kColRows), 128, 0, st>>>(B, kH, H2, d, grads + oW3);
  sum_kernel<<<1, 1024, 0, st>>>(B, d, grads + oB3);
  // gW2[n][k] = sum_b dZ2[b][n] H1[b][k]
  tc_gemm_kernel<0><<<dim3(kH / kTcN, kH / 128, splits), 128, kTcSmem, st>>>(kH, kH, B, dZ2, 1, kH, H1, kH, 1,
                                                                              grads + oW2, kH, nullptr, nullptr, ew);
  colsum_kernel<<<dim3((kH + 127) / 128, (B + kColRows - 1) / kColRows), 128, 0, st>>>(B, kH, dZ2, nullptr, grads + oB2);
  // dZ1 = (dZ2 W2) * (Z1 > 0)            (B(k, n) = W2[k*256 + n])
  tc_gemm_kernel<2><<<dim3(kH / kTcN, row_tiles, 1), 128, kTcSmem, st>>>(B, kH, kH, dZ2, kH, 1, P + oW2, kH, 1,
                                                                          dZ1, kH, nullptr, Z1, ew);
  // gW1[n][k] = sum_b dZ1[b][n] X[b][k]
  tc_gemm_kernel<0><<<dim3(kIn / kTcN, kH / 128, splits), 128, kTcSmem, st>>>(kH, kIn, B, dZ1, 1, kH, X, kIn, 1,
                                                                               grads + oW1, kIn, nullptr, nullptr, ew);
  colsum_kernel<<<dim3((kH + 127) / 128, (B + kColRows - 1) / kColRows), 128, 0, st>>>(B, kH, dZ1, nullptr, grads + oB1);
  adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(kParams, P, grads, adam_m, adam_v, lr, 0.9f, 0.999f, 1e-8f,
                                                     M->counters);
  bump_kernel<<<1, 1, 0, st>>>(M->counters, 1);
  if (M->loss_out && cudaMemcpyAsync(M->loss_out, loss, sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return check_launch("MLP training: loss copy");
  N3_TRY(check_launch("mlp training kernels"));
  return launch_pack(M, st);
}

}  // namespace n3host

extern "C" {

int n3_mlp_param_count(void) { return n3::mlp::kParams; }

int n3_mlp_scratch_floats(int batch) {
  // X [B][192], y, d, Z1, H1, Z2, H2, dZ2, dZ1 [B][256] each, loss
  return batch * (n3::mlp::kIn + 2) + 6 * batch * n3::mlp::kH + 4;
}

int n3_mlp_pack(const n3_mlp* M, void* stream) {
  if (!M || !M->params || !M->w2_img || !M->w1a_img) return n3host::set_error(N3_ERR_ARG, "null MLP buffer");
  return n3host::launch_pack(M, (cudaStream_t)stream);
}

int n3_mlp_candidates(const n3_chains* ch, const n3_mlp* M, uint64_t seed, int bad_bias, void* stream) {
  using namespace n3::mlp;
  if (!ch || !M) return n3host::set_error(N3_ERR_ARG, "null descriptor");
  if (bad_bias < 0 || bad_bias > 100) return n3host::set_error(N3_ERR_ARG, "bad_bias %d outside [0, 100]", bad_bias);
  CandArgs A;
  A.cols = ch->cols;
  A.badness = ch->badness;
  A.ladder_n = ch->ladder_n;
  A.ladder_size = ch->ladder_size;
  A.n_chains = ch->n_chains;
  A.a1_img = M->a1_img;
  A.badn = M->badn;
  A.cand = M->cand;
  A.step = M->counters;
  A.k0 = (uint32_t)seed;
  A.k1 = (uint32_t)(seed >> 32);
  A.bad_bias = bad_bias;
  cudaStream_t st = (cudaStream_t)stream;
  candidates_kernel<<<ch->n_chains, kCand, 0, st>>>(A);
  N3_TRY(n3host::check_launch("candidates_kernel"));
  // Chain part of layer 1 for every chain, c1 = badn W1b^T + b1 (W1b: the 150
  // chain columns of W1, B(k, n) = W1[n * 192 + 12 + k]), on the tensor cores
  // with bf16 operands and fp32 accumulation, as the training forward computes
  // the same product.  2048 chains: 16 x 4 CTAs of 128 x 64 outputs, K = 150
  // in three slices.
  const int C = ch->n_chains;
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(tc_gemm_kernel<3>), kTcSmem));
  tc_gemm_kernel<3><<<dim3(kH / kTcN, (C + 127) / 128, 1), 128, kTcSmem, st>>>(
      C, kH, kChainFeat, M->badn, kChainFeat, 1, M->params + oW1 + kCandFeat, 1, kIn, M->c1, kH, M->params + oB1,
      nullptr, M->error_word);
  return n3host::check_launch("chain part (tc_gemm_kernel<3>)");
}

int n3_mlp_infer(const n3_mlp* M, int tiles, void* stream) {
  using namespace n3::mlp;
  if (!M || tiles < 0) return n3host::set_error(N3_ERR_ARG, "bad MLP inference arguments");
  if (tiles == 0) return N3_OK;
  N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(infer_kernel), kInferSmem));
  InferArgs A;
  A.a1_img = M->a1_img;
  A.c1 = M->c1;
  A.w2_img = M->w2_img;
  A.w1a_img = M->w1a_img;
  A.P = M->params;
  A.pred = M->pred;
  A.tiles = tiles;
  A.error_word = M->error_word;
  const int grid = tiles < n3host::sm_count() ? tiles : n3host::sm_count();
  infer_kernel<<<grid, kInferThreads, kInferSmem, (cudaStream_t)stream>>>(A);
  return n3host::check_launch("infer_kernel");
}

int n3_mlp_step_team(const n3_chains* ch, const n3_mlp* M, const float* temps, uint64_t seed, int moves,
                     int threads_per_chain, void* stream) {
  using namespace n3::mlp;
  if (!ch || !M || !temps) return n3host::set_error(N3_ERR_ARG, "null descriptor");
  if (moves < 1 || moves > kCand) return n3host::set_error(N3_ERR_RANGE, "moves per step %d outside [1, 128]", moves);
  if (M->rb_capacity < 1) return n3host::set_error(N3_ERR_ARG, "ring buffer capacity %lld", (long long)M->rb_capacity);
  if (threads_per_chain == 0) threads_per_chain = n3host::default_step_threads(moves);
  if (threads_per_chain != 32 && threads_per_chain != 64)
    return n3host::set_error(N3_ERR_RANGE, "threads per chain %d: the learned step takes 32 or 64", threads_per_chain);
  N3_TRY(n3host::ensure_device_tables());
  const size_t smem = n3host::step_smem();
  StepArgs A;
  A.ch = *ch;
  A.lut = n3host::dir_lut_full_device_ptr();
  A.temps = temps;
  A.cand = M->cand;
  A.pred = M->pred;
  A.step = M->counters;
  A.k0 = (uint32_t)seed;
  A.k1 = (uint32_t)(seed >> 32);
  A.rb_feat = M->rb_feat;
  A.rb_bad = M->rb_bad;
  A.rb_dE = M->rb_dE;
  A.rb_cap = M->rb_capacity;
  A.stats = M->stats;
  A.moves = moves;
  const int grid = (ch->n_chains + kStepChains - 1) / kStepChains;
  if (threads_per_chain == 64) {
    N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(learned_step_kernel<2>), smem));
    learned_step_kernel<2><<<grid, kStepChains * 64, smem, (cudaStream_t)stream>>>(A);
  } else {
    N3_TRY(n3host::allow_smem(reinterpret_cast<const void*>(learned_step_kernel<1>), smem));
    learned_step_kernel<1><<<grid, kStepChains * 32, smem, (cudaStream_t)stream>>>(A);
  }
  N3_TRY(n3host::check_launch("learned_step_kernel"));
  bump_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(M->counters, 0);
  return n3host::check_launch("bump_kernel");
}

int n3_mlp_step(const n3_chains* ch, const n3_mlp* M, const float* temps, uint64_t seed, int moves, void* stream) {
  return n3_mlp_step_team(ch, M, temps, seed, moves, 0, stream);
}

int n3_mlp_train(const n3_mlp* M, int n_chains, int batch, float lr, uint64_t seed, float* scratch, float* grads,
                 float* adam_m, float* adam_v, void* stream) {
  if (!M || !scratch || !grads || !adam_m || !adam_v || batch < 64 || n_chains < 1)
    return n3host::set_error(N3_ERR_ARG, "bad MLP training arguments");
  return n3host::train_step(M, n_chains, batch, lr, seed, scratch, grads, adam_m, adam_v, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Training step that allocates nothing.
//
// n3_mlp_train needs its caller to provide device memory for the batch
// activations and the gradient.  Some callers cannot call cudaMalloc: an
// application that hands all device memory to its own allocator at start-up,
// or a plug-in loaded into a host whose memory manager forbids allocations it
// does not make itself.  For them, n3_mlp_train_noalloc keeps that working
// memory in the file-scope array below, sized for batches of at most
// kNoAllocMaxBatch tuples (about 4 MB).  Every GPU that loads libn3.so holds
// this array until the process exits.
// ---------------------------------------------------------------------------
namespace n3 {
namespace mlp {
constexpr int kNoAllocMaxBatch = 512;
constexpr size_t kNoAllocScratchFloats =
    (size_t)kNoAllocMaxBatch * (kIn + 2) + (size_t)6 * kNoAllocMaxBatch * kH + 4;
constexpr size_t kNoAllocFloats = kNoAllocScratchFloats + kParams;  // scratch, then the gradient
static __device__ __align__(256) float g_noalloc_work[kNoAllocFloats];
}  // namespace mlp
}  // namespace n3

namespace n3host {

// Device address of g_noalloc_work in the current context.  The symbol's
// host-side name is not a device address, so the address is looked up with
// cudaGetSymbolAddress: once per device, and again whenever the device's
// context has changed since (cudaDeviceReset destroys the context and with it
// the address).  Contexts are told apart by the driver's context id; while
// no context is current yet, or where that query is unavailable, the address
// is looked up on every call.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

static bool current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  CUcontext ctx = nullptr;
  return get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx != nullptr &&
         get_id(ctx, id) == CUDA_SUCCESS;
}

static int noalloc_work_ptr(float** out) {
  static std::mutex mu;
  static float* ptrs[64];
  static unsigned long long ctx_ids[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return set_error(N3_ERR_CUDA, "n3_mlp_train_noalloc: no usable current device");
  unsigned long long id = 0;
  const bool have_id = current_context_id(&id);
  std::lock_guard<std::mutex> lock(mu);
  if (ptrs[dev] == nullptr || !have_id || ctx_ids[dev] != id) {
    float* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, n3::mlp::g_noalloc_work);
    if (e != cudaSuccess || p == nullptr)
      return set_error(N3_ERR_CUDA, "n3_mlp_train_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    ptrs[dev] = p;
    ctx_ids[dev] = have_id ? id : 0;
  }
  *out = ptrs[dev];
  return N3_OK;
}

}  // namespace n3host

extern "C" int n3_mlp_train_noalloc(const n3_mlp* M, int n_chains, int batch, float lr, uint64_t seed,
                                    float* adam_m, float* adam_v, void* stream) {
  using namespace n3::mlp;
  if (!M || !adam_m || !adam_v || n_chains < 1) return n3host::set_error(N3_ERR_ARG, "bad MLP training arguments");
  if (batch < 64 || batch > kNoAllocMaxBatch)
    return n3host::set_error(N3_ERR_RANGE, "n3_mlp_train_noalloc: batch %d outside [64, %d] (its static working "
                             "memory holds at most %d tuples)", batch, kNoAllocMaxBatch, kNoAllocMaxBatch);
  float* work = nullptr;
  N3_TRY(n3host::noalloc_work_ptr(&work));
  // the array keeps the previous call's contents; train_step clears the
  // accumulated gradient and loss before use
  return n3host::train_step(M, n_chains, batch, lr, seed, work, work + kNoAllocScratchFloats, adam_m, adam_v,
                            (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Expiry of a bounded wait, on purpose.  The tensor-core pipeline waits on
// mbarriers with the bounded umma::mbar_wait and, when a wait gives up, sets
// kErrTimeout and returns instead of hanging.  wait_expiry_kernel runs that
// same wait where it must give up: one thread initialises an mbarrier that
// nothing ever arrives on, waits for its phase 0 at most `tries` times,
// records the expiry in the error word and invalidates the barrier.  No
// counterpart in the reference (its kernels have no bounded waits).
// ---------------------------------------------------------------------------
namespace n3 {
namespace mlp {
__global__ void wait_expiry_kernel(uint32_t tries, uint32_t* error_word) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(&bar);
  umma::mbar_init(s, 1);
  umma::mbar_fence_init();
  if (!umma::mbar_wait(s, 0, tries)) atomicOr(error_word, kErrTimeout);
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(s) : "memory");
}
}  // namespace mlp
}  // namespace n3

extern "C" int n3_check_bounded_wait(uint32_t tries, uint32_t* error_word, void* stream) {
  if (error_word == nullptr) return n3host::set_error(N3_ERR_ARG, "null error word");
  if (tries < 1 || tries > (1u << 20)) return n3host::set_error(N3_ERR_RANGE, "tries %u outside [1, 2^20]", tries);
  n3::mlp::wait_expiry_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(tries, error_word);
  return n3host::check_launch("wait_expiry_kernel");
}
