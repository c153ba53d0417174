// Instruction-throughput ceiling of the determinant test.
//
// The population scorer's inner step (score.cu, det_pivot_row) performs, per
// four triple tests, two integer multiplies, two multiply-adds and four
// compares.  det_ceiling_kernel runs the same expression on register-resident
// operands with no shared-memory traffic, counting every hit, on every SM: a
// ceiling of that expression.  int_pipe_kernel measures the two integer pipes
// the expression uses on their own (no integer peak is published for B200).
#include "n3_common.cuh"

namespace n3 {

template <int R>
__global__ void __launch_bounds__(256) det_ceiling_kernel(int iters, int seed, unsigned long long* out) {
  int ax[R], bx0[R], bx1[R], k0[R], k1[R];
  const int t = threadIdx.x + seed;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    ax[r] = (t + 3 * r) % 37 - 18;
    bx0[r] = (t * 7 + r) % 41 - 20;
    bx1[r] = (t * 5 + 2 * r) % 43 - 21;
    k0[r] = ax[r] * (t % 29);
    k1[r] = ax[r] * (t % 31);
  }
  int cnt = 0;
  int cx = t & 63, cyv = (t >> 3) & 63, ay = -30;
#pragma unroll 2
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int P0 = ax[r] * cx, P1 = ax[r] * cyv;
      const int T0 = ay * bx0[r] + k0[r], T1 = ay * bx1[r] + k1[r];
      cnt += ((P0 == T0) + (P1 == T0)) + ((P0 == T1) + (P1 == T1));
    }
    // next "row": the scorer loads two columns and bumps the row offset
    cx = (cx + 13) & 63;
    cyv = (cyv + 29) & 63;
    ay += 1;
  }
  if (cnt == 0x7fffffff) out[0] = cnt;  // keeps the loop live
  if (threadIdx.x == 0 && blockIdx.x == 0) out[1] = (unsigned long long)iters;
}

// Pipe ceilings independent of the scorer's expression.  Each thread runs 8
// independent loop-carried chains of one instruction kind on runtime values
// (so nothing folds): an integer multiply-add a = a * b + c (the FMA pipe's
// integer work, as the scorer's products) or a three-input logic op
// a = (a & b) | (a ^ c) (the ALU pipe, as the scorer's compares).  Ops per
// launch = blocks * 256 * iters * 8.
template <int KIND>
__global__ void __launch_bounds__(256) int_pipe_kernel(int iters, int seed, unsigned long long* out) {
  const int t = threadIdx.x + blockIdx.x * 7 + seed;
  const int b = (t | 1) * 0x9E37, c = t * 0x85EB + 11;
  int a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = t + i * 0x632B;
#pragma unroll 4
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = KIND == 0 ? a[i] * b + c : (a[i] & b) | (a[i] ^ c);
  }
  int x = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) x ^= a[i];
  if (x == 0x7fffffff) out[0] = (unsigned long long)x;  // keeps the chains live
}

// Random 4-byte gathers from a table that fits in L2 (the access pattern of
// the pair-table scorer): each thread draws `iters` indices with a 32-bit
// xorshift and sums the entries.  Gathers per launch = blocks * 256 * iters.
__global__ void __launch_bounds__(256) l2_gather_kernel(const int32_t* __restrict__ table, uint32_t entries,
                                                        int iters, int seed, unsigned long long* out) {
  uint32_t x = (threadIdx.x + blockIdx.x * 256u) * 2654435761u + (uint32_t)seed + 1u;
  int sum = 0;
#pragma unroll 8
  for (int it = 0; it < iters; ++it) {
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    sum += __ldg(table + __umulhi(x, entries));
  }
  if (sum == 0x7fffffff) out[0] = (unsigned long long)sum;  // keeps the loads live
}

}  // namespace n3

extern "C" int n3_calibrate_l2_gather(const int32_t* table, int64_t entries, int blocks, int iters,
                                      unsigned long long* scratch2, void* stream) {
  if (!table || entries < 1 || entries > 0xFFFFFFFFll || blocks < 1 || iters < 1 || !scratch2)
    return n3host::set_error(N3_ERR_ARG, "calibrate: bad arguments");
  n3::l2_gather_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(table, (uint32_t)entries, iters, blocks, scratch2);
  return n3host::check_launch("l2_gather_kernel");
}

extern "C" int n3_calibrate_int_pipe(int kind, int blocks, int iters, unsigned long long* scratch2, void* stream) {
  if (blocks < 1 || iters < 1 || scratch2 == nullptr || (kind != 0 && kind != 1))
    return n3host::set_error(N3_ERR_ARG, "calibrate: bad arguments");
  if (kind == 0)
    n3::int_pipe_kernel<0><<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, blocks, scratch2);
  else
    n3::int_pipe_kernel<1><<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, blocks, scratch2);
  return n3host::check_launch("int_pipe_kernel");
}

extern "C" int n3_calibrate_det_ceiling(int blocks, int iters, unsigned long long* scratch2, void* stream) {
  if (blocks < 1 || iters < 1 || scratch2 == nullptr)
    return n3host::set_error(N3_ERR_ARG, "calibrate: bad arguments");
  n3::det_ceiling_kernel<4><<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, blocks, scratch2);
  return n3host::check_launch("det_ceiling_kernel");
}
