// Instruction-throughput ceiling of the determinant test.
//
// The population scorer's inner step (score.cu, det_pivot_row) performs, per
// four triple tests, two IMUL + two IMAD and four compare-and-count pairs.
// This kernel runs that exact expression on register-resident operands with
// no shared-memory traffic, loop-carried only through the counters, on every
// SM.  Its tests/s is the roofline ceiling against which the scorer's
// achieved tests/s is reported (the hot kernels are integer-ALU bound, and no
// integer peak is published for B200).
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

}  // namespace n3

extern "C" int n3_calibrate_det_ceiling(int blocks, int iters, unsigned long long* scratch2, void* stream) {
  if (blocks < 1 || iters < 1 || scratch2 == nullptr)
    return n3host::set_error(N3_ERR_ARG, "calibrate: bad arguments");
  n3::det_ceiling_kernel<4><<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, blocks, scratch2);
  return n3host::check_launch("det_ceiling_kernel");
}
