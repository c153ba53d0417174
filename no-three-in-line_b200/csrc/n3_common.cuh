// Shared definitions of the n3 CUDA library (sm_100a).
//
// State layout in HBM and shared memory: the reference's interleaved slot
// layout (src/no_three_75/accelerated.py:18-24, src/no_three_75/tempering.py:38):
// slot s = 2*row + layer, row(s) = s >> 1, column = cols[s].  A state of an
// n x n grid has m = 2n slots.  Rows are implicit, so a state is m columns.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/n3.h"

namespace n3 {

constexpr int kMaxN = N3_MAX_N;        // 75: 150 slots, the reference's bound
constexpr int kMaxM = 2 * N3_MAX_N;    // 150
constexpr int kLutW = 2 * kMaxN - 1;   // dy in [-(kMaxN-1), kMaxN-1]
constexpr int kLutSize = kMaxN * kLutW;  // dx in [0, kMaxN-1]

// Device error word bits (written by kernels, read by the host after a sync).
enum : uint32_t {
  kErrColumnRange = 1u << 0,   // a column outside [0, n)
  kErrDuplicate = 1u << 1,     // two points of one row coincide
  kErrMismatch = 1u << 2,      // determinant and slope counts disagree
  kErrTimeout = 1u << 3,       // a bounded wait gave up
  kErrAudit = 1u << 4,         // incremental energy differs from a full recompute
  kErrCapacity = 1u << 5,      // an output list was longer than the caller's capacity
};

__device__ __forceinline__ int warp_sum(int v) { return __reduce_add_sync(0xffffffffu, v); }

}  // namespace n3

// Host-side helpers shared by the .cu files (defined in capi.cu).
namespace n3host {
int set_error(int code, const char* fmt, ...);
int check_launch(const char* what);
int ensure_device_tables();
int sm_count();
int allow_smem(const void* kernel, size_t bytes);
}  // namespace n3host

#define N3_TRY(expr)                      \
  do {                                    \
    const int n3_rc_ = (expr);            \
    if (n3_rc_ != N3_OK) return n3_rc_;   \
  } while (0)
