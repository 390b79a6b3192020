// Device helpers shared by the persistent (cooperative) kernels.
#pragma once

#include "gkw_internal.cuh"

namespace gkw {

// Grid barrier for a cooperative launch: a counter and a generation word.  A
// CTA that waits longer than kGridBarrierCycles sets *err and leaves; every
// later barrier then reports failure, so the kernel ends with an error status
// instead of a hang.
constexpr long long kGridBarrierCycles = 4000000000ll;   // ~2 s at 2 GHz

__device__ __forceinline__ bool grid_barrier(GridBarrier* b, i32* err, i32* s_flag) {
  if (gridDim.x == 1) {   // a one-CTA launch: the block barrier is the grid barrier
    __syncthreads();
    return true;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile u32* vgen = &b->gen;
    const u32 g = *vgen;
    __threadfence();
    const u32 arrived = atomicAdd(&b->count, 1u);
    if (arrived == gridDim.x - 1) {
      b->count = 0;
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      const long long t0 = clock64();
      while (*vgen == g) {
        if (clock64() - t0 > kGridBarrierCycles) {
          atomicExch(err, 1);
          break;
        }
        __nanosleep(20);
      }
    }
    __threadfence();
    *s_flag = *(volatile i32*)err;
  }
  __syncthreads();
  return *s_flag == 0;
}

__device__ __forceinline__ i32 ldcg(const i32* p) { return __ldcg(p); }
__device__ __forceinline__ u32 ldcg(const u32* p) { return __ldcg(p); }
__device__ __forceinline__ u64 ldcg(const u64* p) {
  return (u64)__ldcg(reinterpret_cast<const unsigned long long*>(p));
}

}  // namespace gkw
