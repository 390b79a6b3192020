// Device helpers shared by the persistent (cooperative) kernels.
#pragma once

#include "gkw_internal.cuh"

namespace gkw {

// Grid barrier for a cooperative launch, on one 32-bit word.  Each CTA adds
// to the word with release semantics: CTA 0 adds 2^31 - (gridDim - 1), the
// others add 1, so the top bit flips exactly when the last CTA arrives and
// the low 31 bits are back at zero for the next barrier.  Waiters spin on an
// acquire load until the top bit differs from what their own add returned.
// A CTA that waits longer than kGridBarrierCycles sets *err and returns false
// (the kernel then leaves; the host zeroes the word before the next launch).
constexpr long long kGridBarrierCycles = 4000000000ll;   // ~2 s at 2 GHz

__device__ __forceinline__ u32 atom_add_release_gpu(u32* p, u32 v) {
  u32 old;
  asm volatile("atom.add.release.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ u32 ld_acquire_gpu(const u32* p) {
  u32 v;
  asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ u32 cluster_ncta() {
  u32 r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ bool grid_barrier(GridBarrier* b, i32* err, i32* s_flag) {
  if (gridDim.x == 1) {   // a one-CTA launch: the block barrier is the grid barrier
    __syncthreads();
    return true;
  }
  if (cluster_ncta() == gridDim.x) {
    // the grid is one thread-block cluster (launch_coop): the hardware
    // cluster barrier, release/acquire at cluster scope
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
    return true;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const u32 add = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u;
    const u32 old = atom_add_release_gpu(&b->count, add);
    i32 bad = 0;
    if (((old ^ ld_acquire_gpu(&b->count)) & 0x80000000u) == 0) {
      const long long t0 = clock64();
      while (((old ^ ld_acquire_gpu(&b->count)) & 0x80000000u) == 0) {
        if (clock64() - t0 > kGridBarrierCycles) {
          atomicExch(err, 1);
          bad = 1;
          break;
        }
      }
    }
    *s_flag = bad;
  }
  __syncthreads();
  return *s_flag == 0;
}

// Grid barrier that also sums one count per CTA (thread 0's `mine`: the CTA's
// list appends in the phase before the barrier), so that the phase after it
// knows the list's length without another round trip to L2.  Three 64-bit
// words rotate: barrier k adds (mine << 32 | arrival) to word k % 3, whose
// arrival parts flip bit 31 exactly when the last CTA arrives, as in
// grid_barrier (the word starts at zero, so the low half never carries into
// the count).  The last CTA to arrive clears word (k + 2) % 3: every CTA has
// passed that word's last use (barrier k - 1), and none can reach its next use
// (barrier k + 2) before this CTA's release at barrier k + 1.  After the flip
// a word does not change until it is cleared, so every CTA reads the same
// total.  Words 0 and 1 must be zero before the first of these barriers (the
// level kernel's block 0 clears all three before an ordinary grid barrier
// that every CTA passes first).  A one-CTA or
// one-cluster grid sums nothing: *total = -1 and the caller loads its counter.
__device__ __forceinline__ u64 atom_add_release_gpu_u64(u64* p, u64 v) {
  u64 old;
  asm volatile("atom.add.release.gpu.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}

__device__ __forceinline__ u64 ld_acquire_gpu_u64(const u64* p) {
  u64 v;
  asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_barrier_count(CountBarrier* cb, u32 k, i32* err, i32* s_flag, i32* s_total,
                                                   u32 mine, i32* total) {
  if (gridDim.x == 1 || cluster_ncta() == gridDim.x) {
    *total = -1;
    return grid_barrier(nullptr, err, s_flag);   // these forms use no barrier word
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    u64* w = reinterpret_cast<u64*>(&cb->w[k % 3]);
    const u64 add = ((u64)mine << 32) | (u64)(blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u);
    const u64 old = atom_add_release_gpu_u64(w, add);
    u64 cur = old + add;
    i32 bad = 0;
    if (cur & 0x80000000ull) {   // the last arrival: cur is the word's final value
      cb->w[(k + 2) % 3] = 0;
    } else {
      const long long t0 = clock64();
      for (;;) {
        cur = ld_acquire_gpu_u64(w);
        if (cur & 0x80000000ull) break;
        if (clock64() - t0 > kGridBarrierCycles) {
          atomicExch(err, 1);
          bad = 1;
          break;
        }
      }
    }
    *s_flag = bad;
    *s_total = (i32)(u32)(cur >> 32);
  }
  __syncthreads();
  *total = *s_total;
  return *s_flag == 0;
}

__device__ __forceinline__ i32 ldcg(const i32* p) { return __ldcg(p); }
__device__ __forceinline__ u32 ldcg(const u32* p) { return __ldcg(p); }
__device__ __forceinline__ u64 ldcg(const u64* p) {
  return (u64)__ldcg(reinterpret_cast<const unsigned long long*>(p));
}

}  // namespace gkw
