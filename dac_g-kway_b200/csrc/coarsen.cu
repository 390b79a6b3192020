// Coarsening: heavy-edge candidates, union-find grouping, coarse ids, and
// contraction into the coarse CSR.  Semantics follow the reference's
// gkway/coarsen.hpp; the kernels are organised for B200 (sub-warp rows,
// shared-memory hashing, no host round trip per union-find iteration).
#include <algorithm>
#include <climits>
#include <cstddef>

#include "device_util.cuh"

namespace gkw {

static constexpr u32 kFull = 0xffffffffu;

// ===========================================================================
// Heavy-edge candidate (coarsen.hpp:39-78).  G lanes per vertex; each lane
// keeps the best entry of its stride of the row under the key
// (weight desc, neighbour degree asc, position asc), zero weights excluded;
// the G partial results are reduced by shuffles.  This is the serial rule of
// the reference: the first position with minimum degree among the maximum
// weight entries, or the vertex itself when no entry has positive weight.
// ===========================================================================
// Rows longer than kMatchLong are left to k_match_long (one CTA per row), so
// a hub row never holds its group's lanes for thousands of dependent loads.
constexpr i32 kMatchLong = 512;

// the candidate rule's order: weight desc, neighbour degree asc, position asc
__device__ __forceinline__ bool match_better(u32 w, u32 d, i32 pos, u32 bw, u32 bd, i32 bpos) {
  return w > bw || (w == bw && (d < bd || (d == bd && pos < bpos)));
}

template <int G>
__global__ void __launch_bounds__(256) k_match(i32 n, const i32* __restrict__ xadj,
                                               const i32* __restrict__ adjncy,
                                               const i32* __restrict__ adjwgt, i32* __restrict__ cand,
                                               i32* __restrict__ longlist, i32* __restrict__ longcnt) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i32 v = (i32)(t / G);
  const int sub = threadIdx.x & (G - 1);
  u32 bw = 0, bd = kFull;
  i32 bpos = INT_MAX, bu = -1;
  bool skip = false;
  if (v < n) {
    const i32 beg = __ldg(xadj + v), end = __ldg(xadj + v + 1);
    skip = longlist != nullptr && end - beg > kMatchLong;   // uniform within the group
    if (skip) {
      if (sub == 0) longlist[atomicAdd(longcnt, 1)] = v;
    } else {
      for (i32 e = beg + sub; e < end; e += G) {
        const u32 w = (u32)__ldg(adjwgt + e);
        if (w == 0 || w < bw) continue;
        const i32 u = __ldg(adjncy + e);
        const u32 d = (u32)(__ldg(xadj + u + 1) - __ldg(xadj + u));
        if (w > bw || d < bd) { bw = w; bd = d; bpos = e; bu = u; }
      }
    }
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    const u32 ow = __shfl_xor_sync(kFull, bw, o, G);
    const u32 od = __shfl_xor_sync(kFull, bd, o, G);
    const i32 op = __shfl_xor_sync(kFull, bpos, o, G);
    const i32 ou = __shfl_xor_sync(kFull, bu, o, G);
    if (match_better(ow, od, op, bw, bd, bpos)) { bw = ow; bd = od; bpos = op; bu = ou; }
  }
  if (v < n && sub == 0 && !skip) cand[v] = bw > 0 ? bu : v;
}

// One CTA per long row (listed by k_match): the threads stride the row --
// its 16-byte-aligned body four entries per load when both arrays are
// 16-byte aligned -- and the per-thread bests are reduced by the same rule.
constexpr int kMatchLongThreads = 256;
__global__ void __launch_bounds__(kMatchLongThreads) k_match_long(const i32* __restrict__ xadj,
                                                                  const i32* __restrict__ adjncy,
                                                                  const i32* __restrict__ adjwgt,
                                                                  i32* __restrict__ cand,
                                                                  const i32* __restrict__ longlist,
                                                                  const i32* __restrict__ longcnt) {
  __shared__ u32 s_w[kMatchLongThreads / 32], s_d[kMatchLongThreads / 32];
  __shared__ i32 s_p[kMatchLongThreads / 32], s_u[kMatchLongThreads / 32];
  const i32 nlong = *longcnt;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const bool vec = ((reinterpret_cast<uintptr_t>(adjncy) | reinterpret_cast<uintptr_t>(adjwgt)) & 15) == 0;
  for (i32 r = blockIdx.x; r < nlong; r += gridDim.x) {
    const i32 v = longlist[r];
    const i32 beg = xadj[v], end = xadj[v + 1];
    u32 bw = 0, bd = kFull;
    i32 bpos = INT_MAX, bu = -1;
    auto visit = [&](u32 w, i32 u, i32 e) {
      if (w == 0 || w < bw) return;
      const u32 d = (u32)(__ldg(xadj + u + 1) - __ldg(xadj + u));
      if (match_better(w, d, e, bw, bd, bpos)) { bw = w; bd = d; bpos = e; bu = u; }
    };
    i32 body = beg, tail = end;
    if (vec) {
      body = (beg + 3) & ~3;
      tail = body + ((end - body) & ~3);
      if (tail < body) tail = body;
      for (i32 e = beg + threadIdx.x; e < body && e < end; e += blockDim.x) visit((u32)adjwgt[e], adjncy[e], e);
      for (i32 c = body / 4 + threadIdx.x; c < tail / 4; c += blockDim.x) {
        const int4 w4 = __ldg(reinterpret_cast<const int4*>(adjwgt) + c);
        const int4 u4 = __ldg(reinterpret_cast<const int4*>(adjncy) + c);
        visit((u32)w4.x, u4.x, 4 * c);
        visit((u32)w4.y, u4.y, 4 * c + 1);
        visit((u32)w4.z, u4.z, 4 * c + 2);
        visit((u32)w4.w, u4.w, 4 * c + 3);
      }
      for (i32 e = (tail > body ? tail : body) + threadIdx.x; e < end; e += blockDim.x)
        visit((u32)adjwgt[e], adjncy[e], e);
    } else {
      for (i32 e = beg + threadIdx.x; e < end; e += blockDim.x) visit((u32)adjwgt[e], adjncy[e], e);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const u32 ow = __shfl_xor_sync(kFull, bw, o);
      const u32 od = __shfl_xor_sync(kFull, bd, o);
      const i32 op = __shfl_xor_sync(kFull, bpos, o);
      const i32 ou = __shfl_xor_sync(kFull, bu, o);
      if (match_better(ow, od, op, bw, bd, bpos)) { bw = ow; bd = od; bpos = op; bu = ou; }
    }
    if (lane == 0) {
      s_w[wid] = bw;
      s_d[wid] = bd;
      s_p[wid] = bpos;
      s_u[wid] = bu;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
        if (match_better(s_w[w], s_d[w], s_p[w], bw, bd, bpos)) { bw = s_w[w]; bd = s_d[w]; bpos = s_p[w]; bu = s_u[w]; }
      cand[v] = bw > 0 ? bu : v;
    }
    __syncthreads();
  }
}

i32 match_bucket(const DevGraph& g) {
  const double avg = g.n ? (double)g.m / g.n : 0.0;
  return avg <= 6.5 ? 0 : avg <= 14 ? 1 : avg <= 28 ? 2 : 3;
}

static void launch_match(Handle& h, const DevGraph& g, i32* cand, i32 G, i32* longlist, i32* longcnt) {
  const int threads = 256;
  auto go = [&](auto kern) {
    const i64 tot = (i64)g.n * G;
    launch(kern, (u32)((tot + threads - 1) / threads), threads, 0, h.stream, g.n, g.xadj, g.adjncy, g.adjwgt,
           cand, longlist, longcnt);
  };
  if (G == 2) go(k_match<2>);
  else if (G == 4) go(k_match<4>);
  else if (G == 8) go(k_match<8>);
  else if (G == 16) go(k_match<16>);
  else go(k_match<32>);
}

void time_match_variants(Handle& h, const DevGraph& g, i32* cand) {
  if (g.n == 0) return;
  const i32 b = match_bucket(g);
  cudaEvent_t e0, e1;
  GKW_CUDA(cudaEventCreate(&e0));
  GKW_CUDA(cudaEventCreate(&e1));
  Pool::Mark mk = h.scratch.mark();
  i32* longlist = h.scratch.alloc_n<i32>(g.n);
  i32* longcnt = h.scratch.alloc_n<i32>(1);
  const i32 lanes[kMatchLaneChoices] = {2, 4, 8, 16, 32};
  for (i32 q = 0; q < kMatchLaneChoices; ++q) {
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      GKW_CUDA(cudaMemsetAsync(longcnt, 0, sizeof(i32), h.stream));
      GKW_CUDA(cudaEventRecord(e0, h.stream));
      launch_match(h, g, cand, lanes[q], longlist, longcnt);
      GKW_CUDA(cudaEventRecord(e1, h.stream));
      GKW_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      GKW_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      best = std::min(best, ms);
    }
    h.tune_match_ms[b][q] += best;
  }
  h.scratch.release(mk);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

void run_match(Handle& h, const DevGraph& g, i32* cand, i64 maxdeg) {
  if (g.n == 0) return;
  const bool split = maxdeg < 0 || maxdeg > kMatchLong;
  Pool::Mark mk = h.scratch.mark();
  i32* longlist = split ? h.scratch.alloc_n<i32>(g.n) : nullptr;
  i32* longcnt = split ? h.scratch.alloc_n<i32>(1) : nullptr;
  if (split) GKW_CUDA(cudaMemsetAsync(longcnt, 0, sizeof(i32), h.stream));
  launch_match(h, g, cand, h.tuning.match_lanes[match_bucket(g)], longlist, longcnt);
  if (split)
    launch(k_match_long, (u32)h.sm_count * 2, kMatchLongThreads, 0, h.stream, g.xadj, g.adjncy, g.adjwgt, cand,
           (const i32*)longlist, (const i32*)longcnt);
  GKW_CHECK_LAUNCH();
  h.scratch.release(mk);
}

// ===========================================================================
// Union-find label propagation (coarsen.hpp:80-118, loop :461-469), Jacobi
// schedule, as one persistent cooperative kernel.  Keys are
// (label << 32 | round of last raise).  Round r reads buffer (r-1)&1 and
// raises buffer r&1 with atomicMax; that buffer still holds round r-2's keys,
// which never exceed round r-1's, so max(own key, pushes) is exactly the
// synchronous update.  chg[r&1] records whether round r raised anything; the
// grid barrier separates rounds and the loop ends after the first quiet
// round -- no host round trip per round.
// ===========================================================================
constexpr int kUfThreads = 512;
constexpr int kUfIlp = 2;   // vertices per thread whose loads are issued together

__global__ void __launch_bounds__(kUfThreads, 3) k_uf_persist(i32 n, const i32* __restrict__ cand, u64* k0, u64* k1,
                                                          i32* chg, GridBarrier* bar, i32* err, i32* rounds_out,
                                                          i32 max_rounds) {
  __shared__ i32 s_flag, s_any;
  const i64 stride = (i64)gridDim.x * blockDim.x;
  const i64 t0 = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  for (i64 v = t0; v < n; v += stride) {
    const u64 key = (u64)(u32)v << 32;
    k0[v] = key;
    k1[v] = key;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    chg[0] = 0;
    chg[1] = 0;
    chg[2] = 0;
  }
  if (!grid_barrier(bar, err, &s_flag)) return;
  i32 rounds = -1;
  for (i32 it = 1;; ++it) {
    if (it > max_rounds) {   // uniform across CTAs
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(err, 2);
      return;
    }
    const u64* src = (it & 1) ? k0 : k1;   // round it reads buffer (it-1)&1, raises it&1
    u64* dst = (it & 1) ? k1 : k0;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    bool diff = false;
    for (i64 v0 = t0; v0 < n; v0 += stride * kUfIlp) {
      // kUfIlp vertices at a time: their candidate loads, then their key
      // gathers, then the raises (one vertex's steps in the same order)
      i32 c[kUfIlp];
      u64 kv[kUfIlp], kc[kUfIlp];
#pragma unroll
      for (int q = 0; q < kUfIlp; ++q) {
        const i64 v = v0 + q * stride;
        c[q] = v < n ? cand[v] : 0;
      }
#pragma unroll
      for (int q = 0; q < kUfIlp; ++q) {
        const i64 v = v0 + q * stride;
        if (v < n) {
          kv[q] = ldcg(src + v);
          kc[q] = ldcg(src + c[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < kUfIlp; ++q) {
        const i64 v = v0 + q * stride;
        if (v >= n) continue;
        const u32 a = (u32)(kv[q] >> 32), b = (u32)(kc[q] >> 32);
        atomicMax((unsigned long long*)&dst[v], (unsigned long long)kv[q]);
        if (a > b) {
          atomicMax((unsigned long long*)&dst[c[q]], (unsigned long long)(((u64)a << 32) | (u32)it));
          diff = true;
        } else if (a < b) {
          atomicMax((unsigned long long*)&dst[v], (unsigned long long)(((u64)b << 32) | (u32)it));
          diff = true;
        }
      }
    }
    if (diff) s_any = 1;
    __syncthreads();
    // change flags rotate over three words: round it raises chg[it % 3], which
    // every thread reads after this round's barrier; block 0 clears
    // chg[(it + 1) % 3] now, whose last reads (round it - 2) all happened
    // before their CTAs arrived at the previous barrier
    if (threadIdx.x == 0 && s_any) atomicOr(&chg[it % 3], 1);
    if (blockIdx.x == 0 && threadIdx.x == 0) chg[(it + 1) % 3] = 0;
    if (!grid_barrier(bar, err, &s_flag)) return;
    if (ldcg(&chg[it % 3]) == 0) {
      rounds = it;
      break;
    }
  }
  // after the first quiet round both buffers hold the fixed point
  if (blockIdx.x == 0 && threadIdx.x == 0) *rounds_out = rounds;
}

// Writes the final keys to keys_out and the reference's round-launch count
// to *d_rounds (device).  No host synchronisation.
void run_union_find(Handle& h, i32 n, const i32* cand, u64* keys_out, i32* d_rounds) {
  if (n == 0) {
    const i32 one = 1;
    GKW_CUDA(cudaMemcpyAsync(d_rounds, &one, sizeof(i32), cudaMemcpyHostToDevice, h.stream));
    return;
  }
  Pool::Mark mk = h.scratch.mark();
  u64* kb = h.scratch.alloc_n<u64>(n);
  i32* chg = h.scratch.alloc_n<i32>(3);
  static int bps = 0;   // the same on every device of the process (one B200 model)
  if (!bps) GKW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_uf_persist, kUfThreads, 0));
  GKW_REQUIRE(bps >= 1, GKW_E_INTERNAL, "union-find kernel does not fit on an SM");
  i32 grid = std::min<i32>(h.sm_count * std::min(bps, 4), (i32)ceil_div(n, kUfThreads));
  grid = coop_grid(h, (const void*)k_uf_persist, grid, kUfThreads, 0);
  i32 max_rounds = n + 2;
  GridBarrier* barp = &h.coop->bar;
  i32* errp = &h.coop->err;
  void* args[] = {&n, &cand, &keys_out, &kb, &chg, &barp, &errp, &d_rounds, &max_rounds};
  launch_coop(h, (const void*)k_uf_persist, grid, kUfThreads, 0, args);
  h.scratch.release(mk);
}

// ===========================================================================
// Coarse ids (coarsen.hpp:351-421, 120-155, 474-481).  Sorted order is
// (root, dist, id); each root's run is cut into chunks of group_cap.  A
// group of size s gets ceil(s/cap) consecutive coarse ids starting at the
// exclusive scan of chunk counts over roots in id order.  Groups larger than
// the cap need the rank of each member in (dist, id) order: a warp sorts
// groups of <= 32 members in registers, a CTA sorts groups up to
// kGroupSmem members in shared memory, and bigger groups are sorted by a
// global bitonic network.
// ===========================================================================
constexpr i32 kGroupSmem = 4096;

__global__ void k_group_count(i32 n, const u64* __restrict__ keys, i32* __restrict__ gsize) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) atomicAdd(&gsize[(u32)(keys[v] >> 32)], 1);
}

// Coarse ids per root: ceil(size / cap) (scanned afterwards).  A group above
// the cap also takes its block of the member list here, from a counter with
// one atomic per warp: the blocks' order does not matter, since every group
// is ordered by (dist, id) within its own block.
__global__ void k_group_chunks(i32 n, const i32* __restrict__ gsize, i32 cap, i32* __restrict__ chunks,
                               i32* __restrict__ goff, i32* __restrict__ mcounter) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  i32 s = 0;
  if (v < n) {
    s = gsize[v];
    chunks[v] = (s + cap - 1) / cap;
  }
  const i32 big = s > cap ? s : 0;
  i32 inc = big;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const i32 y = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += y;
  }
  const i32 tot = __shfl_sync(kFull, inc, 31);
  i32 base = 0;
  if (lane == 31 && tot) base = atomicAdd(mcounter, tot);
  base = __shfl_sync(kFull, base, 31);
  if (big) goff[v] = base + inc - big;
}

// counts[]: [0] groups of 7..32 members (warp sort), [1] groups above kGroupSmem
// (global sort), [2] n_c, [3] members of big groups, [4] groups of
// 33..kGroupSmem members (CTA sort)
__global__ void k_group_scatter(i32 n, const u64* __restrict__ keys, const i32* __restrict__ gsize,
                                const i32* __restrict__ cbase, const i32* __restrict__ goff,
                                i32* __restrict__ gcur, i32 cap, i32* __restrict__ cmap,
                                i32* __restrict__ members, i32* __restrict__ biglist,
                                i32* __restrict__ ctalist, i32* __restrict__ giantlist, i32* __restrict__ counts) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 r = (i32)(u32)(keys[v] >> 32);
  const i32 s = gsize[r];
  if (s <= cap) {
    cmap[v] = cbase[r];
  } else {
    const i32 slot = atomicAdd(&gcur[r], 1);
    members[goff[r] + slot] = (i32)v;
    if (r == (i32)v) {
      if (s <= 32) biglist[atomicAdd(&counts[0], 1)] = r;
      else if (s <= kGroupSmem) ctalist[atomicAdd(&counts[4], 1)] = r;
      else giantlist[atomicAdd(&counts[1], 1)] = r;
    }
  }
}

__device__ __forceinline__ u64 umin64(u64 a, u64 b) { return a < b ? a : b; }
__device__ __forceinline__ u64 umax64(u64 a, u64 b) { return a < b ? b : a; }

// one warp per big group with <= 32 members (CTAs [0, nblocks) of the launch)
__device__ void group_sort_warps(const i32* __restrict__ biglist, const i32* __restrict__ counts,
                                 const u64* __restrict__ keys, const i32* __restrict__ gsize,
                                 const i32* __restrict__ goff, const i32* __restrict__ cbase,
                                 const i32* __restrict__ members, i32 cap, i32* __restrict__ cmap, u32 nblocks) {
  const i32 nbig = counts[0];
  const int lane = threadIdx.x & 31;
  const i64 warp0 = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const i64 nwarps = ((i64)nblocks * blockDim.x) >> 5;
  for (i64 w = warp0; w < nbig; w += nwarps) {
    const i32 r = biglist[w];
    const i32 s = gsize[r];
    if (s > 32) continue;   // warp-uniform
    u64 key = ~0ull;
    if (lane < s) {
      const i32 m = members[goff[r] + lane];
      key = ((keys[m] & 0xffffffffull) << 32) | (u32)m;   // (dist, id)
    }
#pragma unroll
    for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
      for (int j = kk >> 1; j > 0; j >>= 1) {
        const u64 o = __shfl_xor_sync(kFull, key, j);
        const bool up = (lane & kk) == 0;
        const bool lower = (lane & j) == 0;
        key = (lower == up) ? umin64(key, o) : umax64(key, o);
      }
    }
    if (lane < s) cmap[(u32)key] = cbase[r] + lane / cap;
  }
}

// Ascending bitonic sort of a[0..P) (P a power of two) by one CTA.
__device__ void cta_bitonic_u64(u64* a, i32 P) {
  for (i32 kk = 2; kk <= P; kk <<= 1) {
    for (i32 j = kk >> 1; j > 0; j >>= 1) {
      for (i32 i = threadIdx.x; i < P; i += blockDim.x) {
        const i32 l = i ^ j;
        if (l > i) {
          const u64 x = a[i], y = a[l];
          const bool up = (i & kk) == 0;
          if (up ? (x > y) : (x < y)) { a[i] = y; a[l] = x; }
        }
      }
      __syncthreads();
    }
  }
}

// one CTA per big group with 33..kGroupSmem members (CTA `cta` of `nctas`)
__device__ void group_sort_ctas(const i32* __restrict__ biglist, const i32* __restrict__ counts,
                                const u64* __restrict__ keys, const i32* __restrict__ gsize,
                                const i32* __restrict__ goff, const i32* __restrict__ cbase,
                                const i32* __restrict__ members, i32 cap, i32* __restrict__ cmap, u32 cta,
                                u32 nctas) {
  __shared__ u64 sk[kGroupSmem];
  const i32 nbig = counts[4];
  for (i32 b = (i32)cta; b < nbig; b += (i32)nctas) {
    const i32 r = biglist[b];
    const i32 s = gsize[r];
    i32 P = 64;
    while (P < s) P <<= 1;
    for (i32 i = threadIdx.x; i < P; i += blockDim.x) {
      u64 key = ~0ull;
      if (i < s) {
        const i32 m = members[goff[r] + i];
        key = ((keys[m] & 0xffffffffull) << 32) | (u32)m;
      }
      sk[i] = key;
    }
    __syncthreads();
    cta_bitonic_u64(sk, P);
    for (i32 i = threadIdx.x; i < s; i += blockDim.x) cmap[(u32)sk[i]] = cbase[r] + i / cap;
    __syncthreads();
  }
}

// The group orders of one level in one launch: CTAs [0, nwarp_blocks) sort
// the groups of up to 32 members by warps, the CTAs after them the groups of
// up to kGroupSmem members, one CTA each.
__global__ void k_group_sort(const i32* __restrict__ wlist, const i32* __restrict__ clist,
                             const i32* __restrict__ counts, const u64* __restrict__ keys,
                             const i32* __restrict__ gsize, const i32* __restrict__ goff,
                             const i32* __restrict__ cbase, const i32* __restrict__ members, i32 cap,
                             i32* __restrict__ cmap, u32 nwarp_blocks) {
  if (blockIdx.x < nwarp_blocks)
    group_sort_warps(wlist, counts, keys, gsize, goff, cbase, members, cap, cmap, nwarp_blocks);
  else
    group_sort_ctas(clist, counts, keys, gsize, goff, cbase, members, cap, cmap, blockIdx.x - nwarp_blocks,
                    gridDim.x - nwarp_blocks);
}

// Giant groups (more than kGroupSmem members, rare): every CTA of one
// cooperative launch sorts each giant group in turn with a bitonic network in
// global scratch, grid barriers between the stages.
__global__ void __launch_bounds__(512) k_giant_sort(const i32* __restrict__ giantlist, const i32* __restrict__ counts,
                                                    const u64* __restrict__ keys, const i32* __restrict__ gsize,
                                                    const i32* __restrict__ goff, const i32* __restrict__ cbase,
                                                    const i32* __restrict__ members, i32 cap, i32* __restrict__ cmap,
                                                    u64* a, GridBarrier* bar, i32* err) {
  __shared__ i32 s_flag;
  const i32 ng = counts[1];
  if (ng == 0) return;   // uniform: no barrier is entered
  const i64 stride = (i64)gridDim.x * blockDim.x;
  const i64 t0 = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  for (i32 gi = 0; gi < ng; ++gi) {
    const i32 r = giantlist[gi];
    const i32 s = gsize[r];
    i64 P = 1;
    while (P < s) P <<= 1;
    const i32* mem = members + goff[r];
    for (i64 i = t0; i < P; i += stride) {
      u64 key = ~0ull;
      if (i < s) {
        const i32 m = mem[i];
        key = ((keys[m] & 0xffffffffull) << 32) | (u32)m;
      }
      a[i] = key;
    }
    if (!grid_barrier(bar, err, &s_flag)) return;
    for (i64 kk = 2; kk <= P; kk <<= 1) {
      for (i64 j = kk >> 1; j > 0; j >>= 1) {
        for (i64 i = t0; i < P; i += stride) {
          const i64 l = i ^ j;
          if (l > i) {
            const u64 x = ldcg(a + i), y = ldcg(a + l);
            const bool up = (i & kk) == 0;
            if (up ? (x > y) : (x < y)) { a[i] = y; a[l] = x; }
          }
        }
        if (!grid_barrier(bar, err, &s_flag)) return;
      }
    }
    const i32 base = cbase[r];
    for (i64 i = t0; i < s; i += stride) cmap[(u32)ldcg(a + i)] = base + (i32)(i / cap);
    if (!grid_barrier(bar, err, &s_flag)) return;
  }
}

// cmap for every vertex and *d_nc = n_c (device).  No host synchronisation.
void run_group_map(Handle& h, i32 n, const u64* keys, i32 cap, i32* cmap, i32* d_nc) {
  GKW_REQUIRE(cap >= 1, GKW_E_INVALID, "group_cap must be >= 1");
  if (n == 0) {
    GKW_CUDA(cudaMemsetAsync(d_nc, 0, sizeof(i32), h.stream));
    return;
  }
  Pool::Mark mk = h.scratch.mark();
  const u32 nb = ceil_div(n, 256);
  i32* gsize = h.scratch.alloc_n<i32>(n);
  i32* chunks = h.scratch.alloc_n<i32>(n);
  i32* bigsz = h.scratch.alloc_n<i32>(n);
  i32* gcur = h.scratch.alloc_n<i32>(n);
  i32* members = h.scratch.alloc_n<i32>(n);
  i32* biglist = h.scratch.alloc_n<i32>(n);
  i32* giantlist = h.scratch.alloc_n<i32>(n);
  i32* ctalist = h.scratch.alloc_n<i32>(n);
  i32* counts = h.scratch.alloc_n<i32>(8);
  u64* gscratch = h.scratch.alloc_n<u64>(2 * (size_t)n);
  GKW_CUDA(cudaMemsetAsync(gsize, 0, sizeof(i32) * n, h.stream));
  GKW_CUDA(cudaMemsetAsync(gcur, 0, sizeof(i32) * n, h.stream));
  GKW_CUDA(cudaMemsetAsync(counts, 0, sizeof(i32) * 8, h.stream));
  launch(k_group_count, nb, 256, 0, h.stream, n, keys, gsize);
  launch(k_group_chunks, nb, 256, 0, h.stream, n, gsize, cap, chunks, bigsz, counts + 3);
  GKW_CHECK_LAUNCH();
  exclusive_scan_i32(h, chunks, chunks, n, d_nc);   // chunks -> chunk base, total = n_c
  launch(k_group_scatter, nb, 256, 0, h.stream, n, keys, gsize, chunks, bigsz, gcur, cap, cmap, members,
         biglist, ctalist, giantlist, counts);
  const u32 ng = std::max<u32>(1, std::min<u32>(ceil_div(n, 8 * 32), (u32)h.sm_count * 16));
  launch(k_group_sort, ng + (u32)h.sm_count * 2, 256, 0, h.stream, biglist, ctalist, counts, keys, gsize, bigsz,
         chunks, members, cap, cmap, ng);
  GKW_CHECK_LAUNCH();
  {
    const i32* gl = giantlist;
    const i32* cn = counts;
    const i32* gs = gsize;
    const i32* go = bigsz;
    const i32* cb = chunks;
    const i32* mb = members;
    i32 capv = cap;
    GridBarrier* barp = &h.coop->bar;
    i32* errp = &h.coop->err;
    void* args[] = {&gl, &cn, (void*)&keys, &gs, &go, &cb, &mb, &capv, &cmap, &gscratch, &barp, &errp};
    const i32 grid = coop_grid(h, (const void*)k_giant_sort, h.sm_count, 512, 0);
    launch_coop(h, (const void*)k_giant_sort, grid, 512, 0, args);
  }
  h.scratch.release(mk);
}

// ===========================================================================
// Contraction (coarsen.hpp:157-349).  Members of each coarse vertex are
// listed (at most group_cap of them); then one warp per coarse vertex hashes
// the mapped neighbour ids of all its members into shared memory, summing
// weights, drops the self id, sorts the distinct ids and writes the row to a
// staging area at an upper-bound offset; a scan of the row lengths gives the
// coarse xadj and a copy compacts the rows.  Rows longer than the warp's
// table go to a CTA with a larger shared table, and rows longer than that to
// a CTA with a table in global scratch.
// ===========================================================================
__global__ void k_coarse_accum(i32 n, const i32* __restrict__ xadj, const i32* __restrict__ vwgt,
                               const i32* __restrict__ cmap, i32 cap, i32* __restrict__ cvwgt,
                               i32* __restrict__ rowlen, i32* __restrict__ mcnt, i32* __restrict__ memtab,
                               ArenaHdr* arena) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v == 0 && arena) {
    arena->used = 0;
    arena->need = 0;
    arena->overflow = 0;
  }
  if (v >= n) return;
  const i32 c = cmap[v];
  atomicAdd((u32*)&cvwgt[c], (u32)vwgt[v]);
  atomicAdd(&rowlen[c], xadj[v + 1] - xadj[v]);
  const i32 slot = atomicAdd(&mcnt[c], 1);
  memtab[(i64)c * cap + slot] = (i32)v;
}

__device__ __forceinline__ u32 hash_u32(u32 x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

static constexpr u32 kEmpty = 0xffffffffu;

// Insert (key, w) into an open-addressing table of size hsz (power of two).
// The table always has free slots (hsz >= 2 * entries), so the probe ends;
// the probe count is still bounded by hsz.
__device__ __forceinline__ void table_add(u32* keys, u32* vals, u32 hsz, u32 key, u32 w) {
  u32 s = hash_u32(key) & (hsz - 1);
  for (u32 probe = 0; probe < hsz; ++probe) {
    const u32 prev = atomicCAS(&keys[s], kEmpty, key);
    if (prev == kEmpty || prev == key) {
      atomicAdd(&vals[s], w);
      return;
    }
    s = (s + 1) & (hsz - 1);
  }
}

template <int WCAP>
struct WarpTable {
  u32 keys[2 * WCAP];
  u32 vals[2 * WCAP];
  u64 out[WCAP];
};

// Warp-level ascending bitonic sort of a[0..P) in shared memory, P power of 2 >= 32.
__device__ void warp_bitonic_u64(u64* a, i32 P, int lane) {
  for (i32 kk = 2; kk <= P; kk <<= 1) {
    for (i32 j = kk >> 1; j > 0; j >>= 1) {
      for (i32 i = lane; i < P; i += 32) {
        const i32 l = i ^ j;
        if (l > i) {
          const u64 x = a[i], y = a[l];
          const bool up = (i & kk) == 0;
          if (up ? (x > y) : (x < y)) { a[i] = y; a[l] = x; }
        }
      }
      __syncwarp();
    }
  }
}

template <int WCAP, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_contract_warp(
    const i32* __restrict__ ncp, const i32* __restrict__ xadj, const i32* __restrict__ adjncy, const i32* __restrict__ adjwgt,
    const i32* __restrict__ cmap, const i32* __restrict__ memtab, const i32* __restrict__ mcnt, i32 cap,
    const i32* __restrict__ rowlen, const i32* __restrict__ ub, i32* __restrict__ sadj,
    i32* __restrict__ swgt, i32* __restrict__ cnt, i32* __restrict__ heavy, i32* __restrict__ nheavy) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpTable<WCAP>* tabs = reinterpret_cast<WarpTable<WCAP>*>(smem_raw);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  WarpTable<WCAP>& T = tabs[wid];
  const i32 nc = *ncp;
  const i64 nw = (i64)gridDim.x * WARPS;
  // The next coarse vertex's header (row length, member count, this lane's
  // member) is loaded while the current one is contracted: two of the five
  // dependent loads of a coarse row leave the chain.
  i64 c = (i64)blockIdx.x * WARPS + wid;
  i32 nL = 0, nnm = 0, nmv = 0;
  auto header = [&](i64 cc) {
    if (cc < nc) {
      nL = rowlen[cc];
      nnm = mcnt[cc];
      nmv = lane < cap ? memtab[cc * (i64)cap + lane] : 0;
    }
  };
  header(c);
  for (; c < nc; c += nw) {
    const i32 L = nL, nm = nnm, mv = nmv;
    header(c + nw);
    if (L > WCAP || nm > 32) {
      if (lane == 0) heavy[atomicAdd(nheavy, 1)] = (i32)c;
      continue;
    }
    // lane j < nm: member j's row; exclusive prefix of the row lengths
    i32 mbeg = 0, mlen = 0;
    if (lane < nm) {
      mbeg = xadj[mv];
      mlen = xadj[mv + 1] - mbeg;
    }
    const i32 o = ub[c];   // needed only at the writes
    i32 moff = mlen;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const i32 y = __shfl_up_sync(kFull, moff, o);
      if (lane >= o) moff += y;
    }
    moff -= mlen;
    // entry i of the concatenated rows -> its CSR position
    auto entry_pos = [&](i32 i) {
      i32 pos = -1;
      for (i32 jm = 0; jm < nm; ++jm) {
        const i32 oj = __shfl_sync(kFull, moff, jm);
        const i32 lj = __shfl_sync(kFull, mlen, jm);
        const i32 bj = __shfl_sync(kFull, mbeg, jm);
        if (i >= oj && i < oj + lj) pos = bj + (i - oj);
      }
      return pos;
    };
    // Rows whose entries other than self loops fit one per lane merge in
    // registers: every row of up to 32 entries, and rows of up to 64 entries
    // with at most 32 left after the self loops (the members' edges to one
    // another) are dropped -- most coarse rows of a mesh.
    u64 kv = ~0ull;
    bool in_regs = false;
    if (L <= 32) {
      const i32 pos = entry_pos(lane);
      if (lane < L) {
        const u32 key = (u32)cmap[adjncy[pos]];
        if (key != (u32)c) kv = ((u64)key << 32) | (u32)adjwgt[pos];
      }
      in_regs = true;
    } else if (L <= 64) {
      const i32 p0 = entry_pos(lane), p1 = entry_pos(lane + 32);
      u64 e0 = ~0ull, e1 = ~0ull;
      {
        const u32 k0 = (u32)cmap[adjncy[p0]];
        if (k0 != (u32)c) e0 = ((u64)k0 << 32) | (u32)adjwgt[p0];
      }
      if (lane + 32 < L) {
        const u32 k1 = (u32)cmap[adjncy[p1]];
        if (k1 != (u32)c) e1 = ((u64)k1 << 32) | (u32)adjwgt[p1];
      }
      const u32 m0 = __ballot_sync(kFull, e0 != ~0ull), m1 = __ballot_sync(kFull, e1 != ~0ull);
      const i32 n0 = __popc(m0), tot = n0 + __popc(m1);
      if (tot <= 32) {   // warp-uniform: compact the kept entries to one per lane
        const u32 lt = (1u << lane) - 1u;
        if (e0 != ~0ull) T.out[__popc(m0 & lt)] = e0;
        if (e1 != ~0ull) T.out[n0 + __popc(m1 & lt)] = e1;
        __syncwarp();
        kv = lane < tot ? T.out[lane] : ~0ull;
        __syncwarp();
        in_regs = true;
      }
    }
    if (in_regs) {
      // sort (key, w), merge equal keys (self loops are already out)
#pragma unroll
      for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
        for (int jj = kk >> 1; jj > 0; jj >>= 1) {
          const u64 ot = __shfl_xor_sync(kFull, kv, jj);
          const bool up = (lane & kk) == 0;
          const bool lower = (lane & jj) == 0;
          kv = (lower == up) ? umin64(kv, ot) : umax64(kv, ot);
        }
      }
      const u32 key = (u32)(kv >> 32);
      const u32 w = (u32)kv;
      const u32 kprev = __shfl_up_sync(kFull, key, 1);
      const u32 knext = __shfl_down_sync(kFull, key, 1);
      const bool head = lane == 0 || kprev != key;
      const bool last = lane == 31 || knext != key;
      // inclusive prefix sum of w (mod 2^32) and the start lane of each run
      u32 S = w;
      i32 start = head ? lane : 0;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const u32 y = __shfl_up_sync(kFull, S, d);
        const i32 z = __shfl_up_sync(kFull, start, d);
        if (lane >= d) {
          S += y;
          start = start > z ? start : z;
        }
      }
      const u32 before = __shfl_sync(kFull, S, start > 0 ? start - 1 : 0);
      const u32 total = S - (start > 0 ? before : 0u);
      const bool valid = last && key != 0xffffffffu;
      const u32 bal = __ballot_sync(kFull, valid);
      if (valid) {
        const i32 at = o + __popc(bal & ((1u << lane) - 1));
        sadj[at] = (i32)key;
        swgt[at] = (i32)total;
      }
      if (lane == 0) cnt[c] = __popc(bal);
      continue;
    }
    u32 hsz = 64;
    while (hsz < 2u * (u32)L) hsz <<= 1;
    for (u32 i = lane; i < hsz; i += 32) { T.keys[i] = kEmpty; T.vals[i] = 0; }
    __syncwarp();
    for (i32 b = 0; b < L; b += 32) {
      const i32 i = b + lane;
      const i32 pos = entry_pos(i);
      if (i < L) {
        const u32 key = (u32)cmap[adjncy[pos]];
        if (key != (u32)c) table_add(T.keys, T.vals, hsz, key, (u32)adjwgt[pos]);
      }
    }
    __syncwarp();
    // compact occupied slots
    i32 U = 0;
    for (u32 base = 0; base < hsz; base += 32) {
      const u32 sl = base + lane;
      const bool occ = T.keys[sl] != kEmpty;
      const u32 bal = __ballot_sync(kFull, occ);
      if (occ) {
        const i32 at = U + __popc(bal & ((1u << lane) - 1));
        T.out[at] = ((u64)T.keys[sl] << 32) | T.vals[sl];
      }
      U += __popc(bal);
    }
    __syncwarp();
    if (U <= 32) {
      u64 key = lane < U ? T.out[lane] : ~0ull;
#pragma unroll
      for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
        for (int jj = kk >> 1; jj > 0; jj >>= 1) {
          const u64 ot = __shfl_xor_sync(kFull, key, jj);
          const bool up = (lane & kk) == 0;
          const bool lower = (lane & jj) == 0;
          key = (lower == up) ? umin64(key, ot) : umax64(key, ot);
        }
      }
      if (lane < U) {
        sadj[o + lane] = (i32)(u32)(key >> 32);
        swgt[o + lane] = (i32)(u32)key;
      }
    } else {
      i32 P = 64;
      while (P < U) P <<= 1;
      for (i32 i = U + lane; i < P; i += 32) T.out[i] = ~0ull;
      __syncwarp();
      warp_bitonic_u64(T.out, P, lane);
      for (i32 i = lane; i < U; i += 32) {
        const u64 kv = T.out[i];
        sadj[o + i] = (i32)(u32)(kv >> 32);
        swgt[o + i] = (i32)(u32)kv;
      }
    }
    if (lane == 0) cnt[c] = U;
    __syncwarp();
  }
}

// One CTA per heavy coarse row.  Table in dynamic shared memory when the row
// fits (L <= cta_cap); longer rows take their table from the handle's arena
// (bump allocation: keys and values of hsz words each, then hsz/2 sorted
// outputs as u64).  A row that does not fit in the arena records the words it
// needs and sets the overflow flag; the host grows the arena and runs the
// contraction again.  Both kinds of row run in one launch.
__global__ void __launch_bounds__(512) k_contract_cta(
    const i32* __restrict__ heavy, const i32* __restrict__ nheavy, i32 cta_cap,
    const i32* __restrict__ xadj, const i32* __restrict__ adjncy, const i32* __restrict__ adjwgt,
    const i32* __restrict__ cmap, const i32* __restrict__ memtab, const i32* __restrict__ mcnt, i32 cap,
    const i32* __restrict__ rowlen, const i32* __restrict__ ub, i32* __restrict__ sadj,
    i32* __restrict__ swgt, i32* __restrict__ cnt, ArenaHdr* arena, u32* arena_words, u64 arena_cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ i32 s_count;
  __shared__ u64 s_off;
  const i32 nh = *nheavy;
  for (i32 b = blockIdx.x; b < nh; b += gridDim.x) {
    const i32 c = heavy[b];
    const i32 L = rowlen[c];
    const bool global_table = L > cta_cap;   // block-uniform
    u32 hsz = 64;
    while (hsz < 2u * (u32)L) hsz <<= 1;
    u32 *keys, *vals;
    u64* out;
    if (global_table) {
      const u64 words = 3ull * hsz;   // keys + vals + hsz/2 u64 outputs
      if (threadIdx.x == 0) {
        const u64 off = atomicAdd((unsigned long long*)&arena->used, (unsigned long long)words);
        if (off + words > arena_cap) {
          atomicAdd((unsigned long long*)&arena->need, (unsigned long long)words);
          atomicExch(&arena->overflow, 1);
          s_off = ~0ull;
        } else {
          s_off = off;
        }
      }
      __syncthreads();
      const u64 off = s_off;
      __syncthreads();   // every thread has read s_off before thread 0 can set it for the next row
      if (off == ~0ull) continue;   // block-uniform; redone after the arena grows
      keys = arena_words + off;
      vals = keys + hsz;
      out = reinterpret_cast<u64*>(vals + hsz);
    } else {
      keys = reinterpret_cast<u32*>(smem_raw);
      vals = keys + 2 * cta_cap;
      out = reinterpret_cast<u64*>(vals + 2 * cta_cap);
    }
    for (u32 i = threadIdx.x; i < hsz; i += blockDim.x) { keys[i] = kEmpty; vals[i] = 0; }
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    const i32 nm = mcnt[c];
    for (i32 j = 0; j < nm; ++j) {
      const i32 v = memtab[c * (i64)cap + j];
      const i32 beg = xadj[v], end = xadj[v + 1];
      for (i32 e = beg + threadIdx.x; e < end; e += blockDim.x) {
        const u32 key = (u32)cmap[adjncy[e]];
        if (key != (u32)c) table_add(keys, vals, hsz, key, (u32)adjwgt[e]);
      }
    }
    __syncthreads();
    for (u32 sl = threadIdx.x; sl < hsz; sl += blockDim.x) {
      if (keys[sl] != kEmpty) {
        const i32 pos = atomicAdd(&s_count, 1);
        out[pos] = ((u64)keys[sl] << 32) | vals[sl];
      }
    }
    __syncthreads();
    const i32 U = s_count;
    i32 P = 64;
    while (P < U) P <<= 1;
    for (i32 i = U + threadIdx.x; i < P; i += blockDim.x) out[i] = ~0ull;
    __syncthreads();
    cta_bitonic_u64(out, P);
    const i32 o = ub[c];
    for (i32 i = threadIdx.x; i < U; i += blockDim.x) {
      const u64 kv = out[i];
      sadj[o + i] = (i32)(u32)(kv >> 32);
      swgt[o + i] = (i32)(u32)kv;
    }
    if (threadIdx.x == 0) cnt[c] = U;
    __syncthreads();
  }
}

// One warp per 32 consecutive coarse rows: the lanes scan the rows' lengths
// and copy the 32 rows' entries as one flat range, each lane finding its
// entry's row by a binary search over the lanes' prefix sums.  A hub row of
// thousands of entries is then copied by all 32 lanes, not by one thread.
// Also the level's longest coarse row and heaviest coarse vertex (both
// *maxdeg and *max_cvw start at zero).
__global__ void k_copy_rows(const i32* __restrict__ ncp, const i32* __restrict__ ub, const i32* __restrict__ cnt,
                            const i32* __restrict__ cx, const i32* __restrict__ sadj,
                            const i32* __restrict__ swgt, i32* __restrict__ cadj, i32* __restrict__ cwgt,
                            i32* __restrict__ maxdeg, const i32* __restrict__ cvw, i32* __restrict__ max_cvw) {
  const i32 nc = *ncp;
  const int lane = threadIdx.x & 31;
  const i64 warp = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const i64 nwarps = ((i64)gridDim.x * blockDim.x) >> 5;
  i32 mx = 0, mw = 0;
  for (i64 c0 = warp * 32; c0 < nc; c0 += nwarps * 32) {
    const i64 c = c0 + lane;
    i32 src = 0, dst = 0, len = 0;
    if (c < nc) {
      src = ub[c];
      dst = cx[c];
      len = cnt[c];
      mw = cvw[c] > mw ? cvw[c] : mw;
    }
    mx = len > mx ? len : mx;
    i32 inc = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const i32 y = __shfl_up_sync(kFull, inc, o);
      if (lane >= o) inc += y;
    }
    const i32 total = __shfl_sync(kFull, inc, 31);
    const i32 exc = inc - len;
    for (i32 base = 0; base < total; base += 32) {   // warp-uniform: every lane takes every shuffle
      const i32 idx = base + lane;
      // the row r with exc_r <= idx < inc_r: the first lane whose inclusive sum exceeds idx
      i32 r = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const i32 probe = __shfl_sync(kFull, inc, r + step - 1);
        if (probe <= idx) r += step;
      }
      r = r < 31 ? r : 31;
      const i32 rs = __shfl_sync(kFull, src, r), rd = __shfl_sync(kFull, dst, r), re = __shfl_sync(kFull, exc, r);
      if (idx < total) {
        cadj[rd + (idx - re)] = sadj[rs + (idx - re)];
        cwgt[rd + (idx - re)] = swgt[rs + (idx - re)];
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const i32 y = __shfl_xor_sync(kFull, mx, o);
    mx = mx > y ? mx : y;
    const i32 z = __shfl_xor_sync(kFull, mw, o);
    mw = mw > z ? mw : z;
  }
  if (lane == 0 && mx > 0) atomicMax(maxdeg, mx);
  if (lane == 0 && mw > 0) atomicMax(max_cvw, mw);
}

void ensure_arena(Handle& h, u64 words) {
  if (h.arena && h.arena_words >= words) return;
  GKW_REQUIRE(!h.capturing, GKW_E_INTERNAL, "arena grown during a graph capture");
  graph_cache_clear(h);   // graphs hold the old arena's address
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  if (h.arena) GKW_CUDA(cudaFree(h.arena));
  h.arena = nullptr;
  h.arena_words = 0;
  GKW_CUDA(cudaMalloc(&h.arena, sizeof(ArenaHdr) + sizeof(u32) * words));
  // on the handle's stream: that stream does not wait for the legacy stream
  GKW_CUDA(cudaMemsetAsync(h.arena, 0, sizeof(ArenaHdr), h.stream));
  h.arena_words = words;
}

void run_contract(Handle& h, const DevGraph& g, const i32* cmap, const i32* d_nc, i32 nc_ub, i32 cap, i32* cxadj,
                  i32* cadjncy, i32* cadjwgt, i32* cvwgt, i32* d_mc) {
  Pool::Mark mk = h.scratch.mark();
  const i32 n = g.n;
  const i64 nu = (i64)nc_ub + 1;
  const u32 nb = ceil_div(std::max(n, 1), 256);
  i32* rowlen = h.scratch.alloc_n<i32>(nu);
  i32* ub = h.scratch.alloc_n<i32>(nu);
  i32* mcnt = h.scratch.alloc_n<i32>(nu);
  i32* memtab = h.scratch.alloc_n<i32>((i64)nc_ub * cap + 1);
  i32* cnt = h.scratch.alloc_n<i32>(nu);
  i32* heavy = h.scratch.alloc_n<i32>(nu);
  i32* misc = h.scratch.alloc_n<i32>(8);   // [0] heavy rows, [1] ub total
  i32* sadj = h.scratch.alloc_n<i32>(std::max<i64>(g.m, 1));
  i32* swgt = h.scratch.alloc_n<i32>(std::max<i64>(g.m, 1));
  ensure_arena(h, u64(4) << 20);   // 16 MB of long-row tables to start with
  GKW_CUDA(cudaMemsetAsync(cvwgt, 0, sizeof(i32) * std::max(nc_ub, 1), h.stream));
  GKW_CUDA(cudaMemsetAsync(rowlen, 0, sizeof(i32) * nu, h.stream));
  GKW_CUDA(cudaMemsetAsync(mcnt, 0, sizeof(i32) * nu, h.stream));
  GKW_CUDA(cudaMemsetAsync(cnt, 0, sizeof(i32) * nu, h.stream));
  GKW_CUDA(cudaMemsetAsync(misc, 0, sizeof(i32) * 8, h.stream));
  if (n > 0)
    launch(k_coarse_accum, nb, 256, 0, h.stream, n, g.xadj, g.vwgt, cmap, cap, cvwgt, rowlen, mcnt, memtab, h.arena);
  GKW_CHECK_LAUNCH();
  exclusive_scan_i32(h, rowlen, ub, nu, misc + 1);   // rows beyond n_c have length 0
  const double avgL = nc_ub ? (double)g.m / nc_ub : 0.0;
  const u32 gridw = std::max<u32>(1, std::min<u32>(ceil_div(std::max(nc_ub, 1), 8), (u32)h.sm_count * 32));
  u32* words = reinterpret_cast<u32*>(h.arena + 1);
  if (avgL <= 48) {
    constexpr int W = 128, WARPS = 8;
    const size_t sm = sizeof(WarpTable<W>) * WARPS;
    if (!h.capturing)
      GKW_CUDA(cudaFuncSetAttribute(k_contract_warp<W, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    launch(k_contract_warp<W, WARPS>, gridw, WARPS * 32, sm, h.stream, d_nc, g.xadj, g.adjncy, g.adjwgt, cmap,
           memtab, mcnt, cap, rowlen, ub, sadj, swgt, cnt, heavy, misc);
  } else {
    constexpr int W = 512, WARPS = 8;
    const size_t sm = sizeof(WarpTable<W>) * WARPS;
    if (!h.capturing)
      GKW_CUDA(cudaFuncSetAttribute(k_contract_warp<W, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    launch(k_contract_warp<W, WARPS>, gridw, WARPS * 32, sm, h.stream, d_nc, g.xadj, g.adjncy, g.adjwgt, cmap,
           memtab, mcnt, cap, rowlen, ub, sadj, swgt, cnt, heavy, misc);
  }
  GKW_CHECK_LAUNCH();
  // heavy rows: a shared-memory table up to kCtaCap entries, the arena beyond
  // (2*kCtaCap table slots, a power of two, + kCtaCap sorted outputs: 96 KB)
  constexpr i32 kCtaCap = 4096;
  const size_t csm = (size_t)kCtaCap * 2 * 4 * 2 + (size_t)kCtaCap * 8;
  if (!h.capturing)
    GKW_CUDA(cudaFuncSetAttribute(k_contract_cta, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm));
  launch(k_contract_cta, (u32)h.sm_count * 2, 512, csm, h.stream, heavy, misc, kCtaCap, g.xadj, g.adjncy,
         g.adjwgt, cmap, memtab, mcnt, cap, rowlen, ub, sadj, swgt, cnt, h.arena, words, h.arena_words);
  GKW_CHECK_LAUNCH();
  exclusive_scan_i32(h, cnt, cxadj, nu, d_mc);   // cxadj[n_c] = m_c (rows beyond n_c are empty)
  if (nc_ub > 0)
    launch(k_copy_rows, ceil_div(nc_ub, 256), 256, 0, h.stream, d_nc, ub, cnt, cxadj, sadj, swgt, cadjncy,
           cadjwgt, &h.coop->maxdeg, (const i32*)cvwgt, &h.coop->max_cvw);
  GKW_CHECK_LAUNCH();
  h.scratch.release(mk);
}

CoopState read_coop(Handle& h) {
  CoopState* hc = reinterpret_cast<CoopState*>(h.h_pinned);
  static_assert(sizeof(CoopState) + sizeof(ArenaHdr) + 8 <= 64 * sizeof(i64), "pinned staging too small");
  GKW_CUDA(cudaMemcpyAsync(hc, h.coop, sizeof(CoopState), cudaMemcpyDeviceToHost, h.stream));
  ArenaHdr* ha = reinterpret_cast<ArenaHdr*>(hc + 1);
  if (h.arena) GKW_CUDA(cudaMemcpyAsync(ha, h.arena, sizeof(ArenaHdr), cudaMemcpyDeviceToHost, h.stream));
  i32* hs = reinterpret_cast<i32*>(ha + 1);
  if (h.scan) GKW_CUDA(cudaMemcpyAsync(hs, &h.scan->err, sizeof(i32), cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  CoopState c = *hc;
  c.arena_overflow = h.arena ? ha->overflow : 0;
  c.arena_need = h.arena ? (i64)ha->need : 0;
  c.scan_err = h.scan ? *hs : 0;
  if (c.err || c.scan_err) {   // report once, leave the handle usable
    GKW_CUDA(cudaMemsetAsync(h.coop, 0, sizeof(CoopState), h.stream));
    if (h.scan) GKW_CUDA(cudaMemsetAsync(&h.scan->err, 0, sizeof(i32), h.stream));
    GKW_CUDA(cudaStreamSynchronize(h.stream));
  }
  if (c.err == 1) throw Error{GKW_E_INTERNAL, "cooperative kernel: grid barrier timed out"};
  if (c.err == 2) throw Error{GKW_E_INTERNAL, "union-find did not converge"};
  if (c.scan_err) throw Error{GKW_E_INTERNAL, "scan: look-back wait timed out"};
  return c;
}

// ===========================================================================
// Fused coarsening step: one persistent launch per level runs every phase of
// the step above -- heavy-edge candidates, union-find rounds, group sizes and
// coarse ids, group orders, member lists, contraction, coarse xadj and row
// compaction -- with grid barriers between the phases instead of about twenty
// kernel launches and ten memsets.  The phase bodies apply the same rules to
// the same keys as the per-phase kernels, so the level is identical; the
// scans are grid-wide (each CTA scans a contiguous range after a barrier
// publishes the CTA sums).  Data written by other CTAs in the launch is read
// with ld.global.cg.  Dynamic shared memory (96 KB) is shared by the phases:
// the warps' contraction tables, the CTA group sorts and the CTA table of
// heavy coarse rows.
// ===========================================================================
constexpr int kFusedThreads = 512;
constexpr int kFusedWarps = kFusedThreads / 32;
constexpr i32 kFusedWcap = 128;      // warp table entries (as k_contract_warp<128, 8>)
constexpr i32 kFusedCtaCap = 4096;   // heavy rows up to this length use the shared table
constexpr size_t kFusedSmem = (size_t)kFusedCtaCap * 2 * 4 * 2 + (size_t)kFusedCtaCap * 8;   // 96 KB
static_assert(kFusedSmem >= sizeof(WarpTable<kFusedWcap>) * kFusedWarps, "warp tables fit");
static_assert(kFusedSmem >= sizeof(u64) * kGroupSmem, "CTA group sort fits");

// misc counters of the fused step (zeroed by the host before the launch)
enum { kFzLong = 0, kFzWarpG = 1, kFzGiant = 2, kFzCtaG = 3, kFzHeavy = 4, kFzBig = 5, kFzUb = 6, kFzWords = 8 };

struct FusedArgs {
  i32 n;
  i64 m;
  const i32* xadj;
  const i32* adjncy;
  const i32* adjwgt;
  const i32* vwgt;
  i32 lanes;     // match lanes per vertex (4, 8, 16, 32)
  i32 split;     // rows above kMatchLong may exist
  i32 cap;       // group cap
  i32 max_rounds;
  // outputs (coarse level at upper bounds)
  i32* cmap;
  i32* cxadj;
  i32* cadjncy;
  i32* cadjwgt;
  i32* cvwgt;
  // scratch
  i32* cand;
  u64* k0;
  u64* k1;
  i32* chg;        // [3]
  i32* longlist;   // [n]
  i32* gsize;      // [n]
  i32* cbase;      // [n] first coarse id of each root
  i32* goff;       // [n] member offset of each big group
  i32* gcur;       // [n]
  i32* members;    // [n]
  i32* wlist;      // [n] groups sorted by a warp
  i32* clist;      // [n] groups sorted by a CTA
  i32* glist;      // [n] giant groups
  u64* gscratch;   // [2n] giant sort network
  i32* rowlen;     // [n + 1]
  i32* ub;         // [n + 1]
  i32* mcnt;       // [n + 1]
  i32* memtab;     // [n * cap + 1]
  i32* cnt;        // [n + 1]
  i32* heavy;      // [n + 1]
  i32* sadj;       // [m]
  i32* swgt;       // [m]
  i32* partial;    // [2 * grid] CTA sums of the grid scans
  i32* misc;       // [kFzWords]
  // per-level scalars and barrier (CoopState)
  GridBarrier* bar;
  i32* err;
  i32* nc_out;
  i32* mc_out;
  i32* uf_rounds_out;
  i32* maxdeg_out;
  i32* max_cvw_out;
  ArenaHdr* arena;
  u32* arena_words;
  u64 arena_cap;
};

template <int G>
__device__ void fz_match(const FusedArgs& a) {
  const i64 tot = (i64)a.n * G;
  const i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 base = (i64)blockIdx.x * blockDim.x; base < tot; base += stride) {   // block-uniform trip count
    const i64 t = base + threadIdx.x;
    const i32 v = (i32)(t / G);
    const int sub = threadIdx.x & (G - 1);
    u32 bw = 0, bd = kFull;
    i32 bpos = INT_MAX, bu = -1;
    bool skip = false;
    if (v < a.n) {
      const i32 beg = __ldg(a.xadj + v), end = __ldg(a.xadj + v + 1);
      skip = a.split && end - beg > kMatchLong;   // uniform within the group
      if (skip) {
        if (sub == 0) a.longlist[atomicAdd(a.misc + kFzLong, 1)] = v;
      } else {
        for (i32 e = beg + sub; e < end; e += G) {
          const u32 w = (u32)__ldg(a.adjwgt + e);
          if (w == 0 || w < bw) continue;
          const i32 u = __ldg(a.adjncy + e);
          const u32 d = (u32)(__ldg(a.xadj + u + 1) - __ldg(a.xadj + u));
          if (w > bw || d < bd) { bw = w; bd = d; bpos = e; bu = u; }
        }
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const u32 ow = __shfl_xor_sync(kFull, bw, o, G);
      const u32 od = __shfl_xor_sync(kFull, bd, o, G);
      const i32 op = __shfl_xor_sync(kFull, bpos, o, G);
      const i32 ou = __shfl_xor_sync(kFull, bu, o, G);
      if (match_better(ow, od, op, bw, bd, bpos)) { bw = ow; bd = od; bpos = op; bu = ou; }
    }
    if (v < a.n && sub == 0 && !skip) a.cand[v] = bw > 0 ? bu : v;
  }
}

// Long rows listed by fz_match: one CTA per row, as k_match_long (the rule's
// order is total, so the thread count does not change the pick).
__device__ void fz_match_long(const FusedArgs& a) {
  __shared__ u32 s_w[kFusedWarps], s_d[kFusedWarps];
  __shared__ i32 s_p[kFusedWarps], s_u[kFusedWarps];
  const i32 nlong = ldcg(a.misc + kFzLong);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const bool vec = ((reinterpret_cast<uintptr_t>(a.adjncy) | reinterpret_cast<uintptr_t>(a.adjwgt)) & 15) == 0;
  for (i32 r = blockIdx.x; r < nlong; r += gridDim.x) {
    const i32 v = ldcg(a.longlist + r);
    const i32 beg = a.xadj[v], end = a.xadj[v + 1];
    u32 bw = 0, bd = kFull;
    i32 bpos = INT_MAX, bu = -1;
    auto visit = [&](u32 w, i32 u, i32 e) {
      if (w == 0 || w < bw) return;
      const u32 d = (u32)(__ldg(a.xadj + u + 1) - __ldg(a.xadj + u));
      if (match_better(w, d, e, bw, bd, bpos)) { bw = w; bd = d; bpos = e; bu = u; }
    };
    if (vec) {
      i32 body = (beg + 3) & ~3;
      i32 tail = body + ((end - body) & ~3);
      if (tail < body) tail = body;
      for (i32 e = beg + threadIdx.x; e < body && e < end; e += blockDim.x) visit((u32)a.adjwgt[e], a.adjncy[e], e);
      for (i32 c = body / 4 + threadIdx.x; c < tail / 4; c += blockDim.x) {
        const int4 w4 = __ldg(reinterpret_cast<const int4*>(a.adjwgt) + c);
        const int4 u4 = __ldg(reinterpret_cast<const int4*>(a.adjncy) + c);
        visit((u32)w4.x, u4.x, 4 * c);
        visit((u32)w4.y, u4.y, 4 * c + 1);
        visit((u32)w4.z, u4.z, 4 * c + 2);
        visit((u32)w4.w, u4.w, 4 * c + 3);
      }
      for (i32 e = (tail > body ? tail : body) + threadIdx.x; e < end; e += blockDim.x)
        visit((u32)a.adjwgt[e], a.adjncy[e], e);
    } else {
      for (i32 e = beg + threadIdx.x; e < end; e += blockDim.x) visit((u32)a.adjwgt[e], a.adjncy[e], e);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const u32 ow = __shfl_xor_sync(kFull, bw, o);
      const u32 od = __shfl_xor_sync(kFull, bd, o);
      const i32 op = __shfl_xor_sync(kFull, bpos, o);
      const i32 ou = __shfl_xor_sync(kFull, bu, o);
      if (match_better(ow, od, op, bw, bd, bpos)) { bw = ow; bd = od; bpos = op; bu = ou; }
    }
    if (lane == 0) {
      s_w[wid] = bw;
      s_d[wid] = bd;
      s_p[wid] = bpos;
      s_u[wid] = bu;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < kFusedWarps; ++w)
        if (match_better(s_w[w], s_d[w], s_p[w], bw, bd, bpos)) { bw = s_w[w]; bd = s_d[w]; bpos = s_p[w]; bu = s_u[w]; }
      a.cand[v] = bw > 0 ? bu : v;
    }
    __syncthreads();
  }
}

// Block-wide exclusive scan of two i32 per thread; the block totals in tx, ty.
__device__ __forceinline__ void fz_block_exscan2(i32& x, i32& y, i32* s_warp, i32& tx, i32& ty) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  i32 ix = x, iy = y;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const i32 px = __shfl_up_sync(kFull, ix, o), py = __shfl_up_sync(kFull, iy, o);
    if (lane >= o) { ix += px; iy += py; }
  }
  if (lane == 31) { s_warp[wid] = ix; s_warp[32 + wid] = iy; }
  __syncthreads();
  if (wid == 0) {
    const i32 wx = lane < kFusedWarps ? s_warp[lane] : 0, wy = lane < kFusedWarps ? s_warp[32 + lane] : 0;
    i32 sx = wx, sy = wy;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const i32 px = __shfl_up_sync(kFull, sx, o), py = __shfl_up_sync(kFull, sy, o);
      if (lane >= o) { sx += px; sy += py; }
    }
    if (lane < kFusedWarps) { s_warp[lane] = sx - wx; s_warp[32 + lane] = sy - wy; }
    if (lane == kFusedWarps - 1) { s_warp[64] = sx; s_warp[65] = sy; }
  }
  __syncthreads();
  x = ix - x + s_warp[wid];
  y = iy - y + s_warp[32 + wid];
  tx = s_warp[64];
  ty = s_warp[65];
  __syncthreads();
}

// Grid-wide exclusive scan of two sequences of N items inside the launch.
// CTA b owns the contiguous range [b*span, (b+1)*span): pass 1 sums it, a
// grid barrier publishes the CTA sums, pass 2 scans the range starting from
// the sum of the lower CTAs.  item(i) -> (x, y); out(i, ex, ey) stores.  The
// last CTA stores the totals through tot(tx, ty).  Integer sums: the result
// equals a sequential exclusive scan.  Returns false if the barrier failed.
template <class Item, class Out, class Tot>
__device__ bool fz_grid_scan2(const FusedArgs& a, i64 N, Item item, Out out, Tot tot, i32* s_flag) {
  __shared__ i32 s_warp[66];
  __shared__ i32 s_pre[2];
  const i64 span = (N + gridDim.x - 1) / gridDim.x;
  const i64 lo = (i64)blockIdx.x * span, hi = lo + span < N ? lo + span : N;
  i32 sx = 0, sy = 0;
  for (i64 i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    i32 x, y;
    item(i, x, y);
    sx += x;
    sy += y;
  }
  i32 tx, ty;
  fz_block_exscan2(sx, sy, s_warp, tx, ty);
  if (threadIdx.x == 0) {
    a.partial[2 * blockIdx.x] = tx;
    a.partial[2 * blockIdx.x + 1] = ty;
  }
  if (!grid_barrier(a.bar, a.err, s_flag)) return false;
  if (threadIdx.x < 32) {
    i32 px = 0, py = 0;
    for (i32 b = threadIdx.x; b < (i32)blockIdx.x; b += 32) {
      px += ldcg(a.partial + 2 * b);
      py += ldcg(a.partial + 2 * b + 1);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      px += __shfl_xor_sync(kFull, px, o);
      py += __shfl_xor_sync(kFull, py, o);
    }
    if (threadIdx.x == 0) { s_pre[0] = px; s_pre[1] = py; }
  }
  __syncthreads();
  i32 cx = s_pre[0], cy = s_pre[1];
  for (i64 b0 = lo; b0 < hi; b0 += blockDim.x) {   // block-uniform trip count
    const i64 i = b0 + threadIdx.x;
    i32 x = 0, y = 0;
    if (i < hi) item(i, x, y);
    i32 ex = x, ey = y, bx, by;
    fz_block_exscan2(ex, ey, s_warp, bx, by);
    if (i < hi) out(i, cx + ex, cy + ey);
    cx += bx;
    cy += by;
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) tot(cx, cy);
  return true;
}

__global__ void __launch_bounds__(kFusedThreads, 2) k_coarsen_fused(FusedArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ i32 s_flag, s_any, s_count;
  __shared__ u64 s_off;
  const i32 n = a.n;
  const i64 stride = (i64)gridDim.x * blockDim.x;
  const i64 t0 = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;

  // ---- clear and initialise (the per-phase path's memsets) ----
  for (i64 v = t0; v <= n; v += stride) {
    if (v < n) {
      const u64 key = (u64)(u32)v << 32;
      a.k0[v] = key;
      a.k1[v] = key;
      a.gsize[v] = 0;
      a.gcur[v] = 0;
      a.cvwgt[v] = 0;
    }
    a.rowlen[v] = 0;
    a.mcnt[v] = 0;
    a.cnt[v] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.chg[0] = 0;
    a.chg[1] = 0;
    a.chg[2] = 0;
    a.arena->used = 0;
    a.arena->need = 0;
    a.arena->overflow = 0;
    *a.maxdeg_out = 0;
    *a.max_cvw_out = 0;
  }
  // ---- heavy-edge candidates (coarsen.hpp:39-78) ----
  switch (a.lanes) {
    case 2: fz_match<2>(a); break;
    case 4: fz_match<4>(a); break;
    case 8: fz_match<8>(a); break;
    case 16: fz_match<16>(a); break;
    default: fz_match<32>(a); break;
  }
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  if (a.split) {
    fz_match_long(a);
    if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  }

  // ---- union-find rounds (coarsen.hpp:80-118, 461-469), as k_uf_persist ----
  {
    i32 rounds = -1;
    for (i32 it = 1;; ++it) {
      if (it > a.max_rounds) {   // uniform across CTAs
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(a.err, 2);
        return;
      }
      const u64* src = (it & 1) ? a.k0 : a.k1;   // round it reads buffer (it-1)&1, raises it&1
      u64* dst = (it & 1) ? a.k1 : a.k0;
      if (threadIdx.x == 0) s_any = 0;
      __syncthreads();
      bool diff = false;
      for (i64 v = t0; v < n; v += stride) {
        const i32 c = ldcg(a.cand + v);
        const u64 kv = ldcg(src + v);
        const u64 kc = ldcg(src + c);
        const u32 x = (u32)(kv >> 32), y = (u32)(kc >> 32);
        atomicMax((unsigned long long*)&dst[v], (unsigned long long)kv);
        if (x > y) {
          atomicMax((unsigned long long*)&dst[c], (unsigned long long)(((u64)x << 32) | (u32)it));
          diff = true;
        } else if (x < y) {
          atomicMax((unsigned long long*)&dst[v], (unsigned long long)(((u64)y << 32) | (u32)it));
          diff = true;
        }
      }
      if (diff) s_any = 1;
      __syncthreads();
      if (threadIdx.x == 0 && s_any) atomicOr(&a.chg[it % 3], 1);
      if (blockIdx.x == 0 && threadIdx.x == 0) a.chg[(it + 1) % 3] = 0;
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
      if (ldcg(&a.chg[it % 3]) == 0) {
        rounds = it;
        break;
      }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.uf_rounds_out = rounds;
  }
  const u64* keys = a.k0;   // both buffers hold the fixed point

  // ---- group sizes (coarsen.hpp:351-359) ----
  for (i64 v = t0; v < n; v += stride) atomicAdd(&a.gsize[(u32)(ldcg(keys + v) >> 32)], 1);
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  // ---- coarse ids: ceil(size/cap) per root, scanned; member offsets of big groups ----
  {
    const i32 cap = a.cap;
    auto item = [&](i64 i, i32& x, i32& y) {
      const i32 s = ldcg(a.gsize + i);
      x = (s + cap - 1) / cap;
      y = s > cap ? s : 0;
    };
    auto out = [&](i64 i, i32 ex, i32 ey) {
      a.cbase[i] = ex;
      a.goff[i] = ey;
    };
    auto tot = [&](i32 tx, i32 ty) {
      *a.nc_out = tx;
      a.misc[kFzBig] = ty;
    };
    if (!fz_grid_scan2(a, n, item, out, tot, &s_flag)) return;
  }
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  // ---- scatter: cmap of small groups, member lists of big ones (coarsen.hpp:361-421) ----
  for (i64 v = t0; v < n; v += stride) {
    const i32 r = (i32)(u32)(ldcg(keys + v) >> 32);
    const i32 s = ldcg(a.gsize + r);
    if (s <= a.cap) {
      a.cmap[v] = ldcg(a.cbase + r);
    } else {
      const i32 slot = atomicAdd(&a.gcur[r], 1);
      a.members[ldcg(a.goff + r) + slot] = (i32)v;
      if (r == (i32)v) {
        if (s <= 32) a.wlist[atomicAdd(a.misc + kFzWarpG, 1)] = r;
        else if (s <= kGroupSmem) a.clist[atomicAdd(a.misc + kFzCtaG, 1)] = r;
        else a.glist[atomicAdd(a.misc + kFzGiant, 1)] = r;
      }
    }
  }
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  // ---- big groups ordered by (dist, id): warps, CTAs, and rare giant groups ----
  {
    const i32 nwg = ldcg(a.misc + kFzWarpG);
    const i64 warp0 = t0 >> 5, nwarps = stride >> 5;
    for (i64 w = warp0; w < nwg; w += nwarps) {
      const i32 r = ldcg(a.wlist + w);
      const i32 s = ldcg(a.gsize + r);
      u64 key = ~0ull;
      if (lane < s) {
        const i32 mb = ldcg(a.members + ldcg(a.goff + r) + lane);
        key = ((ldcg(keys + mb) & 0xffffffffull) << 32) | (u32)mb;   // (dist, id)
      }
#pragma unroll
      for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
        for (int j = kk >> 1; j > 0; j >>= 1) {
          const u64 o = __shfl_xor_sync(kFull, key, j);
          const bool up = (lane & kk) == 0;
          const bool lower = (lane & j) == 0;
          key = (lower == up) ? umin64(key, o) : umax64(key, o);
        }
      }
      if (lane < s) a.cmap[(u32)key] = ldcg(a.cbase + r) + lane / a.cap;
    }
    const i32 ncg = ldcg(a.misc + kFzCtaG);
    u64* sk = reinterpret_cast<u64*>(smem_raw);
    for (i32 b = blockIdx.x; b < ncg; b += gridDim.x) {
      const i32 r = ldcg(a.clist + b);
      const i32 s = ldcg(a.gsize + r);
      i32 P = 64;
      while (P < s) P <<= 1;
      for (i32 i = threadIdx.x; i < P; i += blockDim.x) {
        u64 key = ~0ull;
        if (i < s) {
          const i32 mb = ldcg(a.members + ldcg(a.goff + r) + i);
          key = ((ldcg(keys + mb) & 0xffffffffull) << 32) | (u32)mb;
        }
        sk[i] = key;
      }
      __syncthreads();
      cta_bitonic_u64(sk, P);
      const i32 cb = ldcg(a.cbase + r);
      for (i32 i = threadIdx.x; i < s; i += blockDim.x) a.cmap[(u32)sk[i]] = cb + i / a.cap;
      __syncthreads();
    }
    const i32 ng = ldcg(a.misc + kFzGiant);   // the same on every CTA
    for (i32 gi = 0; gi < ng; ++gi) {
      const i32 r = ldcg(a.glist + gi);
      const i32 s = ldcg(a.gsize + r);
      i64 P = 1;
      while (P < s) P <<= 1;
      const i32 mo = ldcg(a.goff + r);
      u64* g = a.gscratch;
      for (i64 i = t0; i < P; i += stride) {
        u64 key = ~0ull;
        if (i < s) {
          const i32 mb = ldcg(a.members + mo + i);
          key = ((ldcg(keys + mb) & 0xffffffffull) << 32) | (u32)mb;
        }
        g[i] = key;
      }
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
      for (i64 kk = 2; kk <= P; kk <<= 1) {
        for (i64 j = kk >> 1; j > 0; j >>= 1) {
          for (i64 i = t0; i < P; i += stride) {
            const i64 l = i ^ j;
            if (l > i) {
              const u64 x = ldcg(g + i), y = ldcg(g + l);
              const bool up = (i & kk) == 0;
              if (up ? (x > y) : (x < y)) { g[i] = y; g[l] = x; }
            }
          }
          if (!grid_barrier(a.bar, a.err, &s_flag)) return;
        }
      }
      const i32 cb = ldcg(a.cbase + r);
      for (i64 i = t0; i < s; i += stride) a.cmap[(u32)ldcg(g + i)] = cb + (i32)(i / a.cap);
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
    }
  }
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;

  // ---- contraction (coarsen.hpp:157-349) ----
  const i32 cap = a.cap;
  for (i64 v = t0; v < n; v += stride) {   // coarse weights, row lengths, member lists
    const i32 c = ldcg(a.cmap + v);
    atomicAdd((u32*)&a.cvwgt[c], (u32)a.vwgt[v]);
    atomicAdd(&a.rowlen[c], a.xadj[v + 1] - a.xadj[v]);
    const i32 slot = atomicAdd(&a.mcnt[c], 1);
    a.memtab[(i64)c * cap + slot] = (i32)v;
  }
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  {   // upper-bound row offsets: exclusive scan of the row lengths (n + 1 entries)
    auto item = [&](i64 i, i32& x, i32& y) {
      x = ldcg(a.rowlen + i);
      y = 0;
    };
    auto out = [&](i64 i, i32 ex, i32) { a.ub[i] = ex; };
    auto tot = [&](i32 tx, i32) { a.misc[kFzUb] = tx; };
    if (!fz_grid_scan2(a, (i64)n + 1, item, out, tot, &s_flag)) return;
  }
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  const i32 nc = ldcg(a.nc_out);
  {   // one warp per coarse vertex, as k_contract_warp<128, 8>
    WarpTable<kFusedWcap>& T = reinterpret_cast<WarpTable<kFusedWcap>*>(smem_raw)[wid];
    const i64 nw = (i64)gridDim.x * kFusedWarps;
    for (i64 c = (i64)blockIdx.x * kFusedWarps + wid; c < nc; c += nw) {
      const i32 L = ldcg(a.rowlen + c);
      const i32 nm = ldcg(a.mcnt + c);
      if (L > kFusedWcap || nm > 32) {
        if (lane == 0) a.heavy[atomicAdd(a.misc + kFzHeavy, 1)] = (i32)c;
        continue;
      }
      i32 mbeg = 0, mlen = 0;
      if (lane < nm) {
        const i32 v = ldcg(a.memtab + c * (i64)cap + lane);
        mbeg = a.xadj[v];
        mlen = a.xadj[v + 1] - mbeg;
      }
      i32 moff = mlen;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const i32 y = __shfl_up_sync(kFull, moff, o);
        if (lane >= o) moff += y;
      }
      moff -= mlen;
      auto entry_pos = [&](i32 i) {
        i32 pos = -1;
        for (i32 jm = 0; jm < nm; ++jm) {
          const i32 oj = __shfl_sync(kFull, moff, jm);
          const i32 lj = __shfl_sync(kFull, mlen, jm);
          const i32 bj = __shfl_sync(kFull, mbeg, jm);
          if (i >= oj && i < oj + lj) pos = bj + (i - oj);
        }
        return pos;
      };
      const i32 o = ldcg(a.ub + c);
      if (L <= 32) {
        u64 kv = ~0ull;
        const i32 pos = entry_pos(lane);
        if (lane < L) {
          const u32 key = (u32)ldcg(a.cmap + a.adjncy[pos]);
          if (key != (u32)c) kv = ((u64)key << 32) | (u32)a.adjwgt[pos];
        }
#pragma unroll
        for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
          for (int jj = kk >> 1; jj > 0; jj >>= 1) {
            const u64 ot = __shfl_xor_sync(kFull, kv, jj);
            const bool up = (lane & kk) == 0;
            const bool lower = (lane & jj) == 0;
            kv = (lower == up) ? umin64(kv, ot) : umax64(kv, ot);
          }
        }
        const u32 key = (u32)(kv >> 32);
        const u32 w = (u32)kv;
        const u32 kprev = __shfl_up_sync(kFull, key, 1);
        const u32 knext = __shfl_down_sync(kFull, key, 1);
        const bool head = lane == 0 || kprev != key;
        const bool last = lane == 31 || knext != key;
        u32 S = w;
        i32 start = head ? lane : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const u32 y = __shfl_up_sync(kFull, S, d);
          const i32 z = __shfl_up_sync(kFull, start, d);
          if (lane >= d) {
            S += y;
            start = start > z ? start : z;
          }
        }
        const u32 before = __shfl_sync(kFull, S, start > 0 ? start - 1 : 0);
        const u32 total = S - (start > 0 ? before : 0u);
        const bool valid = last && key != 0xffffffffu;
        const u32 bal = __ballot_sync(kFull, valid);
        if (valid) {
          const i32 at = o + __popc(bal & ((1u << lane) - 1));
          a.sadj[at] = (i32)key;
          a.swgt[at] = (i32)total;
        }
        if (lane == 0) a.cnt[c] = __popc(bal);
        continue;
      }
      u32 hsz = 64;
      while (hsz < 2u * (u32)L) hsz <<= 1;
      for (u32 i = lane; i < hsz; i += 32) { T.keys[i] = kEmpty; T.vals[i] = 0; }
      __syncwarp();
      for (i32 b = 0; b < L; b += 32) {
        const i32 i = b + lane;
        const i32 pos = entry_pos(i);
        if (i < L) {
          const u32 key = (u32)ldcg(a.cmap + a.adjncy[pos]);
          if (key != (u32)c) table_add(T.keys, T.vals, hsz, key, (u32)a.adjwgt[pos]);
        }
      }
      __syncwarp();
      i32 U = 0;
      for (u32 base = 0; base < hsz; base += 32) {
        const u32 sl = base + lane;
        const bool occ = T.keys[sl] != kEmpty;
        const u32 bal = __ballot_sync(kFull, occ);
        if (occ) {
          const i32 at = U + __popc(bal & ((1u << lane) - 1));
          T.out[at] = ((u64)T.keys[sl] << 32) | T.vals[sl];
        }
        U += __popc(bal);
      }
      __syncwarp();
      if (U <= 32) {
        u64 key = lane < U ? T.out[lane] : ~0ull;
#pragma unroll
        for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
          for (int jj = kk >> 1; jj > 0; jj >>= 1) {
            const u64 ot = __shfl_xor_sync(kFull, key, jj);
            const bool up = (lane & kk) == 0;
            const bool lower = (lane & jj) == 0;
            key = (lower == up) ? umin64(key, ot) : umax64(key, ot);
          }
        }
        if (lane < U) {
          a.sadj[o + lane] = (i32)(u32)(key >> 32);
          a.swgt[o + lane] = (i32)(u32)key;
        }
      } else {
        i32 P = 64;
        while (P < U) P <<= 1;
        for (i32 i = U + lane; i < P; i += 32) T.out[i] = ~0ull;
        __syncwarp();
        warp_bitonic_u64(T.out, P, lane);
        for (i32 i = lane; i < U; i += 32) {
          const u64 kv = T.out[i];
          a.sadj[o + i] = (i32)(u32)(kv >> 32);
          a.swgt[o + i] = (i32)(u32)kv;
        }
      }
      if (lane == 0) a.cnt[c] = U;
      __syncwarp();
    }
  }
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  {   // heavy coarse rows, one CTA each: the shared table, or the arena beyond kFusedCtaCap
    const i32 nh = ldcg(a.misc + kFzHeavy);
    for (i32 b = blockIdx.x; b < nh; b += gridDim.x) {
      const i32 c = ldcg(a.heavy + b);
      const i32 L = ldcg(a.rowlen + c);
      const bool global_table = L > kFusedCtaCap;
      u32 hsz = 64;
      while (hsz < 2u * (u32)L) hsz <<= 1;
      u32 *tk, *tv;
      u64* out;
      if (global_table) {
        const u64 words = 3ull * hsz;   // keys + vals + hsz/2 u64 outputs
        if (threadIdx.x == 0) {
          const u64 off = atomicAdd((unsigned long long*)&a.arena->used, (unsigned long long)words);
          if (off + words > a.arena_cap) {
            atomicAdd((unsigned long long*)&a.arena->need, (unsigned long long)words);
            atomicExch(&a.arena->overflow, 1);
            s_off = ~0ull;
          } else {
            s_off = off;
          }
        }
        __syncthreads();
        const u64 off = s_off;
        __syncthreads();   // every thread has read s_off before thread 0 can set it for the next row
        if (off == ~0ull) continue;   // block-uniform; the level is redone after the arena grows
        tk = a.arena_words + off;
        tv = tk + hsz;
        out = reinterpret_cast<u64*>(tv + hsz);
      } else {
        tk = reinterpret_cast<u32*>(smem_raw);
        tv = tk + 2 * kFusedCtaCap;
        out = reinterpret_cast<u64*>(tv + 2 * kFusedCtaCap);
      }
      for (u32 i = threadIdx.x; i < hsz; i += blockDim.x) { tk[i] = kEmpty; tv[i] = 0; }
      if (threadIdx.x == 0) s_count = 0;
      __syncthreads();
      const i32 nm = ldcg(a.mcnt + c);
      for (i32 j = 0; j < nm; ++j) {
        const i32 v = ldcg(a.memtab + c * (i64)cap + j);
        const i32 beg = a.xadj[v], end = a.xadj[v + 1];
        for (i32 e = beg + threadIdx.x; e < end; e += blockDim.x) {
          const u32 key = (u32)ldcg(a.cmap + a.adjncy[e]);
          if (key != (u32)c) table_add(tk, tv, hsz, key, (u32)a.adjwgt[e]);
        }
      }
      __syncthreads();
      for (u32 sl = threadIdx.x; sl < hsz; sl += blockDim.x) {
        if (tk[sl] != kEmpty) {
          const i32 pos = atomicAdd(&s_count, 1);
          out[pos] = ((u64)tk[sl] << 32) | tv[sl];
        }
      }
      __syncthreads();
      const i32 U = s_count;
      i32 P = 64;
      while (P < U) P <<= 1;
      for (i32 i = U + threadIdx.x; i < P; i += blockDim.x) out[i] = ~0ull;
      __syncthreads();
      cta_bitonic_u64(out, P);
      const i32 o = ldcg(a.ub + c);
      for (i32 i = threadIdx.x; i < U; i += blockDim.x) {
        const u64 kv = out[i];
        a.sadj[o + i] = (i32)(u32)(kv >> 32);
        a.swgt[o + i] = (i32)(u32)kv;
      }
      if (threadIdx.x == 0) a.cnt[c] = U;
      __syncthreads();
    }
  }
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  {   // coarse xadj: exclusive scan of the row counts (rows beyond n_c are empty)
    auto item = [&](i64 i, i32& x, i32& y) {
      x = ldcg(a.cnt + i);
      y = 0;
    };
    auto out = [&](i64 i, i32 ex, i32) { a.cxadj[i] = ex; };
    auto tot = [&](i32 tx, i32) { *a.mc_out = tx; };
    if (!fz_grid_scan2(a, (i64)n + 1, item, out, tot, &s_flag)) return;
  }
  if (!grid_barrier(a.bar, a.err, &s_flag)) return;
  {   // compact the rows (one warp per 32 rows, as k_copy_rows); longest row, heaviest vertex
    const i64 warp = t0 >> 5, nwarps = stride >> 5;
    i32 mx = 0, mw = 0;
    for (i64 c0 = warp * 32; c0 < nc; c0 += nwarps * 32) {
      const i64 c = c0 + lane;
      i32 src = 0, dst = 0, len = 0;
      if (c < nc) {
        src = ldcg(a.ub + c);
        dst = ldcg(a.cxadj + c);
        len = ldcg(a.cnt + c);
        const i32 w = ldcg(a.cvwgt + c);
        mw = w > mw ? w : mw;
      }
      mx = len > mx ? len : mx;
      i32 inc = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const i32 y = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += y;
      }
      const i32 total = __shfl_sync(kFull, inc, 31);
      const i32 exc = inc - len;
      for (i32 base = 0; base < total; base += 32) {
        const i32 idx = base + lane;
        i32 r = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const i32 probe = __shfl_sync(kFull, inc, r + step - 1);
          if (probe <= idx) r += step;
        }
        r = r < 31 ? r : 31;
        const i32 rs = __shfl_sync(kFull, src, r), rd = __shfl_sync(kFull, dst, r), re = __shfl_sync(kFull, exc, r);
        if (idx < total) {
          a.cadjncy[rd + (idx - re)] = ldcg(a.sadj + rs + (idx - re));
          a.cadjwgt[rd + (idx - re)] = ldcg(a.swgt + rs + (idx - re));
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const i32 y = __shfl_xor_sync(kFull, mx, o);
      mx = mx > y ? mx : y;
      const i32 z = __shfl_xor_sync(kFull, mw, o);
      mw = mw > z ? mw : z;
    }
    if (lane == 0 && mx > 0) atomicMax(a.maxdeg_out, mx);
    if (lane == 0 && mw > 0) atomicMax(a.max_cvw_out, mw);
  }
}

static int fused_blocks_per_sm() {
  static int bps = -1;   // the same on every device of the process (one B200 model)
  if (bps < 0) {
    int b = 0;
    if (cudaFuncSetAttribute(k_coarsen_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFusedSmem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_coarsen_fused, kFusedThreads, kFusedSmem) !=
            cudaSuccess) {
      cudaGetLastError();
      b = 0;
    }
    bps = b;
  }
  return bps;
}

// Whether a level runs as one fused launch: levels of at most the handle's
// fused_max_n vertices whose rows are short on average (long coarse rows are
// the per-phase path's wide warp tables), never while the tuner times the
// match variants.
static bool use_fused(Handle& h, const DevGraph& g) {
  return !h.tune_collect && g.n > 0 && (i64)g.n <= (i64)h.tuning.coarsen_fused_max_n &&
         (double)g.m <= 48.0 * (double)g.n && fused_blocks_per_sm() >= 1;
}

static void run_coarsen_fused(Handle& h, const DevGraph& g, i32 cap, CoarsenOut& out) {
  if (!h.capturing)   // per device (the occupancy probe set it on the first device only)
    GKW_CUDA(cudaFuncSetAttribute(k_coarsen_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFusedSmem));
  Pool::Mark mk = h.scratch.mark();
  const i32 n = g.n;
  const i64 nu = (i64)n + 1;
  const i32 bps = fused_blocks_per_sm();
  const i32 vpc = std::max(64, h.tuning.coarsen_verts_per_cta);
  i32 grid = (i32)std::min<i64>((i64)h.sm_count * bps, std::max<i64>(1, ((i64)n + vpc - 1) / vpc));
  grid = coop_grid(h, (const void*)k_coarsen_fused, grid, kFusedThreads, kFusedSmem);
  FusedArgs a;
  a.n = n;
  a.m = g.m;
  a.xadj = g.xadj;
  a.adjncy = g.adjncy;
  a.adjwgt = g.adjwgt;
  a.vwgt = g.vwgt;
  a.lanes = h.tuning.match_lanes[match_bucket(g)];
  a.split = g.maxdeg < 0 || g.maxdeg > kMatchLong;
  a.cap = cap;
  a.max_rounds = n + 2;
  a.cmap = out.cmap;
  a.cxadj = out.cxadj;
  a.cadjncy = out.cadjncy;
  a.cadjwgt = out.cadjwgt;
  a.cvwgt = out.cvwgt;
  a.cand = h.scratch.alloc_n<i32>(n);
  a.k0 = h.scratch.alloc_n<u64>(n);
  a.k1 = h.scratch.alloc_n<u64>(n);
  a.chg = h.scratch.alloc_n<i32>(4);
  a.longlist = h.scratch.alloc_n<i32>(n);
  a.gsize = h.scratch.alloc_n<i32>(n);
  a.cbase = h.scratch.alloc_n<i32>(n);
  a.goff = h.scratch.alloc_n<i32>(n);
  a.gcur = h.scratch.alloc_n<i32>(n);
  a.members = h.scratch.alloc_n<i32>(n);
  a.wlist = h.scratch.alloc_n<i32>(n);
  a.clist = h.scratch.alloc_n<i32>(n);
  a.glist = h.scratch.alloc_n<i32>(n);
  a.gscratch = h.scratch.alloc_n<u64>(2 * (size_t)n);
  a.rowlen = h.scratch.alloc_n<i32>(nu);
  a.ub = h.scratch.alloc_n<i32>(nu);
  a.mcnt = h.scratch.alloc_n<i32>(nu);
  a.memtab = h.scratch.alloc_n<i32>((i64)n * cap + 1);
  a.cnt = h.scratch.alloc_n<i32>(nu);
  a.heavy = h.scratch.alloc_n<i32>(nu);
  a.sadj = h.scratch.alloc_n<i32>(std::max<i64>(g.m, 1));
  a.swgt = h.scratch.alloc_n<i32>(std::max<i64>(g.m, 1));
  a.partial = h.scratch.alloc_n<i32>(2 * (size_t)grid);
  a.misc = h.scratch.alloc_n<i32>(kFzWords);
  a.bar = &h.coop->bar;
  a.err = &h.coop->err;
  a.nc_out = &h.coop->nc;
  a.mc_out = &h.coop->mc;
  a.uf_rounds_out = &h.coop->uf_rounds;
  a.maxdeg_out = &h.coop->maxdeg;
  a.max_cvw_out = &h.coop->max_cvw;
  a.arena = h.arena;
  a.arena_words = reinterpret_cast<u32*>(h.arena + 1);
  a.arena_cap = h.arena_words;
  GKW_CUDA(cudaMemsetAsync(a.misc, 0, sizeof(i32) * kFzWords, h.stream));
  void* args[] = {&a};
  launch_coop(h, (const void*)k_coarsen_fused, grid, kFusedThreads, kFusedSmem, args);
  h.scratch.release(mk);
}

// The key of one level's launch sequence in the handle's graph cache:
// everything the launches depend on.
static std::string level_key(const Handle& h, const DevGraph& g, i32 cap, const CoarsenOut& out) {
  struct K {
    i64 n, m, maxdeg, cap;
    const void* in[4];
    const void* outp[5];
    const void* sbase;
    size_t stop;
    gkw_tuning tuning;
    i32 narrow, sms;
    const void* arena;
    u64 arena_words;
    const void* scan;
  } k;
  memset(&k, 0, sizeof(k));
  k.n = g.n;
  k.m = g.m;
  k.maxdeg = g.maxdeg;
  k.cap = cap;
  k.in[0] = g.xadj;
  k.in[1] = g.adjncy;
  k.in[2] = g.adjwgt;
  k.in[3] = g.vwgt;
  k.outp[0] = out.cmap;
  k.outp[1] = out.cxadj;
  k.outp[2] = out.cvwgt;
  k.outp[3] = out.cadjncy;
  k.outp[4] = out.cadjwgt;
  const auto fp = h.scratch.fingerprint();
  k.sbase = fp.first;
  k.stop = fp.second;
  k.tuning = h.tuning;
  k.narrow = h.narrow;
  k.sms = h.sm_count;
  k.arena = h.arena;
  k.arena_words = h.arena_words;
  k.scan = h.scan;
  return std::string("level", 5) + std::string(reinterpret_cast<const char*>(&k), sizeof(k));
}

// One coarsening step.  Its launch sequence (about twenty kernels and ten
// memsets, all sized by the level's n and m) runs through the handle's graph
// cache: repeated partitions of the same graph replay it as one CUDA graph.
// One host sync per level reads the coarse sizes.
void coarsen_level(Handle& h, const DevGraph& g, i32 cap, CoarsenOut& out) {
  // coarse arrays at upper bounds (n_c <= n, m_c <= m)
  out.cmap = h.hier.alloc_n<i32>(std::max(g.n, 1));
  out.cxadj = h.hier.alloc_n<i32>((i64)g.n + 1);
  out.cvwgt = h.hier.alloc_n<i32>(std::max(g.n, 1));
  out.cadjncy = h.hier.alloc_n<i32>(std::max<i64>(g.m, 1));
  out.cadjwgt = h.hier.alloc_n<i32>(std::max<i64>(g.m, 1));
  ensure_arena(h, u64(4) << 20);   // never inside a capture
  const bool tune = h.tune_collect;
  auto body = [&] {
    Pool::Mark mk = h.scratch.mark();
    i32* cand = h.scratch.alloc_n<i32>(std::max(g.n, 1));
    u64* keys = h.scratch.alloc_n<u64>(std::max(g.n, 1));
    if (tune) time_match_variants(h, g, cand);
    run_match(h, g, cand, g.maxdeg);
    run_union_find(h, g.n, cand, keys, &h.coop->uf_rounds);
    run_group_map(h, g.n, keys, cap, out.cmap, &h.coop->nc);
    h.scratch.release(mk);
    static_assert(offsetof(CoopState, maxdeg) == offsetof(CoopState, max_cvw) + sizeof(i32),
                  "max_cvw and maxdeg are cleared together");
    GKW_CUDA(cudaMemsetAsync(&h.coop->max_cvw, 0, 2 * sizeof(i32), h.stream));
    run_contract(h, g, out.cmap, &h.coop->nc, g.n, cap, out.cxadj, out.cadjncy, out.cadjwgt, out.cvwgt,
                 &h.coop->mc);
  };
  if (use_fused(h, g)) {
    // one launch: no graph needed (a launch is as cheap as a graph of one)
    run_coarsen_fused(h, g, cap, out);
  } else if (tune) {
    body();   // the tuner's timings synchronise: never captured
  } else {
    graph_run(h, level_key(h, g, cap, out), body);
  }
  CoopState c = read_coop(h);
  if (c.arena_overflow) {   // very long coarse rows: grow the arena and redo the step
    ensure_arena(h, (u64)((double)(h.arena_words + (u64)c.arena_need) * 1.25) + 1024);
    GKW_CUDA(cudaMemsetAsync(&h.coop->maxdeg, 0, sizeof(i32), h.stream));
    run_contract(h, g, out.cmap, &h.coop->nc, g.n, cap, out.cxadj, out.cadjncy, out.cadjwgt, out.cvwgt,
                 &h.coop->mc);
    c = read_coop(h);
    GKW_REQUIRE(!c.arena_overflow, GKW_E_INTERNAL, "long-row arena overflow after growth");
  }
  out.nc = c.nc;
  out.mc = c.mc;
  out.uf_rounds = c.uf_rounds;
  out.max_cvw = c.max_cvw;
  out.maxdeg = c.maxdeg;
}

}  // namespace gkw
