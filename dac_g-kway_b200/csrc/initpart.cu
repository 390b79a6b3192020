// Device initial partition of the coarsest graph: recursive bisection by
// greedy graph growing (GGGP, Karypis & Kumar's multilevel partitioning
// scheme), replacing the reference's host METIS call
// (gkway/metis_partition.hpp:46-47).
//
// Each recursion depth is one launch.  A sub-problem is the set of vertices
// whose part range is [p0, p1); it is bisected into [p0, pm) and [pm, p1),
// pm = p0 + (p1 - p0) / 2, with the left side's target weight
// TL = W(S) * (pm - p0) / (p1 - p0).  One CTA handles one sub-problem; each
// warp runs one trial from its own seed vertex:
//   growth      repeatedly add the unassigned vertex with the best key
//               (frontier first, then cut gain 2*conn - deg_S, then the
//               smaller member index) while the region weight is below TL;
//               a vertex that would overshoot TL by more than the region is
//               short of it is not added and growth stops;
//   refinement  move the vertex with the largest positive cut gain to the
//               other side while the receiving side stays within
//               target * (1 + eps/2); at most s/4 + 32 moves.
// The trial with the smallest cut (then smallest |W(R) - TL|, then lowest
// trial index) wins.  Seeds: trial t of sub-problem p0 starts at member
// index mix(seed, p0, t) mod s.  Deterministic for a given seed.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gkw_internal.cuh"

namespace gkw {

static constexpr u32 kFull32 = 0xffffffffu;
constexpr int kInitTrials = 8;

__device__ __forceinline__ u32 mix32(u64 x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return (u32)x;
}

__global__ void k_init_count(i32 n, const i32* __restrict__ lo, i32* __restrict__ cnt) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) atomicAdd(&cnt[lo[v]], 1);
}

// Warp maximum of a 64-bit key in two 32-bit reductions (redux.sync): the
// largest high half, then the largest low half among the lanes holding it --
// two dependent steps instead of five shuffle rounds on a growth step's chain.
__device__ __forceinline__ u64 warp_max_u64(u64 x) {
  const u32 hi = (u32)(x >> 32), lo = (u32)x;
  const u32 mh = __reduce_max_sync(kFull32, hi);
  const u32 ml = __reduce_max_sync(kFull32, hi == mh ? lo : 0u);
  return ((u64)mh << 32) | ml;
}

__device__ __forceinline__ i64 warp_sum_i64(i64 x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull32, x, o);
  return x;
}

// growth key: frontier bit, gain (order-preserving bias), smaller index wins
__device__ __forceinline__ u64 grow_key(bool frontier, i32 g, i32 idx) {
  return (1ull << 63) | ((u64)(frontier ? 1 : 0) << 62) | ((u64)((u32)g ^ 0x80000000u) << 30) |
         (u64)(0x3fffffffu - (u32)idx);
}

// refinement key: gain, smaller index wins; top bit marks a valid entry
__device__ __forceinline__ u64 move_key2(i32 g, i32 idx) {
  return (1ull << 63) | ((u64)((u32)g ^ 0x80000000u) << 30) | (u64)(0x3fffffffu - (u32)idx);
}

__device__ __forceinline__ i32 key_idx(u64 key) { return (i32)(0x3fffffffu - (u32)(key & 0x3fffffffu)); }

typedef uint8_t u8;

// A large sub-problem handed from the depth kernel to the per-trial kernel.
struct BigParams {
  i64 TL, WS, capL, capR;
  i32 pm, p1;
};

// Topology of one sub-problem in local (member) indices: row i holds the
// member's neighbours inside the sub-problem.
struct LocalTopo {
  const i32* rb;     // row start in nb/nw
  const i32* rn;     // neighbours inside the sub-problem
  const i32* nb;     // local neighbour index
  const i32* nw;     // edge weight
  const i32* degS;   // weight to other members
  const i32* vw;     // vertex weight
};

// Growth keys of one trial: K[i] = grow_key of unassigned member i (0 once
// assigned), B1[b] = max of K over members [32b, 32b + 32), B2[c] = max of B1
// over blocks [32c, 32c + 32).  A key only rises while its member is
// unassigned (conn only grows), so updates are atomic maxima; assigning a
// member recomputes its two blocks.  The argmax over all unassigned members
// is then a scan of B2.
struct TrialState {
  i32* C;      // connection weight to the region R
  i32* R;      // in R
  u64* K;
  u64* B1;
  u64* B2;
};

__host__ __device__ __forceinline__ i32 gggp_nb1(i32 s) { return (s + 31) >> 5; }
__host__ __device__ __forceinline__ i32 gggp_nb2(i32 s) { return (s + 1023) >> 10; }
// i32 words of one trial's state in shared memory (C, R, K, B1, B2; even, so
// every trial's u64 arrays stay 8-byte aligned)
__host__ __device__ __forceinline__ i32 gggp_state_words(i32 s) {
  return 2 * s + 2 * s + 2 * gggp_nb1(s) + 2 * gggp_nb2(s) + ((2 * s) & 1);
}

// Refinement moves of one trial: s/4 + 32, at most 256 (each move scans the
// whole sub-problem).
__host__ __device__ __forceinline__ i32 gggp_max_moves(i32 s) { return s / 4 + 32 < 256 ? s / 4 + 32 : 256; }

// Growth of small sub-problems: F = members outside R with conn > 0; a
// frontier member always outranks a non-frontier one, so the argmax over F
// equals the argmax over all unassigned members, and the full scan is only
// needed when F is empty.  F and posF use the trial's key array.  Returns W(R).
__device__ i64 grow_scan(const LocalTopo& T, const TrialState& S, i32 s, i32 pick, i64 TL) {
  const int lane = threadIdx.x & 31;
  i32* C = S.C;
  i32* R = S.R;
  i32* F = reinterpret_cast<i32*>(S.K);
  i32* posF = F + s;
  i64 wR = 0;
  i32 nF = 0;
  for (i32 step = 0; step < s; ++step) {
    if (step > 0) {
      u64 best = 0;
      if (nF > 0) {
        for (i32 f = lane; f < nF; f += 32) {
          const i32 i = F[f];
          const i32 c = C[i];
          const u64 key = grow_key(true, 2 * c - T.degS[i], i);
          best = best > key ? best : key;
        }
      } else {
        for (i32 i = lane; i < s; i += 32) {
          if (!R[i]) {
            const i32 c = C[i];
            const u64 key = grow_key(c > 0, 2 * c - T.degS[i], i);
            best = best > key ? best : key;
          }
        }
      }
      best = warp_max_u64(best);
      if (best == 0) break;
      pick = key_idx(best);
      const i64 vw = (u32)T.vw[pick];
      if (wR + vw > TL && (wR + vw - TL) > (TL - wR)) break;
    }
    const i32 cp = C[pick];
    if (lane == 0) {
      R[pick] = 1;
      if (cp > 0) {   // leave the frontier (swap-remove)
        const i32 at = posF[pick];
        const i32 last = F[nF - 1];
        F[at] = last;
        posF[last] = at;
      }
    }
    if (cp > 0) --nF;
    wR += (u32)T.vw[pick];
    __syncwarp();
    const i32 rb = T.rb[pick], rn = T.rn[pick];
    for (i32 j0 = 0; j0 < rn; j0 += 32) {
      const i32 j = j0 + lane;
      bool join = false;
      i32 u = 0;
      if (j < rn) {
        u = T.nb[rb + j];
        const i32 w = T.nw[rb + j];
        const i32 old = atomicAdd(&C[u], w);   // a row may list a neighbour twice
        join = !R[u] && old <= 0 && old + w > 0;
      }
      const u32 m = __ballot_sync(kFull32, join);
      if (join) {
        const i32 at = nF + __popc(m & ((1u << lane) - 1));
        F[at] = u;
        posF[u] = at;
      }
      nF += __popc(m);
    }
    __syncwarp();
    if (wR >= TL) break;
  }
  return wR;
}

// Growth of large sub-problems over the block maxima of the growth keys
// (TrialState); the same picks as grow_scan.  Returns W(R).
__device__ i64 grow_blocks(const LocalTopo& T, const TrialState& S, i32 s, i32 pick, i64 TL) {
  const int lane = threadIdx.x & 31;
  i32* C = S.C;
  i32* R = S.R;
  u64* K = S.K;
  u64* B1 = S.B1;
  u64* B2 = S.B2;
  const i32 nb1 = gggp_nb1(s), nb2 = gggp_nb2(s);
  for (i32 i = lane; i < s; i += 32) K[i] = grow_key(false, -T.degS[i], i);
  __syncwarp();
  for (i32 b = lane; b < nb1; b += 32) {
    u64 m = 0;
    for (i32 i = b << 5; i < s && i < (b + 1) << 5; ++i) m = m > K[i] ? m : K[i];
    B1[b] = m;
  }
  __syncwarp();
  for (i32 c = lane; c < nb2; c += 32) {
    u64 m = 0;
    for (i32 b = c << 5; b < nb1 && b < (c + 1) << 5; ++b) m = m > B1[b] ? m : B1[b];
    B2[c] = m;
  }
  __syncwarp();
  i64 wR = 0;
  for (i32 step = 0; step < s; ++step) {
    if (step > 0) {
      u64 best = 0;
      for (i32 c = lane; c < nb2; c += 32) best = best > B2[c] ? best : B2[c];
      best = warp_max_u64(best);
      if (best == 0) break;
      pick = key_idx(best);
    }
    // the picked member's weight and row, loaded together
    const i64 vw = (u32)T.vw[pick];
    const i32 rb = T.rb[pick], rn = T.rn[pick];
    if (step > 0 && wR + vw > TL && (wR + vw - TL) > (TL - wR)) break;
    if (lane == 0) {
      R[pick] = 1;
      K[pick] = 0;
    }
    wR += vw;
    __syncwarp();
    // neighbours, four per lane per pass: the row loads, then the state loads
    // and connection updates of all four are issued together.  R[u] and
    // degS[u] do not change in this step (u != pick).
    constexpr i32 kU = 4;
    for (i32 j0 = lane; j0 < rn; j0 += 32 * kU) {
      i32 u[kU], w[kU], ru[kU], du[kU], c[kU];
#pragma unroll
      for (i32 q = 0; q < kU; ++q) {
        const i32 j = j0 + 32 * q;
        u[q] = j < rn ? T.nb[rb + j] : -1;
        w[q] = j < rn ? T.nw[rb + j] : 0;
      }
#pragma unroll
      for (i32 q = 0; q < kU; ++q) {
        if (u[q] >= 0) {
          ru[q] = R[u[q]];
          du[q] = T.degS[u[q]];
          c[q] = atomicAdd(&C[u[q]], w[q]) + w[q];
        }
      }
#pragma unroll
      for (i32 q = 0; q < kU; ++q) {
        if (u[q] >= 0 && !ru[q]) {
          const unsigned long long key = grow_key(c[q] > 0, 2 * c[q] - du[q], u[q]);
          atomicMax(reinterpret_cast<unsigned long long*>(&K[u[q]]), key);
          atomicMax(reinterpret_cast<unsigned long long*>(&B1[u[q] >> 5]), key);
          atomicMax(reinterpret_cast<unsigned long long*>(&B2[u[q] >> 10]), key);
        }
      }
    }
    __syncwarp();
    // the picked member leaves its blocks
    {
      const i32 b = pick >> 5, i = (b << 5) + lane;
      const u64 m = warp_max_u64(i < s ? K[i] : 0ull);
      if (lane == 0) B1[b] = m;
      __syncwarp();
      const i32 c = pick >> 10, bb = (c << 5) + lane;
      const u64 m2 = warp_max_u64(bb < nb1 ? B1[bb] : 0ull);
      if (lane == 0) B2[c] = m2;
      __syncwarp();
    }
    if (wR >= TL) break;
  }
  return wR;
}

// Sub-problems above this size grow over block maxima; smaller ones scan
// their (small) frontier, which is cheaper per step.
constexpr i32 kGggpBlockMin = 2048;

// One GGGP trial by one warp (growth then positive-gain refinement); see the
// file comment for the rules.  Returns the trial's cut and |W(R) - TL|.
__device__ void gggp_trial(const LocalTopo& T, const TrialState& S, i32 s, i32 pick, i64 TL, i64 WS, i64 capL,
                           i64 capR, i64& cut_out, i64& dev_out, unsigned long long* prof) {
  const int lane = threadIdx.x & 31;
  i32* C = S.C;
  i32* R = S.R;
  for (i32 i = lane; i < s; i += 32) {
    R[i] = 0;
    C[i] = 0;
  }
  __syncwarp();
  const long long c0 = clock64();
  i64 wR = s > kGggpBlockMin ? grow_blocks(T, S, s, pick, TL) : grow_scan(T, S, s, pick, TL);
  const long long c1 = clock64();
  // ---- refinement: positive-gain moves within the side caps ----
  const i32 max_moves = gggp_max_moves(s);
  for (i32 mv = 0; mv < max_moves; ++mv) {
    u64 best = 0;
    // four members per lane per pass, their loads issued together
    constexpr i32 kU = 4;
    for (i32 i0 = lane; i0 < s; i0 += 32 * kU) {
      i32 r[kU], c[kU], d[kU], w[kU];
#pragma unroll
      for (i32 u = 0; u < kU; ++u) {
        const i32 i = i0 + 32 * u;
        const bool in = i < s;
        r[u] = in ? R[i] : 0;
        c[u] = in ? C[i] : 0;
        d[u] = in ? T.degS[i] : 0;
        w[u] = in ? T.vw[i] : 0;
      }
#pragma unroll
      for (i32 u = 0; u < kU; ++u) {
        const i32 g = r[u] ? (d[u] - 2 * c[u]) : (2 * c[u] - d[u]);
        const i64 vw = (u32)w[u];
        const bool ok = r[u] ? ((WS - wR) + vw <= capR) : (wR + vw <= capL);
        if (g > 0 && ok) {   // out-of-range lanes have g = 0
          const u64 key = move_key2(g, i0 + 32 * u);
          best = best > key ? best : key;
        }
      }
    }
    best = warp_max_u64(best);
    if (best == 0) break;
    const i32 i = key_idx(best);
    const i32 r = R[i];
    __syncwarp();
    if (lane == 0) R[i] = r ^ 1;
    wR += r ? -(i64)(u32)T.vw[i] : (i64)(u32)T.vw[i];
    const i32 sign = r ? -1 : 1;
    const i32 rb = T.rb[i], rn = T.rn[i];
    for (i32 j = lane; j < rn; j += 32) atomicAdd(&C[T.nb[rb + j]], sign * T.nw[rb + j]);
    __syncwarp();
  }
  i64 cut = 0;
  for (i32 i = lane; i < s; i += 32)
    if (R[i]) cut += T.degS[i] - C[i];
  cut = warp_sum_i64(cut);
  cut_out = cut;
  dev_out = wR > TL ? wR - TL : TL - wR;
  if (prof && lane == 0) {   // diagnostic timeline: slowest trial's growth and refinement cycles
    const long long c2 = clock64();
    atomicMax(prof, (unsigned long long)(c1 - c0));
    atomicMax(prof + 1, (unsigned long long)(c2 - c1));
  }
}

// Exclusive scan of a[0..s) in shared memory by the whole block (total out).
__device__ i32 block_exscan_smem(i32* a, i32 s, i32* s_warp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  i32 carry = 0;
  for (i32 base = 0; base < s; base += blockDim.x) {
    const i32 i = base + threadIdx.x;
    const i32 x = i < s ? a[i] : 0;
    i32 inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const i32 y = __shfl_up_sync(kFull32, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
      const i32 w = lane < nw ? s_warp[lane] : 0;
      i32 wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const i32 y = __shfl_up_sync(kFull32, wi, o);
        if (lane >= o) wi += y;
      }
      if (lane < nw) s_warp[lane] = wi - w;
      if (lane == nw - 1) s_warp[32] = wi;
    }
    __syncthreads();
    if (i < s) a[i] = carry + inc - x + s_warp[wid];
    carry += s_warp[32];
    __syncthreads();
  }
  return carry;
}

constexpr size_t kGggpSmem = 200 * 1024;   // dynamic shared memory of the depth kernel
constexpr i32 kGggpLongRow = 64;            // rows longer than this are read by a whole warp
constexpr i32 kGggpLongMax = 1024;          // long-row members listed in shared memory

__global__ void __launch_bounds__(kInitTrials * 32) k_gggp_depth(
    i32 n, const i32* __restrict__ xadj, const i32* __restrict__ adjncy, const i32* __restrict__ adjwgt,
    const i32* __restrict__ vwgt, const i32* __restrict__ lo, const i32* __restrict__ hi,
    const i32* __restrict__ cnt, const i32* __restrict__ off, i32* __restrict__ mlist, i32* __restrict__ loc,
    i32* __restrict__ lo_out, i32* __restrict__ hi_out, u64 seed, double eps, i32 trials,
    i32* g_rb, i32* g_rn, i32* g_deg, i32* g_vw, i32* g_nb, i32* g_nw, i32* g_state, u64* g_keys,
    u64* g_b1, u64* g_b2, size_t b1_stride, size_t b2_stride, const i32* __restrict__ part_base, const i32* __restrict__ part_v0,
    const i32* __restrict__ part_v1, unsigned long long* prof, i32* bigcount, i32* biglist, BigParams* bigp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ i32 s_cnt;
  __shared__ i32 s_warp[33];
  __shared__ i64 s_wsum[kInitTrials];
  __shared__ i64 s_cut[kInitTrials];
  __shared__ i64 s_dev[kInitTrials];
  __shared__ i32 s_best;
  const i32 p0 = blockIdx.x;
  const i32 s = cnt[p0];
  if (s == 0) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const i32 base_off = off[p0];
  i32* M = mlist + base_off;
  // deterministic member list: all vertices with lo == p0, in id order
  // (batched levels: only the part's own graph holds them)
  const i32 v_lo = part_v0 ? part_v0[p0] : 0, v_hi = part_v1 ? part_v1[p0] : n;
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  for (i32 base = v_lo; base < v_hi; base += blockDim.x) {
    const i32 v = base + threadIdx.x;
    const bool mine = v < v_hi && lo[v] == p0;
    const u32 bal = __ballot_sync(kFull32, mine);
    if (lane == 0) s_warp[wid] = __popc(bal);
    __syncthreads();
    i32 woff = 0, tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      if (w < wid) woff += s_warp[w];
      tot += s_warp[w];
    }
    if (mine) {
      const i32 idx = s_cnt + woff + __popc(bal & ((1u << lane) - 1));
      M[idx] = v;
      loc[v] = idx;
    }
    __syncthreads();
    if (threadIdx.x == 0) s_cnt += tot;
    __syncthreads();
  }
  const i32 p1 = hi[M[0]];
  if (p1 - p0 < 2) {
    for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
      lo_out[M[i]] = p0;
      hi_out[M[i]] = p1;
    }
    return;
  }
  const i32 pm = p0 + (p1 - p0) / 2;
  // per member: neighbours inside the sub-problem, weight to them, W(S).
  // Rows longer than kGggpLongRow are read by a whole warp (hubs would stall
  // one thread for thousands of dependent loads).  Their members are listed
  // in s_long; when there are more than it holds, the warps find them by
  // scanning all members instead.
  __shared__ i32 s_long[kGggpLongMax];
  __shared__ i32 s_nlong;
  if (threadIdx.x == 0) s_nlong = 0;
  __syncthreads();
  i64 wpart = 0, epart = 0;
  for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
    const i32 v = M[i];
    const i32 b = xadj[v], e1 = xadj[v + 1];
    g_vw[base_off + i] = vwgt[v];
    wpart += (u32)vwgt[v];
    if (e1 - b > kGggpLongRow) {
      const i32 at = atomicAdd(&s_nlong, 1);
      if (at < kGggpLongMax) s_long[at] = i;
      continue;
    }
    i32 d = 0, c = 0;
    for (i32 e = b; e < e1; ++e)
      if (lo[adjncy[e]] == p0) {
        d += adjwgt[e];
        ++c;
      }
    g_rn[base_off + i] = c;
    g_deg[base_off + i] = d;
    epart += c;
  }
  __syncthreads();
  const bool listed = s_nlong <= kGggpLongMax;   // block-uniform
  const i32 nq = listed ? s_nlong : s;
  for (i32 q = wid; q < nq; q += (i32)(blockDim.x >> 5)) {
    const i32 i = listed ? s_long[q] : q;
    const i32 v = M[i];
    const i32 b = xadj[v], e1 = xadj[v + 1];
    if (e1 - b <= kGggpLongRow) continue;   // warp-uniform (scan mode only)
    i64 d = 0;
    i32 c = 0;
    for (i32 e = b + lane; e < e1; e += 32)
      if (lo[adjncy[e]] == p0) {
        d += adjwgt[e];
        ++c;
      }
    d = warp_sum_i64(d);
    c = (i32)warp_sum_i64(c);
    if (lane == 0) {
      g_rn[base_off + i] = c;
      g_deg[base_off + i] = (i32)d;
      epart += c;
    }
  }
  wpart = warp_sum_i64(wpart);
  epart = warp_sum_i64(epart);
  if (lane == 0) {
    s_wsum[wid] = wpart;
    s_cut[wid] = epart;
  }
  __syncthreads();
  i64 WS = 0, ES = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    WS += s_wsum[w];
    ES += s_cut[w];
  }
  __syncthreads();
  const i64 TL = WS * (pm - p0) / (p1 - p0);
  const i64 capL = (i64)((double)TL * (1.0 + eps * 0.5));
  const i64 capR = (i64)((double)(WS - TL) * (1.0 + eps * 0.5));
  // Sub-problems above kGggpBlockMin members (when the caller passes the
  // big-list): the local CSR goes to the global arrays and the trials run in
  // k_gggp_big_trial, one CTA each.
  const bool big = bigcount != nullptr && s > kGggpBlockMin;   // block-uniform
  // shared memory when the local CSR and the trials' state fit
  const i32 stw = gggp_state_words(s);
  const size_t need = sizeof(i32) * ((size_t)4 * s + 2 * (size_t)ES + (size_t)stw * trials);
  const bool in_smem = !big && need <= kGggpSmem;   // block-uniform
  LocalTopo T;
  i32 *rb, *rn, *deg, *vw, *nb, *nw, *state;
  if (in_smem) {
    i32* p = reinterpret_cast<i32*>(smem_raw);
    rb = p; p += s;
    rn = p; p += s;
    deg = p; p += s;
    vw = p; p += s;
    nb = p; p += ES;
    nw = p; p += ES;
    state = p;
    for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
      rn[i] = g_rn[base_off + i];
      rb[i] = rn[i];
      deg[i] = g_deg[base_off + i];
      vw[i] = g_vw[base_off + i];
    }
    __syncthreads();
    block_exscan_smem(rb, s, s_warp);
  } else {
    // rows in the global arrays at the members' own CSR positions
    rb = g_rb + base_off;
    rn = g_rn + base_off;
    deg = g_deg + base_off;
    vw = g_vw + base_off;
    nb = g_nb;
    nw = g_nw;
    state = nullptr;
    for (i32 i = threadIdx.x; i < s; i += blockDim.x) rb[i] = xadj[M[i]];
    __syncthreads();
  }
  for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
    const i32 v = M[i];
    const i32 b = xadj[v], e1 = xadj[v + 1];
    if (e1 - b > kGggpLongRow) continue;   // a warp fills it below
    i32 j = rb[i];
    for (i32 e = b; e < e1; ++e) {
      const i32 u = adjncy[e];
      if (lo[u] == p0) {
        nb[j] = loc[u];
        nw[j] = adjwgt[e];
        ++j;
      }
    }
  }
  // long rows: one warp each, kept neighbours in row order
  for (i32 q = wid; q < nq; q += (i32)(blockDim.x >> 5)) {
    const i32 i = listed ? s_long[q] : q;
    const i32 v = M[i];
    const i32 b = xadj[v], e1 = xadj[v + 1];
    if (e1 - b <= kGggpLongRow) continue;   // warp-uniform (scan mode only)
    i32 j = rb[i];
    for (i32 e0 = b; e0 < e1; e0 += 32) {
      const i32 e = e0 + lane;
      i32 u = 0;
      bool keep = false;
      if (e < e1) {
        u = adjncy[e];
        keep = lo[u] == p0;
      }
      const u32 m = __ballot_sync(kFull32, keep);
      if (keep) {
        const i32 at = j + __popc(m & ((1u << lane) - 1));
        nb[at] = loc[u];
        nw[at] = adjwgt[e];
      }
      j += __popc(m);
    }
  }
  __syncthreads();
  if (big) {
    if (threadIdx.x == 0) {
      BigParams bp;
      bp.TL = TL;
      bp.WS = WS;
      bp.capL = capL;
      bp.capR = capR;
      bp.pm = pm;
      bp.p1 = p1;
      bigp[p0] = bp;
      biglist[atomicAdd(bigcount, 1)] = p0;
    }
    return;
  }
  T.rb = rb;
  T.rn = rn;
  T.nb = nb;
  T.nw = nw;
  T.degS = deg;
  T.vw = vw;
  const i32 t = wid;
  if (t < trials) {
    TrialState S;
    if (in_smem) {
      i32* q = state + (size_t)t * stw;   // [C | R | K | B1 | B2]
      S.C = q;
      S.R = q + s;
      S.K = reinterpret_cast<u64*>(q + 2 * s);
      S.B1 = S.K + s;
      S.B2 = S.B1 + gggp_nb1(s);
    } else {
      // [C | R] of n each per trial, this sub-problem at base_off; key blocks
      // at base_off / 32 + p0 and base_off / 1024 + p0 (disjoint across the
      // sub-problems, which lie in part order)
      i32* q = g_state + (size_t)t * 2 * n;
      S.C = q + base_off;
      S.R = q + n + base_off;
      S.K = g_keys + (size_t)t * n + base_off;
      const size_t nbw = (size_t)gggp_nb1(s) + gggp_nb2(s);
      if (nbw * sizeof(u64) * trials <= kGggpSmem) {
        // the block maxima fit in shared memory (the topology and the rest
        // of the state did not): every scan and block update stays on chip
        S.B1 = reinterpret_cast<u64*>(smem_raw) + (size_t)t * nbw;
        S.B2 = S.B1 + gggp_nb1(s);
      } else {
        S.B1 = g_b1 + (size_t)t * b1_stride + (base_off >> 5) + p0;
        S.B2 = g_b2 + (size_t)t * b2_stride + (base_off >> 10) + p0;
      }
    }
    // the seed names the part by its own graph's id (batched levels: parts are global)
    const i32 p0_local = part_base ? p0 - part_base[p0] : p0;
    const i32 pick = (i32)(mix32(seed * 0x9e3779b97f4a7c15ull + (u64)p0_local * 1315423911ull + (u64)t) % (u32)s);
    i64 cut, dev;
    gggp_trial(T, S, s, pick, TL, WS, capL, capR, cut, dev, prof);
    if (lane == 0) {
      s_cut[t] = cut;
      s_dev[t] = dev;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    i32 b = 0;
    for (i32 q = 1; q < trials; ++q)
      if (s_cut[q] < s_cut[b] || (s_cut[q] == s_cut[b] && s_dev[q] < s_dev[b])) b = q;
    s_best = b;
  }
  __syncthreads();
  const i32* Rb = in_smem ? state + (size_t)s_best * stw + s : g_state + (size_t)s_best * 2 * n + n + base_off;
  for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
    const i32 v = M[i];
    if (Rb[i]) { lo_out[v] = p0; hi_out[v] = pm; }
    else { lo_out[v] = pm; hi_out[v] = p1; }
  }
}

// ---------------------------------------------------------------------------
// Large sub-problems: one CTA per (sub-problem, trial).  The depth kernel has
// built the local CSR in the global arrays (rows at the members' CSR
// positions) and listed the sub-problem; here the trial's state -- C, R and
// the block maxima of the growth keys, and, when they fit, the members'
// weights to the sub-problem and vertex weights -- sits in the CTA's shared
// memory, so a growth step is a chain of on-chip accesses instead of L2 round
// trips, and the eight trials run on eight SMs.  A member's growth key is a
// function of C, R and degS (it only rises while the member is unassigned),
// so it is recomputed instead of stored.  Growth is one warp (the picks are
// sequential); the refinement scans and the final cut use the whole CTA.
// The picks, moves and results are those of gggp_trial.
// ---------------------------------------------------------------------------
constexpr int kBigThreads = 512;
constexpr size_t kGggpBigSmem = 224 * 1024;

__device__ __forceinline__ u64 member_key(const i32* C, const u8* R, const i32* deg, i32 i) {
  if (R[i]) return 0ull;
  const i32 c = C[i];
  return grow_key(c > 0, 2 * c - deg[i], i);
}

__device__ __forceinline__ u64 block_max_u64(u64 x, u64* s_red) {
  x = warp_max_u64(x);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = x;
  __syncthreads();
  u64 r = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = r > s_red[w] ? r : s_red[w];
  return r;
}

__device__ __forceinline__ i64 block_sum_i64(i64 x, i64* s_red) {
  x = warp_sum_i64(x);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = x;
  __syncthreads();
  i64 r = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += s_red[w];
  return r;
}

__global__ void __launch_bounds__(kBigThreads, 1) k_gggp_big_trial(
    i32 n, const i32* __restrict__ cnt, const i32* __restrict__ off, const i32* __restrict__ bigcount,
    const i32* __restrict__ biglist, const BigParams* __restrict__ bigp, i32 trials, u64 seed,
    const i32* __restrict__ part_base, const i32* __restrict__ g_rb, const i32* __restrict__ g_rn,
    const i32* __restrict__ g_deg, const i32* __restrict__ g_vw, const i32* __restrict__ g_nb,
    const i32* __restrict__ g_nw, i32* g_C, u8* g_R, i64* tcut, i64* tdev, unsigned long long* prof) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ u64 s_red[kBigThreads / 32];
  __shared__ i64 s_red64[kBigThreads / 32];
  __shared__ i64 s_wR;
  const i32 j = blockIdx.x / trials, t = blockIdx.x % trials;
  if (j >= *bigcount) return;
  const i32 p0 = biglist[j];
  const i32 s = cnt[p0], base = off[p0];
  const BigParams P = bigp[p0];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const i32* rb = g_rb + base;
  const i32* rn = g_rn + base;
  const i32* nbr = g_nb;
  const i32* nwt = g_nw;
  const i32 nb1 = gggp_nb1(s), nb2 = gggp_nb2(s);
  // shared layout: B1 | B2 | C | deg | vw | R, tiers by size (block-uniform)
  u64* B1 = reinterpret_cast<u64*>(smem_raw);
  u64* B2 = B1 + nb1;
  unsigned char* q = reinterpret_cast<unsigned char*>(B2 + nb2);
  const size_t fixed = sizeof(u64) * ((size_t)nb1 + nb2);
  const size_t all = fixed + (size_t)13 * s, mid = fixed + (size_t)5 * s;
  i32* C;
  const i32 *deg, *vw;
  u8* R;
  if (all <= kGggpBigSmem) {
    i32* sc = reinterpret_cast<i32*>(q);
    i32* sd = sc + s;
    i32* sv = sd + s;
    for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
      sd[i] = g_deg[base + i];
      sv[i] = g_vw[base + i];
    }
    C = sc;
    deg = sd;
    vw = sv;
    R = reinterpret_cast<u8*>(sv + s);
  } else if (mid <= kGggpBigSmem) {
    C = reinterpret_cast<i32*>(q);
    R = reinterpret_cast<u8*>(C + s);
    deg = g_deg + base;
    vw = g_vw + base;
  } else {
    C = g_C + (size_t)t * n + base;
    R = g_R + (size_t)t * n + base;
    deg = g_deg + base;
    vw = g_vw + base;
  }
  for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
    C[i] = 0;
    R[i] = 0;
  }
  __syncthreads();
  // block maxima of the initial keys (C = 0): one warp per block of 32 members
  for (i32 b = wid; b < nb1; b += nw) {
    const i32 i = (b << 5) + lane;
    const u64 m = warp_max_u64(i < s ? grow_key(false, -deg[i], i) : 0ull);
    if (lane == 0) B1[b] = m;
  }
  __syncthreads();
  for (i32 c = wid; c < nb2; c += nw) {
    const i32 b = (c << 5) + lane;
    const u64 m = warp_max_u64(b < nb1 ? B1[b] : 0ull);
    if (lane == 0) B2[c] = m;
  }
  __syncthreads();
  const long long c0 = clock64();
  if (wid == 0) {
    // ---- growth: the picks of grow_blocks ----
    const i32 p0_local = part_base ? p0 - part_base[p0] : p0;
    i32 pick = (i32)(mix32(seed * 0x9e3779b97f4a7c15ull + (u64)p0_local * 1315423911ull + (u64)t) % (u32)s);
    i64 wR = 0;
    for (i32 step = 0; step < s; ++step) {
      if (step > 0) {
        u64 best = 0;
        for (i32 c = lane; c < nb2; c += 32) best = best > B2[c] ? best : B2[c];
        best = warp_max_u64(best);
        if (best == 0) break;
        pick = key_idx(best);
      }
      const i64 w = (u32)vw[pick];
      const i32 r0 = rb[pick], rc = rn[pick];
      if (step > 0 && wR + w > P.TL && (wR + w - P.TL) > (P.TL - wR)) break;
      if (lane == 0) R[pick] = 1;
      wR += w;
      __syncwarp();
      constexpr i32 kU = 4;
      for (i32 j0 = lane; j0 < rc; j0 += 32 * kU) {
        i32 u[kU], ew[kU], ru[kU], du[kU], cu[kU];
#pragma unroll
        for (i32 x = 0; x < kU; ++x) {
          const i32 jj = j0 + 32 * x;
          u[x] = jj < rc ? nbr[r0 + jj] : -1;
          ew[x] = jj < rc ? nwt[r0 + jj] : 0;
        }
#pragma unroll
        for (i32 x = 0; x < kU; ++x) {
          if (u[x] >= 0) {
            ru[x] = R[u[x]];
            du[x] = deg[u[x]];
            cu[x] = atomicAdd(&C[u[x]], ew[x]) + ew[x];   // a row may list a neighbour twice
          }
        }
#pragma unroll
        for (i32 x = 0; x < kU; ++x) {
          if (u[x] >= 0 && !ru[x]) {
            const unsigned long long key = grow_key(cu[x] > 0, 2 * cu[x] - du[x], u[x]);
            atomicMax(reinterpret_cast<unsigned long long*>(&B1[u[x] >> 5]), key);
            atomicMax(reinterpret_cast<unsigned long long*>(&B2[u[x] >> 10]), key);
          }
        }
      }
      __syncwarp();
      {   // the picked member leaves its blocks
        const i32 b = pick >> 5, i = (b << 5) + lane;
        const u64 m = warp_max_u64(i < s ? member_key(C, R, deg, i) : 0ull);
        if (lane == 0) B1[b] = m;
        __syncwarp();
        const i32 c = pick >> 10, bb = (c << 5) + lane;
        const u64 m2 = warp_max_u64(bb < nb1 ? B1[bb] : 0ull);
        if (lane == 0) B2[c] = m2;
        __syncwarp();
      }
      if (wR >= P.TL) break;
    }
    if (lane == 0) s_wR = wR;
  }
  __syncthreads();
  const long long c1 = clock64();
  i64 wR = s_wR;
  // ---- refinement: positive-gain moves within the side caps (gggp_trial) ----
  const i32 max_moves = gggp_max_moves(s);
  for (i32 mv = 0; mv < max_moves; ++mv) {
    u64 best = 0;
    for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
      const i32 r = R[i], c = C[i], d = deg[i];
      const i32 g = r ? (d - 2 * c) : (2 * c - d);
      if (g > 0) {
        const i64 w = (u32)vw[i];
        const bool ok = r ? ((P.WS - wR) + w <= P.capR) : (wR + w <= P.capL);
        if (ok) {
          const u64 key = move_key2(g, i);
          best = best > key ? best : key;
        }
      }
    }
    best = block_max_u64(best, s_red);
    if (best == 0) break;
    const i32 i = key_idx(best);
    const i32 r = R[i];
    __syncthreads();   // every thread has read R[i] before it flips
    if (threadIdx.x == 0) R[i] = (u8)(r ^ 1);
    wR += r ? -(i64)(u32)vw[i] : (i64)(u32)vw[i];
    const i32 sign = r ? -1 : 1;
    const i32 r0 = rb[i], rc = rn[i];
    for (i32 jj = threadIdx.x; jj < rc; jj += blockDim.x) atomicAdd(&C[nbr[r0 + jj]], sign * nwt[r0 + jj]);
    __syncthreads();
  }
  i64 cut = 0;
  for (i32 i = threadIdx.x; i < s; i += blockDim.x)
    if (R[i]) cut += deg[i] - C[i];
  cut = block_sum_i64(cut, s_red64);
  u8* Rout = g_R + (size_t)t * n + base;
  if (Rout != R)
    for (i32 i = threadIdx.x; i < s; i += blockDim.x) Rout[i] = R[i];
  if (threadIdx.x == 0) {
    tcut[(size_t)p0 * trials + t] = cut;
    tdev[(size_t)p0 * trials + t] = wR > P.TL ? wR - P.TL : P.TL - wR;
    if (prof) {
      atomicMax(prof, (unsigned long long)(c1 - c0));
      atomicMax(prof + 1, (unsigned long long)(clock64() - c1));
    }
  }
}

// The winning trial of each large sub-problem (smallest cut, then smallest
// |W(R) - TL|, then the lower trial) splits it, as in k_gggp_depth.
__global__ void k_gggp_big_pick(i32 n, const i32* __restrict__ cnt, const i32* __restrict__ off,
                                const i32* __restrict__ bigcount, const i32* __restrict__ biglist,
                                const BigParams* __restrict__ bigp, i32 trials, const i32* __restrict__ mlist,
                                const u8* __restrict__ g_R, const i64* __restrict__ tcut,
                                const i64* __restrict__ tdev, i32* __restrict__ lo_out, i32* __restrict__ hi_out) {
  const i32 j = blockIdx.x;
  if (j >= *bigcount) return;
  const i32 p0 = biglist[j];
  const i32 s = cnt[p0], base = off[p0];
  const BigParams P = bigp[p0];
  i32 b = 0;
  for (i32 q = 1; q < trials; ++q) {
    const i64 cq = tcut[(size_t)p0 * trials + q], cb = tcut[(size_t)p0 * trials + b];
    if (cq < cb || (cq == cb && tdev[(size_t)p0 * trials + q] < tdev[(size_t)p0 * trials + b])) b = q;
  }
  const u8* R = g_R + (size_t)b * n + base;
  for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
    const i32 v = mlist[base + i];
    if (R[i]) { lo_out[v] = p0; hi_out[v] = P.pm; }
    else { lo_out[v] = P.pm; hi_out[v] = P.p1; }
  }
}

__global__ void k_init_fill(i32 n, i32* lo, i32* hi, i32 k) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) { lo[v] = 0; hi[v] = k; }
}

__global__ void k_init_fill_batch(i32 n, const i32* __restrict__ gid, const i32* __restrict__ gpbase,
                                  const i32* __restrict__ gk, i32* lo, i32* hi) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) {
    const i32 g = gid[v];
    lo[v] = gpbase[g];
    hi[v] = gpbase[g] + gk[g];
  }
}

static void device_init_partition_body(Handle& h, const DevGraph& g, i32 k, double eps, u64 seed, i32 trials,
                                       i32* d_part, const GggpBatch* batch);

// The launch sequence (a handful of launches per recursion depth, sized by n
// and k) runs through the handle's graph cache, except when traced or batched.
void device_init_partition(Handle& h, const DevGraph& g, i32 k, double eps, u64 seed, i32 trials,
                           i32* d_part, const GggpBatch* batch) {
  GKW_REQUIRE(trials >= 1 && trials <= kInitTrials, GKW_E_INVALID, "init trials must be in [1, 8]");
  if (g.n == 0) return;
  GKW_CUDA(cudaFuncSetAttribute(k_gggp_big_trial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGggpBigSmem));
  GKW_CUDA(cudaFuncSetAttribute(k_gggp_depth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGggpSmem));
  const bool trace = getenv("GKW_TRACE") && *getenv("GKW_TRACE") == '1';
  auto body = [&] { device_init_partition_body(h, g, k, eps, seed, trials, d_part, batch); };
  if (trace || batch) {
    body();
    return;
  }
  struct K {
    i64 n, m, k, trials;
    double eps;
    u64 seed;
    const void* p[5];
    const void* sbase;
    size_t stop;
    i32 narrow, sms;
    const void* scan;
  } key;
  memset(&key, 0, sizeof(key));
  key.n = g.n;
  key.m = g.m;
  key.k = k;
  key.trials = trials;
  key.eps = eps;
  key.seed = seed;
  key.p[0] = g.xadj;
  key.p[1] = g.adjncy;
  key.p[2] = g.adjwgt;
  key.p[3] = g.vwgt;
  key.p[4] = d_part;
  const auto fp = h.scratch.fingerprint();
  key.sbase = fp.first;
  key.stop = fp.second;
  key.narrow = h.narrow;
  key.sms = h.sm_count;
  key.scan = h.scan;
  graph_run(h, std::string("gggp", 4) + std::string(reinterpret_cast<const char*>(&key), sizeof(key)), body);
}

static void device_init_partition_body(Handle& h, const DevGraph& g, i32 k, double eps, u64 seed, i32 trials,
                                       i32* d_part, const GggpBatch* batch) {
  const i32 n = g.n;
  Pool::Mark mk = h.scratch.mark();
  i32* lo[2] = {h.scratch.alloc_n<i32>(n), h.scratch.alloc_n<i32>(n)};
  i32* hi[2] = {h.scratch.alloc_n<i32>(n), h.scratch.alloc_n<i32>(n)};
  i32* cnt = h.scratch.alloc_n<i32>(k);
  i32* off = h.scratch.alloc_n<i32>(k);
  i32* mlist = h.scratch.alloc_n<i32>(n);
  i32* loc = h.scratch.alloc_n<i32>(n);
  i32* g_rb = h.scratch.alloc_n<i32>(n);
  i32* g_rn = h.scratch.alloc_n<i32>(n);
  i32* g_deg = h.scratch.alloc_n<i32>(n);
  i32* g_vw = h.scratch.alloc_n<i32>(n);
  i32* g_nb = h.scratch.alloc_n<i32>(std::max<i64>(g.m, 1));
  i32* g_nw = h.scratch.alloc_n<i32>(std::max<i64>(g.m, 1));
  i32* g_state = h.scratch.alloc_n<i32>((size_t)kInitTrials * 2 * n);
  u64* g_keys = h.scratch.alloc_n<u64>((size_t)kInitTrials * n);
  // key blocks: sub-problem p0 at offset base_off uses [base_off/32 + p0, + ceil(s/32))
  const size_t b1_stride = (size_t)n / 32 + (size_t)k + 2, b2_stride = (size_t)n / 1024 + (size_t)k + 2;
  u64* g_b1 = h.scratch.alloc_n<u64>((size_t)kInitTrials * b1_stride);
  u64* g_b2 = h.scratch.alloc_n<u64>((size_t)kInitTrials * b2_stride);
  // large sub-problems (more than kGggpBlockMin members; at most maxbig of
  // them per depth) run their trials as separate CTAs
  const i32 maxbig = n / (kGggpBlockMin + 1);
  i32* bigcount = nullptr;
  i32* biglist = nullptr;
  BigParams* bigp = nullptr;
  i64* tcut = nullptr;
  i64* tdev = nullptr;
  u8* g_R = nullptr;
  if (maxbig > 0) {
    bigcount = h.scratch.alloc_n<i32>(1);
    biglist = h.scratch.alloc_n<i32>(maxbig);
    bigp = h.scratch.alloc_n<BigParams>(k);
    tcut = h.scratch.alloc_n<i64>((size_t)k * kInitTrials);
    tdev = h.scratch.alloc_n<i64>((size_t)k * kInitTrials);
    g_R = h.scratch.alloc_n<u8>((size_t)kInitTrials * n);
  }
  const u32 nb = ceil_div(n, 256);
  i32 depth = 0;
  if (batch) {
    launch(k_init_fill_batch, nb, 256, 0, h.stream, n, batch->gid, batch->gpbase, batch->gk, lo[0], hi[0]);
    depth = batch->depth;
  } else {
    launch(k_init_fill, nb, 256, 0, h.stream, n, lo[0], hi[0], k);
    while ((1 << depth) < k) ++depth;
  }
  GKW_CHECK_LAUNCH();
  const bool trace = getenv("GKW_TRACE") && *getenv("GKW_TRACE") == '1';
  std::vector<cudaEvent_t> ev;
  unsigned long long* prof = nullptr;   // per depth: slowest trial's growth / refinement cycles
  if (trace) {
    prof = reinterpret_cast<unsigned long long*>(h.scratch.alloc_n<u64>(2 * (size_t)std::max(depth, 1)));
    GKW_CUDA(cudaMemsetAsync(prof, 0, sizeof(u64) * 2 * std::max(depth, 1), h.stream));
    ev.resize(depth + 1);
    for (auto& e : ev) GKW_CUDA(cudaEventCreate(&e));
    GKW_CUDA(cudaEventRecord(ev[0], h.stream));
  }
  for (i32 d = 0; d < depth; ++d) {
    const i32 a = d & 1, b = a ^ 1;
    GKW_CUDA(cudaMemsetAsync(cnt, 0, sizeof(i32) * k, h.stream));
    launch(k_init_count, nb, 256, 0, h.stream, n, lo[a], cnt);
    GKW_CHECK_LAUNCH();
    exclusive_scan_i32(h, cnt, off, k, nullptr);
    if (maxbig > 0) GKW_CUDA(cudaMemsetAsync(bigcount, 0, sizeof(i32), h.stream));
    const i32* pbase = batch ? batch->part_base : nullptr;
    launch(k_gggp_depth, k, kInitTrials * 32, kGggpSmem, h.stream, n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, lo[a],
           hi[a], cnt, off, mlist, loc, lo[b], hi[b], seed, eps, trials, g_rb, g_rn, g_deg, g_vw, g_nb, g_nw,
           g_state, g_keys, g_b1, g_b2, b1_stride, b2_stride, pbase,
           batch ? batch->part_v0 : (const i32*)nullptr, batch ? batch->part_v1 : (const i32*)nullptr,
           prof ? prof + 2 * d : nullptr, bigcount, biglist, bigp);
    GKW_CHECK_LAUNCH();
    if (maxbig > 0) {
      launch(k_gggp_big_trial, (u32)maxbig * trials, kBigThreads, kGggpBigSmem, h.stream, n, (const i32*)cnt,
             (const i32*)off, (const i32*)bigcount, (const i32*)biglist, (const BigParams*)bigp, trials, seed, pbase,
             (const i32*)g_rb, (const i32*)g_rn, (const i32*)g_deg, (const i32*)g_vw, (const i32*)g_nb,
             (const i32*)g_nw, g_state, g_R, tcut, tdev, prof ? prof + 2 * d : nullptr);
      GKW_CHECK_LAUNCH();
      launch(k_gggp_big_pick, (u32)maxbig, 256, 0, h.stream, n, (const i32*)cnt, (const i32*)off,
             (const i32*)bigcount, (const i32*)biglist, (const BigParams*)bigp, trials, (const i32*)mlist,
             (const u8*)g_R, (const i64*)tcut, (const i64*)tdev, lo[b], hi[b]);
      GKW_CHECK_LAUNCH();
    }
    if (trace) GKW_CUDA(cudaEventRecord(ev[d + 1], h.stream));
  }
  if (trace) {
    GKW_CUDA(cudaEventSynchronize(ev[depth]));
    std::vector<unsigned long long> hp(2 * (size_t)std::max(depth, 1));
    if (depth) {
      GKW_CUDA(cudaMemcpyAsync(hp.data(), prof, sizeof(u64) * 2 * depth, cudaMemcpyDeviceToHost, h.stream));
      GKW_CUDA(cudaStreamSynchronize(h.stream));
    }
    fprintf(stderr, "[gkw trace] init n=%d k=%d:", n, k);
    for (i32 d = 0; d < depth; ++d) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[d], ev[d + 1]);
      fprintf(stderr, " d%d %.1fus (growth %.2f, refinement %.2f Mcycles)", d, ms * 1e3, hp[2 * d] / 1e6,
              hp[2 * d + 1] / 1e6);
    }
    fprintf(stderr, "\n");
    for (auto& e : ev) cudaEventDestroy(e);
  }
  GKW_CUDA(cudaMemcpyAsync(d_part, lo[depth & 1], sizeof(i32) * n, cudaMemcpyDeviceToDevice, h.stream));
  h.scratch.release(mk);   // stream order keeps the scratch alive for the queued work
}

}  // namespace gkw
