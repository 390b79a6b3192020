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

__device__ __forceinline__ u64 warp_max_u64(u64 x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const u64 y = __shfl_xor_sync(kFull32, x, o);
    x = x > y ? x : y;
  }
  return x;
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

__global__ void __launch_bounds__(kInitTrials * 32) k_gggp_depth(
    i32 n, const i32* __restrict__ xadj, const i32* __restrict__ adjncy, const i32* __restrict__ adjwgt,
    const i32* __restrict__ vwgt, const i32* __restrict__ lo, const i32* __restrict__ hi,
    const i32* __restrict__ cnt, const i32* __restrict__ off, i32* __restrict__ mlist,
    i32* __restrict__ degS, i32* __restrict__ inR, i32* __restrict__ conn, i32* __restrict__ lo_out,
    i32* __restrict__ hi_out, u64 seed, double eps, i32 trials, i32* __restrict__ loc, i32* __restrict__ frontier,
    i32* __restrict__ fpos) {
  __shared__ i32 s_cnt;
  __shared__ i64 s_wsum[kInitTrials];
  __shared__ i64 s_cut[kInitTrials];
  __shared__ i64 s_dev[kInitTrials];
  __shared__ i32 s_best;
  const i32 p0 = blockIdx.x;
  const i32 s = cnt[p0];
  if (s == 0) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  i32* M = mlist + off[p0];
  // deterministic member list: all vertices with lo == p0, in id order
  __shared__ i32 s_wc[kInitTrials];
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  for (i32 base = 0; base < n; base += blockDim.x) {
    const i32 v = base + threadIdx.x;
    const bool mine = v < n && lo[v] == p0;
    const u32 bal = __ballot_sync(kFull32, mine);
    if (lane == 0) s_wc[wid] = __popc(bal);
    __syncthreads();
    i32 woff = 0, tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      if (w < wid) woff += s_wc[w];
      tot += s_wc[w];
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
  // deg_S and W(S)
  i64 wpart = 0;
  for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
    const i32 v = M[i];
    i32 d = 0;
    for (i32 e = xadj[v]; e < xadj[v + 1]; ++e)
      if (lo[adjncy[e]] == p0) d += adjwgt[e];
    degS[v] = d;
    wpart += (u32)vwgt[v];
  }
  wpart = warp_sum_i64(wpart);
  if (lane == 0) s_wsum[wid] = wpart;
  __syncthreads();
  i64 WS = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) WS += s_wsum[w];
  const i64 TL = WS * (pm - p0) / (p1 - p0);
  const i64 capL = (i64)((double)TL * (1.0 + eps * 0.5));
  const i64 capR = (i64)((double)(WS - TL) * (1.0 + eps * 0.5));

  const i32 t = wid;
  if (t < trials) {
    i32* R = inR + (i64)t * n;
    i32* C = conn + (i64)t * n;
    for (i32 i = lane; i < s; i += 32) {
      R[M[i]] = 0;
      C[M[i]] = 0;
    }
    __syncwarp();
    i64 wR = 0;
    // ---- growth ----
    // F = the members outside R with conn > 0 (the frontier).  A frontier
    // vertex always outranks a non-frontier one, so while F is not empty the
    // argmax over F equals the argmax over all unassigned members; the full
    // scan is only needed when F is empty.
    // F holds at most s entries: this sub-problem's slice [off, off + s) of
    // the trial's list (sub-problems of one depth run concurrently)
    i32* F = frontier + (i64)t * n + off[p0];
    i32* posF = fpos + (i64)t * n;
    i32 nF = 0;
    i32 pick = (i32)(mix32(seed * 0x9e3779b97f4a7c15ull + (u64)p0 * 1315423911ull + (u64)t) % (u32)s);
    for (i32 step = 0; step < s; ++step) {
      if (step > 0) {
        u64 best = 0;
        if (nF > 0) {
          for (i32 f = lane; f < nF; f += 32) {
            const i32 v = F[f];
            const i32 c = C[v];
            const u64 key = grow_key(true, 2 * c - degS[v], loc[v]);
            best = best > key ? best : key;
          }
        } else {
          for (i32 i = lane; i < s; i += 32) {
            const i32 v = M[i];
            if (!R[v]) {
              const i32 c = C[v];
              const u64 key = grow_key(c > 0, 2 * c - degS[v], i);
              best = best > key ? best : key;
            }
          }
        }
        best = warp_max_u64(best);
        if (best == 0) break;
        pick = key_idx(best);
        const i64 vw = (u32)vwgt[M[pick]];
        if (wR + vw > TL && (wR + vw - TL) > (TL - wR)) break;
      }
      const i32 v = M[pick];
      // leave the frontier (swap-remove), enter R
      if (lane == 0) {
        R[v] = 1;
        if (C[v] > 0) {
          const i32 at = posF[v];
          const i32 last = F[nF - 1];
          F[at] = last;
          posF[last] = at;
        }
      }
      if (C[v] > 0) --nF;
      wR += (u32)vwgt[v];
      __syncwarp();
      // neighbours gain connection; those reaching conn > 0 join the frontier
      for (i32 e0 = xadj[v]; e0 < xadj[v + 1]; e0 += 32) {
        const i32 e = e0 + lane;
        bool join = false;
        i32 u = 0;
        if (e < xadj[v + 1]) {
          u = adjncy[e];
          if (lo[u] == p0) {
            const i32 old = C[u];
            C[u] = old + adjwgt[e];
            join = !R[u] && old <= 0 && old + adjwgt[e] > 0;
          }
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
    // ---- refinement: positive-gain moves within the side caps ----
    const i32 max_moves = s / 4 + 32;
    for (i32 mv = 0; mv < max_moves; ++mv) {
      u64 best = 0;
      for (i32 i = lane; i < s; i += 32) {
        const i32 v = M[i];
        const i32 r = R[v];
        const i32 c = C[v], d = degS[v];
        const i32 g = r ? (d - 2 * c) : (2 * c - d);
        if (g <= 0) continue;
        const i64 vw = (u32)vwgt[v];
        const bool ok = r ? ((WS - wR) + vw <= capR) : (wR + vw <= capL);
        if (!ok) continue;
        const u64 key = move_key2(g, i);
        best = best > key ? best : key;
      }
      best = warp_max_u64(best);
      if (best == 0) break;
      const i32 v = M[key_idx(best)];
      const i32 r = R[v];
      __syncwarp();
      if (lane == 0) R[v] = r ^ 1;
      wR += r ? -(i64)(u32)vwgt[v] : (i64)(u32)vwgt[v];
      const i32 sign = r ? -1 : 1;
      for (i32 e = xadj[v] + lane; e < xadj[v + 1]; e += 32) {
        const i32 u = adjncy[e];
        if (lo[u] == p0) C[u] += sign * adjwgt[e];
      }
      __syncwarp();
    }
    // ---- cut of this trial ----
    i64 cut = 0;
    for (i32 i = lane; i < s; i += 32) {
      const i32 v = M[i];
      if (R[v]) cut += degS[v] - C[v];
    }
    cut = warp_sum_i64(cut);
    if (lane == 0) {
      s_cut[t] = cut;
      s_dev[t] = wR > TL ? wR - TL : TL - wR;
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
  const i32* R = inR + (i64)s_best * n;
  for (i32 i = threadIdx.x; i < s; i += blockDim.x) {
    const i32 v = M[i];
    if (R[v]) { lo_out[v] = p0; hi_out[v] = pm; }
    else { lo_out[v] = pm; hi_out[v] = p1; }
  }
}

__global__ void k_init_fill(i32 n, i32* lo, i32* hi, i32 k) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) { lo[v] = 0; hi[v] = k; }
}

void device_init_partition(Handle& h, const DevGraph& g, i32 k, double eps, u64 seed, i32 trials,
                           i32* d_part) {
  GKW_REQUIRE(trials >= 1 && trials <= kInitTrials, GKW_E_INVALID, "init trials must be in [1, 8]");
  const i32 n = g.n;
  if (n == 0) return;
  Pool::Mark mk = h.scratch.mark();
  i32* lo[2] = {h.scratch.alloc_n<i32>(n), h.scratch.alloc_n<i32>(n)};
  i32* hi[2] = {h.scratch.alloc_n<i32>(n), h.scratch.alloc_n<i32>(n)};
  i32* cnt = h.scratch.alloc_n<i32>(k);
  i32* off = h.scratch.alloc_n<i32>(k);
  i32* mlist = h.scratch.alloc_n<i32>(n);
  i32* degS = h.scratch.alloc_n<i32>(n);
  i32* inR = h.scratch.alloc_n<i32>((i64)kInitTrials * n);
  i32* conn = h.scratch.alloc_n<i32>((i64)kInitTrials * n);
  i32* loc = h.scratch.alloc_n<i32>(n);
  i32* frontier = h.scratch.alloc_n<i32>((i64)kInitTrials * n);
  i32* fpos = h.scratch.alloc_n<i32>((i64)kInitTrials * n);
  const u32 nb = ceil_div(n, 256);
  launch(k_init_fill, nb, 256, 0, h.stream, n, lo[0], hi[0], k);
  GKW_CHECK_LAUNCH();
  i32 depth = 0;
  while ((1 << depth) < k) ++depth;
  const bool trace = getenv("GKW_TRACE") && *getenv("GKW_TRACE") == '1';
  std::vector<cudaEvent_t> ev;
  if (trace) {
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
    launch(k_gggp_depth, k, kInitTrials * 32, 0, h.stream, n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, lo[a], hi[a],
                                                        cnt, off, mlist, degS, inR, conn, lo[b], hi[b], seed,
                                                        eps, trials, loc, frontier, fpos);
    GKW_CHECK_LAUNCH();
    if (trace) GKW_CUDA(cudaEventRecord(ev[d + 1], h.stream));
  }
  if (trace) {
    GKW_CUDA(cudaEventSynchronize(ev[depth]));
    fprintf(stderr, "[gkw trace] init n=%d k=%d:", n, k);
    for (i32 d = 0; d < depth; ++d) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[d], ev[d + 1]);
      fprintf(stderr, " d%d %.1fus", d, ms * 1e3);
    }
    fprintf(stderr, "\n");
    for (auto& e : ev) cudaEventDestroy(e);
  }
  GKW_CUDA(cudaMemcpyAsync(d_part, lo[depth & 1], sizeof(i32) * n, cudaMemcpyDeviceToDevice, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  h.scratch.release(mk);
}

}  // namespace gkw
