// Projection and independent-set refinement (gkway/uncoarsen.hpp).
//
// The reference scans every vertex of the level in each refinement round.
// Here a round only touches two short lists: P, the vertices whose gain is
// positive (the only ones that can move or block a neighbour), and U, the
// vertices whose gain must be recomputed (moved vertices and their
// neighbours).  Both lists are maintained on the device; a round is five
// kernels and rounds are launched in batches with one host read per batch.
#include <algorithm>
#include <climits>

#include "gkw_internal.cuh"

namespace gkw {

static constexpr u32 kFullMask = 0xffffffffu;
constexpr i32 kSortMax = 4096;      // candidates sorted in one shared-memory pass
constexpr i32 kMaxMoveCap = 2048;   // largest supported move cap
constexpr i32 kBadWords = kMaxMoveCap / 32;

struct RoundState {
  i32 pcount[2];
  i32 pcur;
  i32 ucount;
  i32 ccount;
  i32 B;
  i32 done;
  i32 rounds;
  i64 moves;
  i64 gain_sum;
  u32 bad[kBadWords];
};

struct RefineCtx {
  i32 n_max = 0, k = 0, cap = 0;
  i32* part[2] = {nullptr, nullptr};
  i32* bnd[2] = {nullptr, nullptr};
  i32 cur = 0;
  i32* gain = nullptr;
  i32* target = nullptr;
  i32* updflag = nullptr;
  i32* inP = nullptr;
  i32* U = nullptr;
  i32* P[2] = {nullptr, nullptr};
  u64* cands = nullptr;
  u64* top = nullptr;
  u32* pw = nullptr;
  RoundState* st = nullptr;
  i32 upd_warps = 8;
};

RefineCtx* refine_create(Handle& h, i32 n_max, i32 k, i32 move_cap) {
  GKW_REQUIRE(move_cap >= 1 && move_cap <= kMaxMoveCap, GKW_E_UNSUPPORTED,
              "move_cap must be in [1, 2048]");
  GKW_REQUIRE(k >= 1 && k <= 12288, GKW_E_UNSUPPORTED, "k must be in [1, 12288]");
  RefineCtx* c = new RefineCtx();
  c->n_max = n_max;
  c->k = k;
  c->cap = move_cap;
  const size_t n = std::max(n_max, 1);
  Pool& P = h.hier;
  c->part[0] = P.alloc_n<i32>(n);
  c->part[1] = P.alloc_n<i32>(n);
  c->bnd[0] = P.alloc_n<i32>(n);
  c->bnd[1] = P.alloc_n<i32>(n);
  c->gain = P.alloc_n<i32>(n);
  c->target = P.alloc_n<i32>(n);
  c->updflag = P.alloc_n<i32>(n);
  c->inP = P.alloc_n<i32>(n);
  c->U = P.alloc_n<i32>(n);
  c->P[0] = P.alloc_n<i32>(n);
  c->P[1] = P.alloc_n<i32>(n);
  c->cands = P.alloc_n<u64>(n);
  c->top = P.alloc_n<u64>(kMaxMoveCap);
  c->pw = P.alloc_n<u32>(k);
  c->st = P.alloc_n<RoundState>(1);
  i32 w = (48 * 1024) / (4 * k);
  c->upd_warps = std::max(1, std::min(8, w));
  return c;
}

// A context over caller-owned state arrays (per-phase entry points).
RefineCtx* refine_create_ext(Handle& h, i32 n, i32 k, i32 move_cap, i32* part, i32* bnd, i32* gain,
                             i32* target) {
  GKW_REQUIRE(move_cap >= 1 && move_cap <= kMaxMoveCap, GKW_E_UNSUPPORTED,
              "move_cap must be in [1, 2048]");
  GKW_REQUIRE(k >= 1 && k <= 12288, GKW_E_UNSUPPORTED, "k must be in [1, 12288]");
  RefineCtx* c = new RefineCtx();
  c->n_max = n;
  c->k = k;
  c->cap = move_cap;
  const size_t nn = std::max(n, 1);
  Pool& P = h.scratch;
  c->part[0] = part;
  c->bnd[0] = bnd;
  c->part[1] = nullptr;
  c->bnd[1] = nullptr;
  c->gain = gain;
  c->target = target;
  c->updflag = P.alloc_n<i32>(nn);
  c->inP = P.alloc_n<i32>(nn);
  c->U = P.alloc_n<i32>(nn);
  c->P[0] = P.alloc_n<i32>(nn);
  c->P[1] = P.alloc_n<i32>(nn);
  c->cands = P.alloc_n<u64>(nn);
  c->top = P.alloc_n<u64>(kMaxMoveCap);
  c->pw = P.alloc_n<u32>(k);
  c->st = P.alloc_n<RoundState>(1);
  i32 w = (48 * 1024) / (4 * k);
  c->upd_warps = std::max(1, std::min(8, w));
  return c;
}

void refine_destroy(RefineCtx* c) { delete c; }
i32* refine_part(RefineCtx* c) { return c->part[c->cur]; }
i32* refine_boundary(RefineCtx* c) { return c->bnd[c->cur]; }
i32* refine_gain(RefineCtx* c) { return c->gain; }
i32* refine_target(RefineCtx* c) { return c->target; }
u32* refine_pw(RefineCtx* c) { return c->pw; }

// uncoarsen.hpp:10-21 (is_valid_move): (float)(u32)(dest + vwgt) > MAXW is invalid
__device__ __forceinline__ bool valid_move(u32 dest_w, u32 vw, float maxw) {
  return !(__uint2float_rn(dest_w + vw) > maxw);
}

// candidate key: ascending order = gain descending, vertex id ascending
__device__ __forceinline__ u64 move_key(i32 gain, i32 v) {
  return ((u64)(u32)(INT_MAX - gain) << 32) | (u32)v;
}

// ---------------------------------------------------------------------------
// Coarsest level: boundary flags and part weights of the initial partition
// (metis_partition.hpp:52-71).
// ---------------------------------------------------------------------------
__global__ void k_boundary_pw(i32 n, const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                              const i32* __restrict__ vwgt, const i32* __restrict__ part,
                              i32* __restrict__ bnd, u32* __restrict__ pw) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 p = part[v];
  i32 b = 0;
  for (i32 e = xadj[v]; e < xadj[v + 1]; ++e)
    if (part[adjncy[e]] != p) { b = 1; break; }
  bnd[v] = b;
  atomicAdd(&pw[p], (u32)vwgt[v]);
}

__global__ void k_copy_i32(i32 n, const i32* __restrict__ src, i32* __restrict__ dst) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) dst[v] = src[v];
}

void refine_init_coarsest(Handle& h, RefineCtx* c, const DevGraph& g, const i32* d_part_in) {
  c->cur = 0;
  GKW_CUDA(cudaMemsetAsync(c->pw, 0, sizeof(u32) * c->k, h.stream));
  if (g.n == 0) return;
  const u32 nb = ceil_div(g.n, 256);
  if (d_part_in != c->part[0]) {
    launch(k_copy_i32, nb, 256, 0, h.stream, g.n, d_part_in, c->part[0]);
    GKW_CHECK_LAUNCH();
  }
  launch(k_boundary_pw, nb, 256, 0, h.stream, g.n, g.xadj, g.adjncy, g.vwgt, c->part[0], c->bnd[0], c->pw);
  GKW_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Projection (uncoarsen.hpp:325-356, expand_partition): part and boundary
// inherited from the coarse vertex, gain 0, target = part, boundary vertices
// flagged for update (appended to U).
// ---------------------------------------------------------------------------
__global__ void k_project(i32 n, const i32* __restrict__ cmap, const i32* __restrict__ part_c,
                          const i32* __restrict__ bnd_c, i32* __restrict__ part_f, i32* __restrict__ bnd_f,
                          i32* __restrict__ gain, i32* __restrict__ target, i32* __restrict__ updflag,
                          i32* __restrict__ inP, i32* __restrict__ U, RoundState* __restrict__ st) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 c = cmap[v];
  const i32 p = part_c[c];
  const i32 b = bnd_c[c];
  part_f[v] = p;
  bnd_f[v] = b;
  gain[v] = 0;
  target[v] = p;
  inP[v] = 0;
  updflag[v] = b ? 1 : 0;
  if (b) U[atomicAdd(&st->ucount, 1)] = (i32)v;
}

// ---------------------------------------------------------------------------
// Gain update (uncoarsen.hpp:175-237, update_vertex_info + calculate_gain).
// One warp per vertex of U.  Per-part connection weights accumulate in a
// per-warp shared array of k words (only the touched entries are cleared
// afterwards).  The best part is the max of the UNSIGNED value (ed - id)
// over neighbouring parts other than the own part, ties to the smaller part
// id, and it is taken only if that unsigned value is > 0 -- the reference's
// `if (gain > max_gain)` with an unsigned max_gain.  Vertices whose new gain
// is positive join P.
// ---------------------------------------------------------------------------
__global__ void k_update(const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                         const i32* __restrict__ adjwgt, i32 k, const i32* __restrict__ part,
                         i32* __restrict__ bnd, i32* __restrict__ gain, i32* __restrict__ target,
                         i32* __restrict__ updflag, i32* __restrict__ inP, const i32* __restrict__ U,
                         i32* __restrict__ P0, i32* __restrict__ P1, RoundState* __restrict__ st) {
  extern __shared__ u32 acc_all[];
  if (st->done) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  u32* acc = acc_all + (size_t)wid * k;
  for (i32 q = lane; q < k; q += 32) acc[q] = 0;
  __syncwarp();
  const i32 nU = st->ucount;
  i32* Pout = st->pcur ? P1 : P0;
  i32* pcount = &st->pcount[st->pcur];
  const i64 nw = (i64)gridDim.x * wpb;
  for (i64 i = (i64)blockIdx.x * wpb + wid; i < nU; i += nw) {
    const i32 v = U[i];
    const i32 p = part[v];
    const i32 beg = xadj[v], end = xadj[v + 1];
    bool bl = false;
    for (i32 e = beg + lane; e < end; e += 32) {
      const i32 q = part[adjncy[e]];
      atomicAdd(&acc[q], (u32)adjwgt[e]);
      bl |= (q != p);
    }
    const bool b = __any_sync(kFullMask, bl);
    __syncwarp();
    u32 g = 0, q_best = (u32)p;
    if (b) {
      const u32 id = acc[p];
      u64 best = 0;
      for (i32 e = beg + lane; e < end; e += 32) {
        const i32 q = part[adjncy[e]];
        if (q != p) {
          const u64 key = ((u64)(acc[q] - id) << 32) | (u32)(~(u32)q);
          best = best > key ? best : key;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const u64 ot = __shfl_xor_sync(kFullMask, best, o);
        best = best > ot ? best : ot;
      }
      const u32 gb = (u32)(best >> 32);
      if (gb > 0) { g = gb; q_best = ~(u32)best; }
    }
    if (lane == 0) {
      updflag[v] = 0;
      bnd[v] = b ? 1 : 0;
      gain[v] = (i32)g;
      target[v] = (i32)q_best;
      if ((i32)g > 0 && atomicExch(&inP[v], 1) == 0) Pout[atomicAdd(pcount, 1)] = v;
    }
    __syncwarp();
    for (i32 e = beg + lane; e < end; e += 32) acc[part[adjncy[e]]] = 0;
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Move candidates (uncoarsen.hpp:111-173, create_independent_move_buffer):
// boundary, gain > 0, a valid destination by weight, and no neighbour with a
// smaller id that is itself positive and valid.  P is compacted on the way
// (entries whose gain is no longer positive leave it).
// ---------------------------------------------------------------------------
__global__ void k_candidates(const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                             const i32* __restrict__ vwgt, const i32* __restrict__ part,
                             const i32* __restrict__ bnd, const i32* __restrict__ gain,
                             const i32* __restrict__ target, const u32* __restrict__ pw, float maxw,
                             i32* __restrict__ inP, i32* __restrict__ P0, i32* __restrict__ P1,
                             u64* __restrict__ cands, RoundState* __restrict__ st) {
  if (st->done) return;
  const i32 pc = st->pcur;
  const i32 nP = st->pcount[pc];
  const i32* Pin = pc ? P1 : P0;
  i32* Pout = pc ? P0 : P1;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < nP; i += (i64)gridDim.x * blockDim.x) {
    const i32 v = Pin[i];
    const i32 g = gain[v];
    if (g <= 0) {
      inP[v] = 0;
      continue;
    }
    Pout[atomicAdd(&st->pcount[pc ^ 1], 1)] = v;
    if (!bnd[v]) continue;
    const i32 t = target[v];
    if (!valid_move(pw[t], (u32)vwgt[v], maxw)) continue;
    bool yield = false;
    for (i32 e = xadj[v]; e < xadj[v + 1]; ++e) {
      const i32 u = adjncy[e];
      if (u < v && gain[u] > 0 && valid_move(pw[target[u]], (u32)vwgt[u], maxw)) {
        yield = true;
        break;
      }
    }
    if (!yield) cands[atomicAdd(&st->ccount, 1)] = move_key(g, v);
  }
}

// ---------------------------------------------------------------------------
// Sort the candidates by (gain desc, id asc) and keep the first min(cnt, cap)
// (uncoarsen.hpp:471-476 with move_request.hpp:36-41).  One CTA; more than
// kSortMax candidates are streamed through a shared buffer that keeps the
// running top `cap`.  Also resets the per-round counters.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_select(const u64* __restrict__ cands, u64* __restrict__ top,
                                                 i32 cap, RoundState* __restrict__ st) {
  __shared__ u64 s[kSortMax];
  if (st->done) return;
  const i32 cnt = st->ccount;
  __syncthreads();
  if (cnt == 0) {
    if (threadIdx.x == 0) st->done = 1;
    return;
  }
  const i32 B = cnt < cap ? cnt : cap;
  if (cnt <= kSortMax) {
    i32 P = 32;
    while (P < cnt) P <<= 1;
    for (i32 i = threadIdx.x; i < P; i += blockDim.x) s[i] = i < cnt ? cands[i] : ~0ull;
    __syncthreads();
    for (i32 kk = 2; kk <= P; kk <<= 1)
      for (i32 j = kk >> 1; j > 0; j >>= 1) {
        for (i32 i = threadIdx.x; i < P; i += blockDim.x) {
          const i32 l = i ^ j;
          if (l > i) {
            const u64 x = s[i], y = s[l];
            const bool up = (i & kk) == 0;
            if (up ? (x > y) : (x < y)) { s[i] = y; s[l] = x; }
          }
        }
        __syncthreads();
      }
  } else {
    // running top-cap: s[0..cap) holds the best so far (sorted), the rest is refilled
    i32 next = 0;
    bool first = true;
    while (next < cnt) {
      const i32 lo = first ? 0 : cap;
      for (i32 i = lo + threadIdx.x; i < kSortMax; i += blockDim.x) {
        const i32 src = next + (i - lo);
        s[i] = src < cnt ? cands[src] : ~0ull;
      }
      next += kSortMax - lo;
      first = false;
      __syncthreads();
      for (i32 kk = 2; kk <= kSortMax; kk <<= 1)
        for (i32 j = kk >> 1; j > 0; j >>= 1) {
          for (i32 i = threadIdx.x; i < kSortMax; i += blockDim.x) {
            const i32 l = i ^ j;
            if (l > i) {
              const u64 x = s[i], y = s[l];
              const bool up = (i & kk) == 0;
              if (up ? (x > y) : (x < y)) { s[i] = y; s[l] = x; }
            }
          }
          __syncthreads();
        }
    }
  }
  for (i32 i = threadIdx.x; i < B; i += blockDim.x) top[i] = s[i];
  for (i32 i = threadIdx.x; i < (B + 31) / 32; i += blockDim.x) st->bad[i] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    st->B = B;
    st->ccount = 0;
    st->pcount[st->pcur] = 0;
    st->pcur ^= 1;
    st->ucount = 0;
  }
}

// ---------------------------------------------------------------------------
// Balance check (uncoarsen.hpp:239-288).  CTA p computes the prefix sums of
// part p's weight change over the sorted moves and flags every prefix index j
// whose change is positive and pushes part p over MAXW.  A prefix j is
// balanced when no part flags it.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_balance(const u64* __restrict__ top, const i32* __restrict__ part,
                                                  const i32* __restrict__ target, const i32* __restrict__ vwgt,
                                                  const u32* __restrict__ pw, float maxw,
                                                  RoundState* __restrict__ st) {
  __shared__ i32 s_warp[33];
  if (st->done) return;
  const i32 B = st->B;
  const i32 p = blockIdx.x;
  constexpr int IT = kMaxMoveCap / 1024;
  i32 e[IT];
  i32 sum = 0;
#pragma unroll
  for (int i = 0; i < IT; ++i) {
    const i32 j = threadIdx.x * IT + i;
    i32 d = 0;
    if (j < B) {
      const i32 v = (i32)(u32)top[j];
      const i32 w = vwgt[v];
      if (target[v] == p) d += w;
      if (part[v] == p) d -= w;
    }
    e[i] = d;
    sum += d;
  }
  // block exclusive scan of the per-thread sums
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  i32 inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const i32 y = __shfl_up_sync(kFullMask, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const i32 x = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
    i32 xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const i32 y = __shfl_up_sync(kFullMask, xi, o);
      if (lane >= o) xi += y;
    }
    s_warp[lane] = xi - x;
  }
  __syncthreads();
  i32 run = inc - sum + s_warp[wid];
  const u32 base = pw[p];
#pragma unroll
  for (int i = 0; i < IT; ++i) {
    const i32 j = threadIdx.x * IT + i;
    run += e[i];
    if (j < B && run > 0 && __uint2float_rn((u32)run + base) > maxw)
      atomicOr(&st->bad[j >> 5], 1u << (j & 31));
  }
}

// ---------------------------------------------------------------------------
// Apply the moves 0..pos, pos = the largest balanced prefix index
// (uncoarsen.hpp:284-286 take the max balanced index; prefix 0 is always
// balanced).  Part weights change by the same sums as pw[p] += D[p][pos];
// moved vertices and their neighbours are flagged and appended to U
// (uncoarsen.hpp:290-323).
// ---------------------------------------------------------------------------
__global__ void k_apply(const u64* __restrict__ top, const i32* __restrict__ xadj,
                        const i32* __restrict__ adjncy, const i32* __restrict__ vwgt, i32* __restrict__ part,
                        const i32* __restrict__ target, u32* __restrict__ pw, i32* __restrict__ updflag,
                        i32* __restrict__ U, RoundState* __restrict__ st) {
  if (st->done) return;
  const i32 B = st->B;
  i32 pos = 0;
  const i32 nwords = (B + 31) >> 5;
  for (i32 w = nwords - 1; w >= 0; --w) {
    u32 valid = kFullMask;
    if (w == nwords - 1 && (B & 31)) valid = (1u << (B & 31)) - 1;
    const u32 zeros = ~st->bad[w] & valid;
    if (zeros) {
      pos = w * 32 + 31 - __clz(zeros);
      break;
    }
  }
  const i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (j == 0) {
    st->rounds += 1;
    st->moves += pos + 1;
  }
  if (j > pos) return;
  const u64 key = top[j];
  const i32 v = (i32)(u32)key;
  const i32 g = INT_MAX - (i32)(u32)(key >> 32);
  const i32 s = part[v], d = target[v];
  const u32 w = (u32)vwgt[v];
  atomicAdd(&pw[d], w);
  atomicSub(&pw[s], w);
  part[v] = d;
  atomicAdd((unsigned long long*)&st->gain_sum, (unsigned long long)(i64)g);
  if (atomicExch(&updflag[v], 1) == 0) U[atomicAdd(&st->ucount, 1)] = v;
  for (i32 e = xadj[v]; e < xadj[v + 1]; ++e) {
    const i32 u = adjncy[e];
    if (atomicExch(&updflag[u], 1) == 0) U[atomicAdd(&st->ucount, 1)] = u;
  }
}

// ---------------------------------------------------------------------------
// Host drivers
// ---------------------------------------------------------------------------
static void launch_update(Handle& h, RefineCtx* c, const DevGraph& g, i32 grid_cap) {
  const i32 wpb = c->upd_warps;
  const size_t sm = (size_t)wpb * c->k * sizeof(u32);
  const u32 grid = std::max<u32>(1, std::min<u32>((u32)grid_cap, (u32)h.sm_count * 8));
  launch(k_update, grid, wpb * 32, sm, h.stream, g.xadj, g.adjncy, g.adjwgt, c->k, c->part[c->cur],
                                              c->bnd[c->cur], c->gain, c->target, c->updflag, c->inP,
                                              c->U, c->P[0], c->P[1], c->st);
  GKW_CHECK_LAUNCH();
}

static void reset_state(Handle& h, RefineCtx* c) {
  GKW_CUDA(cudaMemsetAsync(c->st, 0, sizeof(RoundState), h.stream));
}

void refine_project(Handle& h, RefineCtx* c, const DevGraph& fine, const i32* cmap, i32 nc) {
  (void)nc;
  reset_state(h, c);
  const i32 nxt = c->cur ^ 1;
  if (fine.n > 0) {
    launch(k_project, ceil_div(fine.n, 256), 256, 0, h.stream, fine.n, cmap, c->part[c->cur], c->bnd[c->cur],
                                                          c->part[nxt], c->bnd[nxt], c->gain, c->target,
                                                          c->updflag, c->inP, c->U, c->st);
    GKW_CHECK_LAUNCH();
  }
  c->cur = nxt;
  launch_update(h, c, fine, (i32)ceil_div(std::max(fine.n, 1), 8));
}

__global__ void k_build_lists(i32 n, const i32* __restrict__ updated, const i32* __restrict__ gain,
                              i32* __restrict__ updflag, i32* __restrict__ inP, i32* __restrict__ U,
                              i32* __restrict__ P0, RoundState* __restrict__ st) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 u = updated ? (updated[v] != 0) : 0;
  updflag[v] = u;
  if (u) U[atomicAdd(&st->ucount, 1)] = (i32)v;
  const i32 pos = gain[v] > 0;
  inP[v] = pos;
  if (pos) P0[atomicAdd(&st->pcount[0], 1)] = (i32)v;
}

void refine_update_flagged(Handle& h, RefineCtx* c, const DevGraph& g, const i32* d_updated) {
  reset_state(h, c);
  if (g.n > 0) {
    launch(k_build_lists, ceil_div(g.n, 256), 256, 0, h.stream, g.n, d_updated, c->gain, c->updflag, c->inP,
                                                           c->U, c->P[0], c->st);
    GKW_CHECK_LAUNCH();
  }
  launch_update(h, c, g, (i32)ceil_div(std::max(g.n, 1), 8));
}

RefineLevelStats refine_level(Handle& h, RefineCtx* c, const DevGraph& g, const RefineParams& p) {
  GKW_REQUIRE(p.move_cap >= 1 && p.move_cap <= c->cap, GKW_E_INVALID, "move_cap out of range");
  constexpr i32 kBatch = 8;
  const u32 cgrid = std::max<u32>(1, std::min<u32>(ceil_div(std::max(g.n, 1), 256), (u32)h.sm_count * 4));
  const u32 agrid = ceil_div(p.move_cap, 256);
  RoundState* hst = reinterpret_cast<RoundState*>(h.h_pinned);
  static_assert(sizeof(RoundState) <= 64 * sizeof(i64), "pinned staging too small");
  for (;;) {
    for (i32 r = 0; r < kBatch; ++r) {
      launch(k_candidates, cgrid, 256, 0, h.stream, g.xadj, g.adjncy, g.vwgt, c->part[c->cur], c->bnd[c->cur],
                                                c->gain, c->target, c->pw, p.maxw, c->inP, c->P[0], c->P[1],
                                                c->cands, c->st);
      launch(k_select, 1, 1024, 0, h.stream, c->cands, c->top, p.move_cap, c->st);
      launch(k_balance, c->k, 1024, 0, h.stream, c->top, c->part[c->cur], c->target, g.vwgt, c->pw, p.maxw, c->st);
      launch(k_apply, agrid, 256, 0, h.stream, c->top, g.xadj, g.adjncy, g.vwgt, c->part[c->cur], c->target,
                                           c->pw, c->updflag, c->U, c->st);
      launch_update(h, c, g, (i32)ceil_div(std::max(g.n, 1), 8));
    }
    GKW_CHECK_LAUNCH();
    GKW_CUDA(cudaMemcpyAsync(hst, c->st, sizeof(RoundState), cudaMemcpyDeviceToHost, h.stream));
    GKW_CUDA(cudaStreamSynchronize(h.stream));
    if (hst->done) break;
  }
  RefineLevelStats s;
  s.rounds = hst->rounds;
  s.moves = hst->moves;
  s.gain_sum = hst->gain_sum;
  return s;
}

// ---------------------------------------------------------------------------
// Metrics: exact weighted cut over u < v (uncoarsen.hpp:398-424) and part
// weights (cuda_check.hpp:61-73).
// ---------------------------------------------------------------------------
__global__ void k_cut_pw(i32 n, const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                         const i32* __restrict__ adjwgt, const i32* __restrict__ vwgt,
                         const i32* __restrict__ part, i32 k, unsigned long long* __restrict__ cut,
                         unsigned long long* __restrict__ pw, i32* __restrict__ bad) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  u64 c = 0;
  if (v < n) {
    const i32 p = part[v];
    if ((u32)p >= (u32)k) {
      atomicOr(bad, 1);
    } else {
      for (i32 e = xadj[v]; e < xadj[v + 1]; ++e) {
        const i32 u = adjncy[e];
        if (v < u && part[u] != p) c += (u32)adjwgt[e];
      }
      atomicAdd(&pw[p], (unsigned long long)(u32)vwgt[v]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFullMask, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(cut, (unsigned long long)c);
}

__global__ void k_check_parts(i32 n, const i32* __restrict__ part, i32 k, i32* __restrict__ bad) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n && (u32)part[v] >= (u32)k) atomicOr(bad, 1);
}

// Throws GKW_E_INVALID unless every part id is in [0, k) (per-phase entry
// points that take a caller's partition).
void check_parts(Handle& h, i32 n, const i32* part, i32 k) {
  if (n <= 0) return;
  Pool::Mark mk = h.scratch.mark();
  i32* bad = h.scratch.alloc_n<i32>(1);
  GKW_CUDA(cudaMemsetAsync(bad, 0, sizeof(i32), h.stream));
  launch(k_check_parts, ceil_div(n, 256), 256, 0, h.stream, n, part, k, bad);
  GKW_CHECK_LAUNCH();
  GKW_CUDA(cudaMemcpyAsync(h.h_pinned, bad, sizeof(i32), cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  const i32 b = *(i32*)h.h_pinned;
  h.scratch.release(mk);
  GKW_REQUIRE(b == 0, GKW_E_INVALID, "part id out of range [0, k)");
}

void compute_cut_pw(Handle& h, const DevGraph& g, const i32* part, i32 k, i64* d_cut, i64* d_pw) {
  GKW_CUDA(cudaMemsetAsync(d_cut, 0, sizeof(i64) * 2, h.stream));   // [0] cut, [1] bad-part flag
  GKW_CUDA(cudaMemsetAsync(d_pw, 0, sizeof(i64) * k, h.stream));
  if (g.n == 0) return;
  launch(k_cut_pw, ceil_div(g.n, 256), 256, 0, h.stream, g.n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, part, k,
         (unsigned long long*)d_cut, (unsigned long long*)d_pw, (i32*)(d_cut + 1));
  GKW_CHECK_LAUNCH();
}

}  // namespace gkw
