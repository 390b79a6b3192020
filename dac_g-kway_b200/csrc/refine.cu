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
  // balance rounds
  i32 bdone;
  i32 brounds;
  i64 bmoves;
  i32 lcount;
  i32 firstbad;
  i32 light;
  u32 epoch;
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
  // balance rounds: candidate mark (round epoch), destination, gain, list
  u32* bmark = nullptr;
  i32* btarget = nullptr;
  i32* bgain = nullptr;
  i32* blist = nullptr;
  u32* epoch = nullptr;   // never reset: the marks of earlier rounds stay stale
};

static void alloc_balance(Handle& h, Pool& P, RefineCtx* c, size_t n) {
  c->bmark = P.alloc_n<u32>(n);
  c->btarget = P.alloc_n<i32>(n);
  c->bgain = P.alloc_n<i32>(n);
  c->blist = P.alloc_n<i32>(n);
  c->epoch = P.alloc_n<u32>(1);
  GKW_CUDA(cudaMemsetAsync(c->bmark, 0, sizeof(u32) * n, h.stream));
  GKW_CUDA(cudaMemsetAsync(c->epoch, 0, sizeof(u32), h.stream));
}

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
  alloc_balance(h, P, c, n);
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
  alloc_balance(h, P, c, nn);
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
// (INT_MAX - gain fits in 32 bits for every int32 gain)
__device__ __forceinline__ u64 move_key(i32 gain, i32 v) {
  return ((u64)(u32)((i64)INT_MAX - (i64)gain) << 32) | (u32)v;
}
__device__ __forceinline__ i32 key_gain(u64 key) { return (i32)((i64)INT_MAX - (i64)(u32)(key >> 32)); }

static void reset_state(Handle& h, RefineCtx* c) {
  GKW_CUDA(cudaMemsetAsync(c->st, 0, sizeof(RoundState), h.stream));
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
  reset_state(h, c);
  GKW_CUDA(cudaMemsetAsync(c->pw, 0, sizeof(u32) * c->k, h.stream));
  if (g.n == 0) return;
  GKW_CUDA(cudaMemsetAsync(c->updflag, 0, sizeof(i32) * g.n, h.stream));
  GKW_CUDA(cudaMemsetAsync(c->inP, 0, sizeof(i32) * g.n, h.stream));
  GKW_CUDA(cudaMemsetAsync(c->gain, 0, sizeof(i32) * g.n, h.stream));
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
  if (st->done || st->bdone == 1) return;
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
                                                 i32 cap, RoundState* __restrict__ st, i32 balance_mode) {
  __shared__ u64 s[kSortMax];
  if (balance_mode ? st->bdone : st->done) return;
  const i32 cnt = st->ccount;
  __syncthreads();
  if (cnt == 0) {
    if (threadIdx.x == 0) {
      if (balance_mode) st->bdone = 1;
      else st->done = 1;
    }
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
    st->ucount = 0;
    if (balance_mode) {
      st->firstbad = B;
    } else {
      st->pcount[st->pcur] = 0;
      st->pcur ^= 1;
    }
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
  const i32 g = key_gain(key);
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
// Balance rounds (default mode; the reference has none -- an overweight part
// is only reported, cuda_check.hpp:105-113).  One round:
//   k_bal_prep    lightest part (ties: smaller id), new round epoch
//   k_bal_filter  boundary vertices of overweight parts -> list
//   k_bal_eval    per listed vertex (one warp): best neighbouring part with
//                 room by signed gain ed_q - id (ties: smaller q), else the
//                 lightest part if it has room; marks candidates
//   k_bal_emit    candidates without a smaller-id candidate neighbour -> keys
//   k_select      sort by (gain desc, id asc), cap
//   k_bal_check   per part: first move index whose source is no longer
//                 overweight before it or whose destination overflows
//   k_bal_apply   apply the prefix before that index, flag U
//   k_update      refresh gains of U
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool over_cap(u32 w, float cap) { return __uint2float_rn(w) > cap; }

__global__ void k_bal_prep(const u32* __restrict__ pw, i32 k, u32* __restrict__ epoch, RoundState* __restrict__ st) {
  __shared__ u64 s_best[32];
  if (st->bdone) return;
  u64 best = ~0ull;
  for (i32 p = threadIdx.x; p < k; p += blockDim.x) {
    const u64 key = ((u64)pw[p] << 32) | (u32)p;
    best = key < best ? key : best;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const u64 y = __shfl_xor_sync(kFullMask, best, o);
    best = y < best ? y : best;
  }
  if ((threadIdx.x & 31) == 0) s_best[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = s_best[w] < best ? s_best[w] : best;
    best = s_best[0] < best ? s_best[0] : best;
    st->light = (i32)(u32)best;
    st->epoch = ++(*epoch);
    st->lcount = 0;
  }
}

__global__ void k_bal_filter(i32 n, const i32* __restrict__ part, const i32* __restrict__ bnd,
                             const u32* __restrict__ pw, float cap, i32* __restrict__ list,
                             RoundState* __restrict__ st) {
  if (st->bdone) return;
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  if (bnd[v] && over_cap(pw[part[v]], cap)) list[atomicAdd(&st->lcount, 1)] = (i32)v;
}

__global__ void k_bal_eval(const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                           const i32* __restrict__ adjwgt, const i32* __restrict__ vwgt, i32 k,
                           const i32* __restrict__ part, const u32* __restrict__ pw, float cap,
                           const i32* __restrict__ list, u32* __restrict__ bmark, i32* __restrict__ btarget,
                           i32* __restrict__ bgain, RoundState* __restrict__ st) {
  extern __shared__ u32 acc_all[];
  if (st->bdone) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  u32* acc = acc_all + (size_t)wid * k;
  for (i32 q = lane; q < k; q += 32) acc[q] = 0;
  __syncwarp();
  const i32 nl = st->lcount;
  const u32 ep = st->epoch;
  const i32 light = st->light;
  const i64 nw = (i64)gridDim.x * wpb;
  for (i64 i = (i64)blockIdx.x * wpb + wid; i < nl; i += nw) {
    const i32 v = list[i];
    const i32 p = part[v];
    const u32 w = (u32)vwgt[v];
    const i32 beg = xadj[v], end = xadj[v + 1];
    for (i32 e = beg + lane; e < end; e += 32) atomicAdd(&acc[part[adjncy[e]]], (u32)adjwgt[e]);
    __syncwarp();
    const u32 id = acc[p];
    // best neighbouring part with room: max signed gain, then smaller part id
    u64 best = 0;
    for (i32 e = beg + lane; e < end; e += 32) {
      const i32 q = part[adjncy[e]];
      if (q == p || over_cap(pw[q] + w, cap)) continue;
      const i32 g = (i32)(acc[q] - id);
      const u64 key = (1ull << 63) | ((u64)((u32)g ^ 0x80000000u) << 31) | (u64)(0x7fffffffu - (u32)q);
      best = best > key ? best : key;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const u64 y = __shfl_xor_sync(kFullMask, best, o);
      best = best > y ? best : y;
    }
    i32 q_best = -1, g_best = 0;
    if (best) {
      q_best = (i32)(0x7fffffffu - (u32)(best & 0x7fffffffu));
      g_best = (i32)((u32)(best >> 31) ^ 0x80000000u);
    } else if (light != p && !over_cap(pw[light] + w, cap)) {
      q_best = light;
      g_best = (i32)(acc[light] - id);
    }
    if (lane == 0 && q_best >= 0) {
      bmark[v] = ep;
      btarget[v] = q_best;
      bgain[v] = g_best;
    }
    __syncwarp();
    for (i32 e = beg + lane; e < end; e += 32) acc[part[adjncy[e]]] = 0;
    __syncwarp();
  }
}

__global__ void k_bal_emit(const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                           const i32* __restrict__ list, const u32* __restrict__ bmark,
                           const i32* __restrict__ bgain, u64* __restrict__ cands, RoundState* __restrict__ st) {
  if (st->bdone) return;
  const i32 nl = st->lcount;
  const u32 ep = st->epoch;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += (i64)gridDim.x * blockDim.x) {
    const i32 v = list[i];
    if (bmark[v] != ep) continue;
    bool yield = false;
    for (i32 e = xadj[v]; e < xadj[v + 1]; ++e) {
      const i32 u = adjncy[e];
      if (u < v && bmark[u] == ep) { yield = true; break; }
    }
    if (!yield) cands[atomicAdd(&st->ccount, 1)] = move_key(bgain[v], v);
  }
}

// CTA p: exclusive prefix of weight leaving p, inclusive prefix of weight
// entering p, over the sorted moves; the first move that leaves p while p is
// no longer overweight, or enters p beyond cap, bounds the applied prefix.
__global__ void __launch_bounds__(1024) k_bal_check(const u64* __restrict__ top, const i32* __restrict__ part,
                                                    const i32* __restrict__ btarget, const i32* __restrict__ vwgt,
                                                    const u32* __restrict__ pw, float cap,
                                                    RoundState* __restrict__ st) {
  __shared__ i32 s_w[2][33];
  if (st->bdone) return;
  const i32 B = st->B;
  const i32 p = blockIdx.x;
  constexpr int IT = kMaxMoveCap / 1024;
  u32 o_e[IT], i_e[IT];
  bool is_src[IT], is_des[IT];
  u32 so = 0, si = 0;
#pragma unroll
  for (int i = 0; i < IT; ++i) {
    const i32 j = threadIdx.x * IT + i;
    o_e[i] = 0; i_e[i] = 0; is_src[i] = false; is_des[i] = false;
    if (j < B) {
      const i32 v = (i32)(u32)top[j];
      const u32 w = (u32)vwgt[v];
      if (part[v] == p) { o_e[i] = w; is_src[i] = true; }
      if (btarget[v] == p) { i_e[i] = w; is_des[i] = true; }
    }
    so += o_e[i];
    si += i_e[i];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  u32 io = so, ii = si;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 a = __shfl_up_sync(kFullMask, io, o);
    const u32 b = __shfl_up_sync(kFullMask, ii, o);
    if (lane >= o) { io += a; ii += b; }
  }
  if (lane == 31) { s_w[0][wid] = (i32)io; s_w[1][wid] = (i32)ii; }
  __syncthreads();
  if (wid == 0) {
    const bool in = lane < (int)(blockDim.x >> 5);
    u32 a = in ? (u32)s_w[0][lane] : 0, b = in ? (u32)s_w[1][lane] : 0;
    u32 ai = a, bi = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 x = __shfl_up_sync(kFullMask, ai, o);
      const u32 y = __shfl_up_sync(kFullMask, bi, o);
      if (lane >= o) { ai += x; bi += y; }
    }
    s_w[0][lane] = (i32)(ai - a);
    s_w[1][lane] = (i32)(bi - b);
  }
  __syncthreads();
  u32 out_ex = io - so + (u32)s_w[0][wid];   // weight leaving p before this thread's first move
  u32 in_in = ii - si + (u32)s_w[1][wid];
  const u32 base = pw[p];
  i32 first = INT_MAX;
#pragma unroll
  for (int i = 0; i < IT; ++i) {
    const i32 j = threadIdx.x * IT + i;
    in_in += i_e[i];
    if (j < B) {
      if (is_src[i] && !over_cap(base - out_ex, cap)) first = j < first ? j : first;
      if (is_des[i] && over_cap(base + in_in, cap)) first = j < first ? j : first;
    }
    out_ex += o_e[i];
  }
  if (first != INT_MAX) atomicMin(&st->firstbad, first);
}

__global__ void k_bal_apply(const u64* __restrict__ top, const i32* __restrict__ xadj,
                            const i32* __restrict__ adjncy, const i32* __restrict__ vwgt, i32* __restrict__ part,
                            const i32* __restrict__ btarget, u32* __restrict__ pw, i32* __restrict__ updflag,
                            i32* __restrict__ U, RoundState* __restrict__ st) {
  if (st->bdone) return;
  const i32 pos = st->firstbad - 1;
  const i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (j == 0) {
    st->brounds += 1;
    st->bmoves += pos + 1;
  }
  if (j > pos) return;
  const i32 v = (i32)(u32)top[j];
  const i32 s = part[v], d = btarget[v];
  const u32 w = (u32)vwgt[v];
  atomicAdd(&pw[d], w);
  atomicSub(&pw[s], w);
  part[v] = d;
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
  // every round applies >= 1 move of positive gain; 4n+64 rounds is far above
  // anything the cut allows in practice and bounds the host loop
  const i64 max_batches = (4 * (i64)g.n + 64) / kBatch + 1;
  for (i64 b = 0;; ++b) {
    GKW_REQUIRE(b < max_batches, GKW_E_INTERNAL, "refinement did not terminate");
    for (i32 r = 0; r < kBatch; ++r) {
      launch(k_candidates, cgrid, 256, 0, h.stream, g.xadj, g.adjncy, g.vwgt, c->part[c->cur], c->bnd[c->cur],
                                                c->gain, c->target, c->pw, p.maxw, c->inP, c->P[0], c->P[1],
                                                c->cands, c->st);
      launch(k_select, 1, 1024, 0, h.stream, c->cands, c->top, p.move_cap, c->st, 0);
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


RefineLevelStats balance_level(Handle& h, RefineCtx* c, const DevGraph& g, float cap, i32 move_cap) {
  GKW_REQUIRE(move_cap >= 1 && move_cap <= c->cap, GKW_E_INVALID, "move_cap out of range");
  RefineLevelStats s;
  if (g.n == 0) return s;
  constexpr i32 kBatch = 8;
  const i32 wpb = c->upd_warps;
  const size_t sm = (size_t)wpb * c->k * sizeof(u32);
  const u32 nb = ceil_div(g.n, 256);
  const u32 egrid = std::max<u32>(1, std::min<u32>(ceil_div(g.n, wpb), (u32)h.sm_count * 8));
  const u32 tgrid = std::max<u32>(1, std::min<u32>(nb, (u32)h.sm_count * 4));
  const u32 agrid = ceil_div(move_cap, 256);
  // the balance loop shares the round state with refinement: clear its part
  GKW_CUDA(cudaMemsetAsync(&c->st->bdone, 0, sizeof(i32), h.stream));
  GKW_CUDA(cudaMemsetAsync(&c->st->brounds, 0, sizeof(i32), h.stream));
  GKW_CUDA(cudaMemsetAsync(&c->st->bmoves, 0, sizeof(i64), h.stream));
  GKW_CUDA(cudaMemsetAsync(&c->st->ccount, 0, sizeof(i32), h.stream));
  RoundState* hst = reinterpret_cast<RoundState*>(h.h_pinned);
  const i64 max_batches = (4 * (i64)g.n + 64) / kBatch + 1;
  for (i64 b = 0;; ++b) {
    GKW_REQUIRE(b < max_batches, GKW_E_INTERNAL, "balancing did not terminate");
    for (i32 r = 0; r < kBatch; ++r) {
      launch(k_bal_prep, 1, 256, 0, h.stream, c->pw, c->k, c->epoch, c->st);
      launch(k_bal_filter, nb, 256, 0, h.stream, g.n, c->part[c->cur], c->bnd[c->cur], c->pw, cap, c->blist, c->st);
      launch(k_bal_eval, egrid, wpb * 32, sm, h.stream, g.xadj, g.adjncy, g.adjwgt, g.vwgt, c->k, c->part[c->cur],
             c->pw, cap, c->blist, c->bmark, c->btarget, c->bgain, c->st);
      launch(k_bal_emit, tgrid, 256, 0, h.stream, g.xadj, g.adjncy, c->blist, c->bmark, c->bgain, c->cands, c->st);
      launch(k_select, 1, 1024, 0, h.stream, c->cands, c->top, move_cap, c->st, 1);
      launch(k_bal_check, c->k, 1024, 0, h.stream, c->top, c->part[c->cur], c->btarget, g.vwgt, c->pw, cap, c->st);
      launch(k_bal_apply, agrid, 256, 0, h.stream, c->top, g.xadj, g.adjncy, g.vwgt, c->part[c->cur], c->btarget,
             c->pw, c->updflag, c->U, c->st);
      launch_update(h, c, g, (i32)ceil_div(std::max(g.n, 1), 8));
    }
    GKW_CHECK_LAUNCH();
    GKW_CUDA(cudaMemcpyAsync(hst, c->st, sizeof(RoundState), cudaMemcpyDeviceToHost, h.stream));
    GKW_CUDA(cudaStreamSynchronize(h.stream));
    if (hst->bdone) break;
  }
  s.rounds = hst->brounds;
  s.moves = hst->bmoves;
  // clear the flag so that the refinement rounds' gain updates run again
  GKW_CUDA(cudaMemsetAsync(&c->st->bdone, 0, sizeof(i32), h.stream));
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
