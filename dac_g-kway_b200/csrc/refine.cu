// Projection, balance rounds and independent-set refinement of one level
// (gkway/uncoarsen.hpp), as ONE persistent cooperative kernel per level.
//
// The reference runs each refinement round as ~9 launches plus 3 blocking
// device-to-host reads and scans every vertex of the level per round.  Here a
// level is one launch: all CTAs stay resident and step through the phases of
// every round, separated by a grid barrier, until no move is left.  A round
// only touches two short lists: P, the vertices whose gain is positive (the
// only ones that can move or block a neighbour), and U, the vertices whose
// gain must be recomputed (moved vertices and their neighbours).
//
// The grid barrier is a counter + generation word; a CTA that waits longer
// than kGridBarrierCycles sets the error word and every CTA leaves the kernel, so
// a fault in the round logic ends the launch with an error status instead of
// a hang.  Data written by other CTAs within the launch is read with
// ld.global.cg (L2, coherent) after the barrier.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "device_util.cuh"

namespace gkw {

static constexpr u32 kFullMask = 0xffffffffu;
constexpr i32 kSortMax = 4096;      // candidates sorted in one shared-memory pass
constexpr i32 kSelBins = 2048;      // histogram bins of the threshold search above kSortMax
constexpr i32 kMaxMoveCap = 2048;   // largest supported move cap
constexpr int kLevelThreads = 512;
// Level-kernel CTAs: one per gkw_tuning::level_verts_per_cta vertices of the
// level (default 512), at least level_min_ctas (default 32).  Every phase of a
// round is a chain of dependent loads per vertex, so even small levels run
// faster spread over many warps than on the cheaper barrier of a few CTAs.
constexpr i32 kGreedySmemParts = 4096;   // balance greedy pass: part weights in smem up to this k
constexpr i32 kGreedyWords = 3 * kMaxMoveCap + kGreedySmemParts;
static_assert((size_t)kGreedyWords * 4 >= (size_t)kSortMax * 8, "the sort's second buffer aliases the greedy region");
constexpr i32 kStatSlots = GKW_MAX_LEVELS + 2;
constexpr i32 kTraceCap = 4096;   // phase marks per level (diagnostic timeline)

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
  i32 pos;          // refinement: moves 0..pos of top are applied
  i32 bdone;
  i32 brounds;
  i64 bmoves;
  i32 lcount;
  i32 firstbad;
  i32 light;
  u32 epoch;
  u64 rows;   // adjacency entries read by the gain updates of the rounds
  i64 cand_sum;   // refinement candidates over the rounds (diagnostic)
  i32 needcheck;  // some part could exceed MAXW if every candidate moved (plain levels)
};


struct LevelStatsDev {
  i32 rounds, brounds;
  i64 moves, gain_sum, bmoves;
  i64 rows;
  i32 err;
  i32 pad;
  i64 cand_sum;
};

struct RefineCtx {
  i32 n_max = 0, k = 0, cap = 0;
  i32 kacc = 0;   // part-row length of the gain updates (k, or the largest k of a batch)
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
  u32* pwd = nullptr;    // part-weight changes of a round's moves, folded into pw by the gain update
  u32* pin = nullptr;    // weight the round's candidates would bring into each part
  i32* msrc = nullptr;   // source part of each candidate, taken before any move is applied
  u64* cinfo = nullptr;  // per candidate list entry: source part << 32 | destination part
  i32* cw = nullptr;     // per candidate list entry: vertex weight
  u32* risk = nullptr;   // per part: 1 if the round's candidates could push it over MAXW
  i32* pnet = nullptr;   // net weight change of each part if every candidate moved
  RoundState* st = nullptr;
  u32* bmark = nullptr;
  i32* btarget = nullptr;
  i32* bgain = nullptr;
  i32* blist = nullptr;
  u32* brem = nullptr;
  u32* epoch = nullptr;   // never reset: marks of earlier rounds stay stale
  GridBarrier* bar = nullptr;
  CountBarrier* cbar = nullptr;   // the refinement rounds' barriers (zeroed before each launch)
  i32* err = nullptr;
  LevelStatsDev* stats = nullptr;
  u64* trace = nullptr;     // GKW_TRACE=1: per-level phase timelines
  i32* trace_n = nullptr;
  i32 acc_warps = 16;
  size_t smem = 0;
  i32 grid = 0;
};

struct LevelArgs {
  i32 n, k;
  const i32* __restrict__ xadj;
  const i32* __restrict__ adjncy;
  const i32* __restrict__ adjwgt;
  const i32* __restrict__ vwgt;
  float maxw, bcap;
  i32 move_cap;
  i32 flags;
  i64 max_rounds;
  const i32* cmap;       // projection source
  const i32* part_c;
  const i32* bnd_c;
  const i32* updated_in;
  i32 *part, *bnd, *gain, *target, *updflag, *inP, *U, *P0, *P1;
  u64 *cands, *top;
  u32* pw;
  u32* pwd;           // plain levels: refinement moves add their weight changes here
  u32* pin;           // plain levels: per-part inflow of the round's candidates
  i32* msrc;          // plain levels: source part of each candidate
  u64* cinfo;         // plain levels: (source << 32 | destination) of candidate list entry i
  i32* cw;            // plain levels: vertex weight of candidate list entry i
  u32* risk;          // plain levels: 1 if the round's candidates could push the part over MAXW
  i32* pnet;          // plain levels: net weight change of each part over all candidates
  RoundState* st;
  u32* bmark;
  i32 *btarget, *bgain, *blist;
  u32* brem;          // part weights of the balance greedy pass when k > kGreedySmemParts
  u32* epoch;
  GridBarrier* bar;
  CountBarrier* cbar;   // plain levels' refinement rounds: barriers that sum the list appends
  i32* err;
  LevelStatsDev* stat_slot;
  i32 acc_warps;
  i32 upd_lanes;     // lanes per vertex of the first gain pass (8, 16, or 32: a warp)
  u64* trace;        // optional phase timeline: (phase id << 56) | globaltimer ns
  i32 trace_cap;
  i32* trace_n;
  // A batched level is the disjoint union of G independent graphs (batch.cu).
  // Part ids are global (graph g owns [gpbase[g], gpbase[g] + gk[g])), caps
  // are per part, and everything a round decides per graph -- the candidate
  // order, the move cap, the balanced prefix, the lightest part, the end of
  // the rounds -- is decided per graph, so each graph moves exactly as it
  // would alone.
  i32 batch;
  i32 G;
  i32 kacc;             // length of the per-warp part rows (largest k of a graph)
  const i32* gid;       // graph of each vertex
  const i32* gvbase;    // [G + 1] vertex offsets of the graphs at this level
  const i32* gpbase;    // [G] first part of each graph
  const i32* gk;        // [G] parts of each graph
  const i32* gflags;    // [G] bit 0: refinement rounds at this level, bit 1: balance rounds,
                        // bit 2: the graph's coarsest level (it enters with its initial parts)
  const i32* part_init; // entering graphs: cmap[v] = -(1 + i) names entry i of these
  const i32* bnd_init;
  const float* pmaxw;   // [parts] MAXW of each part
  const float* pbcap;   // [parts] balance cap of each part
  i32* gcc;             // [G] candidate counts; graph g's candidates at cands[gvbase[g]..]
  i32* glight;          // [G] lightest part of each graph (balance rounds)
  i32* mcount;          // moves in the flat move list top[]
  i32* anyf;            // [3] rotating flags: some graph had candidates / an overweight part
};

enum : i32 { LF_PROJECT = 1, LF_LISTS = 2, LF_UPDATE = 4, LF_BALANCE = 8, LF_REFINE = 16 };

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ i32 ldc(const i32* p) { return __ldcg(p); }
__device__ __forceinline__ u32 ldc(const u32* p) { return __ldcg(p); }
__device__ __forceinline__ u64 ldc(const u64* p) {
  return (u64)__ldcg(reinterpret_cast<const unsigned long long*>(p));
}
__device__ __forceinline__ i64 ldc(const i64* p) { return (i64)__ldcg(reinterpret_cast<const long long*>(p)); }

// uncoarsen.hpp:10-21 (is_valid_move): (float)(u32)(dest + vwgt) > MAXW is invalid
__device__ __forceinline__ bool valid_move(u32 dest_w, u32 vw, float maxw) {
  return !(__uint2float_rn(dest_w + vw) > maxw);
}
__device__ __forceinline__ bool over_cap(u32 w, float cap) { return __uint2float_rn(w) > cap; }

// per-graph values of a batched level (plain levels: one graph, part base 0)
__device__ __forceinline__ i32 part_base_of(const LevelArgs& a, i32 v) {
  return a.batch ? __ldg(a.gpbase + __ldg(a.gid + v)) : 0;
}
__device__ __forceinline__ float maxw_of(const LevelArgs& a, i32 part) {
  return a.batch ? __ldg(a.pmaxw + part) : a.maxw;
}
__device__ __forceinline__ float bcap_of(const LevelArgs& a, i32 part) {
  return a.batch ? __ldg(a.pbcap + part) : a.bcap;
}
__device__ __forceinline__ bool graph_flag(const LevelArgs& a, i32 v, i32 bit) {
  return !a.batch || ((__ldg(a.gflags + __ldg(a.gid + v)) >> bit) & 1);
}

// candidate key: ascending order = gain descending, vertex id ascending
// (INT_MAX - gain fits in 32 bits for every int32 gain)
__device__ __forceinline__ u64 move_key(i32 gain, i32 v) {
  return ((u64)(u32)((i64)INT_MAX - (i64)gain) << 32) | (u32)v;
}
__device__ __forceinline__ i32 key_gain(u64 key) { return (i32)((i64)INT_MAX - (i64)(u32)(key >> 32)); }

// Warp-aggregated append: every lane of the warp calls it together.
__device__ __forceinline__ void warp_append(bool pred, i32 val, i32* list, i32* counter) {
  const u32 mask = __ballot_sync(kFullMask, pred);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  i32 base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(mask));
  base = __shfl_sync(kFullMask, base, leader);
  if (pred) list[base + __popc(mask & ((1u << lane) - 1))] = val;
}
__device__ __forceinline__ void warp_append64(bool pred, u64 val, u64* list, i32* counter) {
  const u32 mask = __ballot_sync(kFullMask, pred);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  i32 base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(mask));
  base = __shfl_sync(kFullMask, base, leader);
  if (pred) list[base + __popc(mask & ((1u << lane) - 1))] = val;
}

__device__ __forceinline__ u64 globaltimer_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Phase timeline (diagnostic): block 0, thread 0 records each barrier exit.
__device__ __forceinline__ void trace_mark(const LevelArgs& a, u32 phase) {
  if (a.trace && blockIdx.x == 0 && threadIdx.x == 0) {
    const i32 i = *a.trace_n;
    if (i < a.trace_cap) {
      a.trace[i] = ((u64)phase << 56) | (globaltimer_ns() & 0x00ffffffffffffffull);
      *a.trace_n = i + 1;
    }
  }
}

// Block-aggregated append of one u64 per flagged thread: one global atomic
// per CTA.  Every thread of the block calls it (block-uniform control flow).
__device__ __forceinline__ void block_append64(bool pred, u64 val, u64* list, i32* counter, i32* s_cnt,
                                               i32* s_base) {
  if (threadIdx.x == 0) *s_cnt = 0;
  __syncthreads();
  const i32 local = pred ? atomicAdd(s_cnt, 1) : -1;
  __syncthreads();
  if (threadIdx.x == 0 && *s_cnt) *s_base = atomicAdd(counter, *s_cnt);
  __syncthreads();
  if (pred) list[*s_base + local] = val;
  __syncthreads();
}

__device__ __forceinline__ void block_append32(bool pred, i32 val, i32* list, i32* counter, i32* s_cnt,
                                               i32* s_base) {
  if (threadIdx.x == 0) *s_cnt = 0;
  __syncthreads();
  const u32 m = __ballot_sync(kFullMask, pred);   // one shared atomic per warp
  const int lane = threadIdx.x & 31;
  i32 wbase = 0;
  if (lane == 0 && m) wbase = atomicAdd(s_cnt, __popc(m));
  wbase = __shfl_sync(kFullMask, wbase, 0);
  __syncthreads();
  if (threadIdx.x == 0 && *s_cnt) *s_base = atomicAdd(counter, *s_cnt);
  __syncthreads();
  if (pred) list[*s_base + wbase + __popc(m & ((1u << lane) - 1))] = val;
  __syncthreads();
}

// U (or P) appends of one phase, staged per CTA in shared memory (one global
// atomic per CTA); entries beyond the stage go to the list directly.
constexpr i32 kUStage = 1024;
static_assert(kLevelThreads <= kUStage, "the projection's U stage holds at least one chunk");
struct UStage {
  i32 buf[kUStage];
  i32 cnt;
  i32 base;
};
__device__ __forceinline__ void ustage_push(UStage& S, i32 x, i32* U, i32* ucount) {
  const i32 idx = atomicAdd(&S.cnt, 1);
  if (idx < kUStage) S.buf[idx] = x;
  else U[atomicAdd(ucount, 1)] = x;
}
__device__ __forceinline__ void ustage_flush(UStage& S, i32* U, i32* ucount) {
  __syncthreads();
  const i32 c = S.cnt < kUStage ? S.cnt : kUStage;
  if (threadIdx.x == 0 && c) S.base = atomicAdd(ucount, c);
  __syncthreads();
  for (i32 t = threadIdx.x; t < c; t += blockDim.x) U[S.base + t] = S.buf[t];
}

// Maximum of a 64-bit key over a converged warp in two 32-bit reductions
// (redux.sync): the largest high half, then the largest low half among the
// lanes that hold it.
__device__ __forceinline__ u64 warp_max_key(u64 x) {
  const u32 hi = (u32)(x >> 32), lo = (u32)x;
  const u32 mh = __reduce_max_sync(kFullMask, hi);
  const u32 ml = __reduce_max_sync(kFullMask, hi == mh ? lo : 0u);
  return ((u64)mh << 32) | ml;
}

// ---------------------------------------------------------------------------
// Phases.  `base` of every grid-stride loop is warp-uniform so that warp
// collectives run converged.
// ---------------------------------------------------------------------------

// Projection (uncoarsen.hpp:325-356, expand_partition): part and boundary
// inherited from the coarse vertex, gain 0, target = part, boundary vertices
// flagged for the gain update.
// U appends are staged per CTA in shared memory and flushed with one global
// atomic per half-full stage (a million-vertex level would otherwise
// serialise tens of thousands of atomics on the counter), with one block
// barrier per chunk of vertices.
__device__ void ph_project(const LevelArgs& a, UStage& S) {
  if (threadIdx.x == 0) S.cnt = 0;
  __syncthreads();
  const i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 b0 = (i64)blockIdx.x * blockDim.x; b0 < a.n; b0 += stride) {   // block-uniform trip count
    const i64 v = b0 + threadIdx.x;
    if (v < a.n) {
      const i32 c = a.cmap[v];
      i32 p, bc;
      bool enter = false;
      if (a.batch && c < 0) {   // the graph's coarsest level: its initial parts, no gain pass
        p = a.part_init[-1 - c];
        bc = a.bnd_init[-1 - c];
        enter = true;
      } else {
        p = a.part_c[c];
        bc = a.bnd_c[c];
      }
      a.part[v] = p;
      a.bnd[v] = bc;
      a.gain[v] = 0;
      a.target[v] = p;
      a.inP[v] = 0;
      const bool b = bc != 0 && !enter && (!a.batch || __ldg(a.gflags + __ldg(a.gid + v)) != 0);
      a.updflag[v] = b ? 1 : 0;
      if (b) S.buf[atomicAdd(&S.cnt, 1)] = (i32)v;   // room: flushed below once half full
    }
    __syncthreads();
    if (S.cnt > kUStage - (i32)blockDim.x) {   // block-uniform
      if (threadIdx.x == 0) S.base = atomicAdd(&a.st->ucount, S.cnt);
      __syncthreads();
      for (i32 t = threadIdx.x; t < S.cnt; t += blockDim.x) a.U[S.base + t] = S.buf[t];
      __syncthreads();
      if (threadIdx.x == 0) S.cnt = 0;
      __syncthreads();
    }
  }
  ustage_flush(S, a.U, &a.st->ucount);
}

// U from the caller's flags, P from the current gains (per-phase entry points).
__device__ void ph_lists(const LevelArgs& a) {
  const int lane = threadIdx.x & 31;
  const i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 base = (i64)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < a.n; base += stride) {
    const i64 v = base + lane;
    bool u = false, pos = false;
    if (v < a.n) {
      u = a.updated_in ? (a.updated_in[v] != 0) : false;
      pos = a.gain[v] > 0;
      a.updflag[v] = u ? 1 : 0;
      a.inP[v] = pos ? 1 : 0;
    }
    warp_append(u, (i32)v, a.U, &a.st->ucount);
    warp_append(pos, (i32)v, a.P0, &a.st->pcount[0]);
  }
}

// Gain update (uncoarsen.hpp:175-237, update_vertex_info + calculate_gain).
// One warp per vertex of U, per-part connection weights in a per-warp shared
// row of k words (only touched entries are cleared afterwards).  The best part
// is the max of the UNSIGNED value (ed - id) over neighbouring parts other
// than the own part, ties to the smaller part id, taken only if that value is
// > 0 -- the reference's `if (gain > max_gain)` with an unsigned max_gain.
// Vertices whose new gain is positive join P.
// `count`: add the row lengths read to the level's entry counter (the update
// passes of the rounds; the first pass of a level is counted as a full pass).
__device__ void ph_update_rows(const LevelArgs& a, u32* acc_all, bool count, UStage& S, i32 nU_known) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (wid >= a.acc_warps) return;
  u32* acc = acc_all + (size_t)wid * a.kacc;
  RoundState* st = a.st;
  const i32 nU = nU_known >= 0 ? nU_known : ldc(&st->ucount);
  i32* Pout = a.P0;          // P is never compacted within a level: entries whose
  i32* pcount = &st->pcount[0];   // gain dropped stay and are skipped by gain
  const i64 nw = (i64)gridDim.x * a.acc_warps;
  unsigned long long rows = 0;
  for (i64 i = (i64)blockIdx.x * a.acc_warps + wid; i < nU; i += nw) {
    const i32 v = ldc(a.U + i);
    const i32 p = ldc(a.part + v);
    const i32 wasP = ldc(a.inP + v);   // U holds v once: no other warp writes inP[v] in this phase
    const i32 pb = part_base_of(a, v);   // rows are indexed by the graph's own part ids
    u32* accb = acc - pb;
    const i32 beg = a.xadj[v], end = a.xadj[v + 1];
    rows += (unsigned long long)(end - beg);
    u32 g = 0, q_best = (u32)p;
    bool b;
    if (end - beg <= 64) {   // warp-uniform: the row's part ids stay in registers (one load chain)
      const i32 e0 = beg + lane, e1 = e0 + 32;
      const bool h0 = e0 < end, h1 = e1 < end;
      const i32 u0 = h0 ? a.adjncy[e0] : 0, u1 = h1 ? a.adjncy[e1] : 0;
      const u32 w0 = h0 ? (u32)a.adjwgt[e0] : 0u, w1 = h1 ? (u32)a.adjwgt[e1] : 0u;
      const i32 q0 = h0 ? ldc(a.part + u0) : p, q1 = h1 ? ldc(a.part + u1) : p;
      if (h0) atomicAdd(&accb[q0], w0);
      if (h1) atomicAdd(&accb[q1], w1);
      b = __any_sync(kFullMask, q0 != p || q1 != p);
      __syncwarp();
      if (b) {
        const u32 id = accb[p];
        u64 best = 0;
        if (q0 != p) best = ((u64)(accb[q0] - id) << 32) | (u32)(~(u32)q0);
        if (q1 != p) {
          const u64 key = ((u64)(accb[q1] - id) << 32) | (u32)(~(u32)q1);
          best = best > key ? best : key;
        }
        best = warp_max_key(best);
        const u32 gb = (u32)(best >> 32);
        if (gb > 0) { g = gb; q_best = ~(u32)best; }
      }
      if (lane == 0) {
        a.updflag[v] = 0;
        a.bnd[v] = b ? 1 : 0;
        a.gain[v] = (i32)g;
        a.target[v] = (i32)q_best;
        if ((i32)g > 0 && !wasP) {
          a.inP[v] = 1;
          ustage_push(S, v, Pout, pcount);
        }
      }
      __syncwarp();
      if (h0) accb[q0] = 0;
      if (h1) accb[q1] = 0;
      __syncwarp();
      continue;
    }
    bool bl = false;
    for (i32 e = beg + lane; e < end; e += 32) {
      const i32 q = ldc(a.part + a.adjncy[e]);
      atomicAdd(&accb[q], (u32)a.adjwgt[e]);
      bl |= (q != p);
    }
    b = __any_sync(kFullMask, bl);
    __syncwarp();
    if (b) {
      const u32 id = accb[p];
      u64 best = 0;
      for (i32 e = beg + lane; e < end; e += 32) {
        const i32 q = ldc(a.part + a.adjncy[e]);
        if (q != p) {
          const u64 key = ((u64)(accb[q] - id) << 32) | (u32)(~(u32)q);
          best = best > key ? best : key;
        }
      }
      best = warp_max_key(best);
      const u32 gb = (u32)(best >> 32);
      if (gb > 0) { g = gb; q_best = ~(u32)best; }
    }
    if (lane == 0) {
      a.updflag[v] = 0;
      a.bnd[v] = b ? 1 : 0;
      a.gain[v] = (i32)g;
      a.target[v] = (i32)q_best;
      if ((i32)g > 0 && !wasP) {
        a.inP[v] = 1;
        ustage_push(S, v, Pout, pcount);
      }
    }
    __syncwarp();
    for (i32 e = beg + lane; e < end; e += 32) accb[ldc(a.part + a.adjncy[e])] = 0;
    __syncwarp();
  }
  if (count && lane == 0 && rows) atomicAdd(reinterpret_cast<unsigned long long*>(&st->rows), rows);
}

// P appends are staged per CTA in shared memory (S) and flushed with one
// global atomic; every thread of the CTA calls this.
// Returns (thread 0) the CTA's appends to P.  nU_known: the length of U when
// the caller has it (from grid_barrier_count), else -1.
__device__ u32 ph_update(const LevelArgs& a, u32* acc_all, bool count, UStage& S, i32 nU_known = -1) {
  if (threadIdx.x == 0) S.cnt = 0;
  __syncthreads();
  ph_update_rows(a, acc_all, count, S, nU_known);
  ustage_flush(S, a.P0, &a.st->pcount[0]);
  __syncthreads();
  return (u32)S.cnt;
}

// The first gain pass of a level (every boundary vertex of U) on a graph of
// short rows: G lanes per vertex instead of a warp, so 32/G vertices' load
// chains run at once in each warp -- the same rule as ph_update_rows per
// vertex.  Each group's connection row (kacc words) lies in `rows`, the
// level kernel's sort and greedy buffers (free during an update phase); the
// rows are zeroed here and every vertex clears the entries it touched.
template <int G>
__device__ void ph_update_first_groups(const LevelArgs& a, u32* rows, UStage& S) {
  constexpr int kGpw = 32 / G;   // groups per warp
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int sub = lane & (G - 1), grp = lane / G;
  const u32 gmask = (G == 32 ? kFullMask : ((1u << G) - 1u)) << (grp * G);
  const i32 ngrp = (i32)(blockDim.x / G);
  for (i32 q = threadIdx.x; q < ngrp * a.kacc; q += blockDim.x) rows[q] = 0;
  if (threadIdx.x == 0) S.cnt = 0;
  __syncthreads();
  u32* acc = rows + (size_t)(wid * kGpw + grp) * a.kacc;
  RoundState* st = a.st;
  const i32 nU = ldc(&st->ucount);
  i32* Pout = a.P0;
  i32* pcount = &st->pcount[0];
  const i64 step = (i64)gridDim.x * ngrp;
  // warp-uniform trip count: a warp's groups take vertices base .. base + kGpw - 1
  for (i64 base = ((i64)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / G; base < nU; base += step) {
    const i64 i = base + grp;
    const bool act = i < nU;
    i32 v = 0, p = 0, wasP = 1, beg = 0, end = 0;
    if (act) {
      v = ldc(a.U + i);
      p = ldc(a.part + v);
      wasP = ldc(a.inP + v);
      beg = a.xadj[v];
      end = a.xadj[v + 1];
    }
    u32* accb = acc - (act ? part_base_of(a, v) : 0);   // rows are indexed by the graph's own part ids
    // entries sub and sub + G keep their part ids in registers; longer rows reload
    const i32 e0 = beg + sub, e1 = e0 + G;
    const bool h0 = e0 < end, h1 = e1 < end;
    const i32 q0 = h0 ? ldc(a.part + a.adjncy[e0]) : p, q1 = h1 ? ldc(a.part + a.adjncy[e1]) : p;
    bool bl = q0 != p || q1 != p;
    if (h0) atomicAdd(&accb[q0], (u32)a.adjwgt[e0]);
    if (h1) atomicAdd(&accb[q1], (u32)a.adjwgt[e1]);
    for (i32 e = e1 + G; e < end; e += G) {
      const i32 q = ldc(a.part + a.adjncy[e]);
      atomicAdd(&accb[q], (u32)a.adjwgt[e]);
      bl |= q != p;
    }
    const bool b = (__ballot_sync(kFullMask, bl) & gmask) != 0;
    __syncwarp();
    u64 best = 0;
    if (b) {
      const u32 id = accb[p];
      if (q0 != p) best = ((u64)(accb[q0] - id) << 32) | (u32)(~(u32)q0);
      if (q1 != p) {
        const u64 key = ((u64)(accb[q1] - id) << 32) | (u32)(~(u32)q1);
        best = best > key ? best : key;
      }
      for (i32 e = e1 + G; e < end; e += G) {
        const i32 q = ldc(a.part + a.adjncy[e]);
        if (q != p) {
          const u64 key = ((u64)(accb[q] - id) << 32) | (u32)(~(u32)q);
          best = best > key ? best : key;
        }
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const u64 ot = __shfl_xor_sync(kFullMask, best, o, G);
      best = best > ot ? best : ot;
    }
    if (act && sub == 0) {
      u32 g = 0, q_best = (u32)p;
      const u32 gb = (u32)(best >> 32);
      if (b && gb > 0) { g = gb; q_best = ~(u32)best; }
      a.updflag[v] = 0;
      a.bnd[v] = b ? 1 : 0;
      a.gain[v] = (i32)g;
      a.target[v] = (i32)q_best;
      if ((i32)g > 0 && !wasP) {
        a.inP[v] = 1;
        ustage_push(S, v, Pout, pcount);
      }
    }
    __syncwarp();
    if (h0) accb[q0] = 0;
    if (h1) accb[q1] = 0;
    for (i32 e = e1 + G; e < end; e += G) accb[ldc(a.part + a.adjncy[e])] = 0;
    __syncwarp();
  }
  ustage_flush(S, a.P0, &a.st->pcount[0]);
  __syncthreads();
}

// The first gain pass: groups of upd_lanes lanes per vertex, or a warp.
__device__ void ph_update_first(const LevelArgs& a, u32* acc_all, u32* rows, UStage& S) {
  if (a.upd_lanes == 8) ph_update_first_groups<8>(a, rows, S);
  else if (a.upd_lanes == 16) ph_update_first_groups<16>(a, rows, S);
  else ph_update(a, acc_all, false, S);
}


// Move candidates (uncoarsen.hpp:111-173, create_independent_move_buffer):
// boundary, gain > 0, a valid destination by weight, and no neighbour with a
// smaller id that is itself positive and valid.  P is compacted on the way.
// Plain levels also keep each candidate's source part (msrc) and add its
// weight to the inflow bound of its destination (pin): if no part could pass
// MAXW even with every candidate moved in, every prefix of the sorted moves
// is balanced and the select phase needs neither the sort nor the check;
// otherwise the parts that could pass it are flagged in risk.
// Returns (thread 0) the CTA's appended candidates (plain levels).  nP_known:
// the length of P when the caller has it, else -1.
__device__ u32 ph_candidates(const LevelArgs& a, i32* s_cnt, i32* s_base, u32* s_pwc, i32 nP_known = -1) {
  RoundState* st = a.st;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (a.batch) *a.mcount = 0;   // the round's moves
    else st->ucount = 0;          // U was consumed by the last gain update
  }
  const int lane = threadIdx.x & 31;
  // plain levels: the part weights (no move changes them during this phase)
  // in shared memory, which takes two dependent global loads off each
  // candidate's chain
  const bool pwc = !a.batch && a.k <= kGreedyWords;   // block-uniform
  if (pwc) {
    for (i32 q = threadIdx.x; q < a.k; q += blockDim.x) s_pwc[q] = ldc(a.pw + q);
    __syncthreads();
  }
  auto pw_of = [&](i32 q) -> u32 { return pwc ? s_pwc[q] : ldc(a.pw + q); };
  const i32 nP = nP_known >= 0 ? nP_known : ldc(&st->pcount[0]);
  u32 mine = 0;
  // entry r*32*W + lane*W + w goes to warp w, lane `lane`: the entries of a
  // round spread over all warps, so each warp checks at most a few of them
  const i64 W = (i64)gridDim.x * (blockDim.x >> 5);
  const i64 gw = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (i64 r0 = 0; r0 < nP; r0 += 32 * W) {
    const i64 i = r0 + lane * W + gw;
    bool check = false;
    i32 v = 0, g = 0, t = 0, p = 0, xb = 0, xe = 0;
    u32 pwt = 0, vw = 0;
    if (i < nP) {
      v = ldc(a.P0 + i);
      g = ldc(a.gain + v);
      const i32 bv = ldc(a.bnd + v);
      t = ldc(a.target + v);   // loads issued together; used only when v is positive
      vw = (u32)a.vwgt[v];
      xb = a.xadj[v];
      xe = a.xadj[v + 1];
      if (!a.batch) p = ldc(a.part + v);
      if (g > 0 && bv && graph_flag(a, v, 0)) {   // batched: graphs that refine here
        pwt = pw_of(t);
        check = valid_move(pwt, vw, maxw_of(a, t));
      }
    }
    // independent-set test, one candidate at a time, neighbours across lanes
    u32 pend = __ballot_sync(kFullMask, check);
    bool cand = false;
    while (pend) {
      const int src = __ffs(pend) - 1;
      pend &= pend - 1;
      const i32 cv = __shfl_sync(kFullMask, v, src);
      const i32 beg = __shfl_sync(kFullMask, xb, src), end = __shfl_sync(kFullMask, xe, src);
      bool blocked = false;
      for (i32 e = beg + lane; e < end && !blocked; e += 32) {
        const i32 u = a.adjncy[e];
        if (u < cv) {
          const i32 gu = ldc(a.gain + u), tu = ldc(a.target + u);   // issued together
          const u32 vu = (u32)a.vwgt[u];
          if (gu > 0) blocked = valid_move(pw_of(tu), vu, maxw_of(a, tu));
        }
      }
      const bool any_blocked = __any_sync(kFullMask, blocked);
      if (lane == src) cand = !any_blocked;
    }
    if (a.batch) {   // graph g's candidates go to cands[gvbase[g]..]
      if (cand) {
        const i32 gv = __ldg(a.gid + v);
        a.cands[__ldg(a.gvbase + gv) + atomicAdd(a.gcc + gv, 1)] = move_key(g, v);
      }
    } else {
      u32 before = 0;
      if (cand) {
        a.msrc[v] = p;
        before = atomicAdd(a.pin + t, vw);
        atomicAdd(a.pnet + t, (i32)vw);
        atomicSub(a.pnet + p, (i32)vw);
      }
      // CTA-aggregated append of the key with its source, destination and
      // weight (the balance check reads those by list position)
      if (threadIdx.x == 0) *s_cnt = 0;
      __syncthreads();
      const i32 local = cand ? atomicAdd(s_cnt, 1) : -1;
      __syncthreads();
      if (threadIdx.x == 0 && *s_cnt) {
        *s_base = atomicAdd(&st->ccount, *s_cnt);
        mine += (u32)*s_cnt;
      }
      __syncthreads();
      if (cand) {
        const i32 at = *s_base + local;
        a.cands[at] = move_key(g, v);
        a.cinfo[at] = ((u64)(u32)p << 32) | (u32)t;
        a.cw[at] = (i32)vw;
      }
      __syncthreads();
      // the final inflow of t is at least before + vw, and (float)(u32) is
      // monotone, so one add that passes MAXW shows the final sum passes it:
      // part t could pass MAXW, and the select phase checks it
      if (cand) {
        const u64 in = (u64)pwt + before + vw;
        if (in >> 32 || __uint2float_rn((u32)in) > a.maxw) {
          a.risk[t] = 1;
          st->needcheck = 1;
        }
      }
    }
  }  return mine;
}

// Sort the candidates by (gain desc, id asc) and keep the first min(cnt, cap)
// (uncoarsen.hpp:471-476 with move_request.hpp:36-41).  Block 0 only; more than
// kSortMax candidates are streamed through shared memory keeping the running
// top `cap`.  Resets the per-round counters.
// Block-wide exclusive scan of one u32 per thread (blockDim <= 1024).
__device__ __forceinline__ u32 block_exscan_u32(u32 x, u32* s_warp, u32& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  u32 inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 y = __shfl_up_sync(kFullMask, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    const u32 w = lane < nw ? s_warp[lane] : 0;
    u32 wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 y = __shfl_up_sync(kFullMask, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) s_warp[lane] = wi - w;
    if (lane == nw - 1) s_warp[32] = wi;
  }
  __syncthreads();
  const u32 r = inc - x + s_warp[wid];
  total = s_warp[32];
  __syncthreads();
  return r;
}

// Ascending sort of one u64 per lane across a warp (bitonic network).
__device__ __forceinline__ u64 warp_sort_u64(u64 x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const u64 y = __shfl_xor_sync(kFullMask, x, j);
      const bool up = (lane & k) == 0, lower = (lane & j) == 0;
      x = (lower == up) ? (x < y ? x : y) : (x > y ? x : y);
    }
  return x;
}

// Ascending block sort of s[0..P), P a power of two >= 32, by the whole
// block: every warp sorts runs of 32 in registers, then runs are merged
// pairwise (merge path: each thread finds where its outputs start by binary
// search, then merges them sequentially), ping-ponging between s and t.
// Returns the buffer holding the result.
__device__ u64* block_merge_sort(u64* s, u64* t, i32 P) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (i32 r = wid; r < (P >> 5); r += nw) s[r * 32 + lane] = warp_sort_u64(s[r * 32 + lane]);
  __syncthreads();
  u64* src = s;
  u64* dst = t;
  const i32 E = P > (i32)blockDim.x ? P / (i32)blockDim.x : 1;   // outputs per thread
  for (i32 L = 32; L < P; L <<= 1) {
    for (i32 o0 = threadIdx.x * E; o0 < P; o0 += blockDim.x * E) {
      const i32 b = o0 & ~(2 * L - 1);
      const i32 d = o0 - b;
      const u64* A = src + b;
      const u64* Bv = src + b + L;
      i32 lo = d > L ? d - L : 0, hi = d < L ? d : L;
      while (lo < hi) {
        const i32 mid = (lo + hi) >> 1;
        if (A[mid] <= Bv[d - 1 - mid]) lo = mid + 1;
        else hi = mid;
      }
      i32 i = lo, j = d - lo;
      for (i32 e = 0; e < E; ++e) {
        const bool takeA = j >= L || (i < L && A[i] <= Bv[j]);
        dst[o0 + e] = takeA ? A[i++] : Bv[j++];
      }
    }
    __syncthreads();
    u64* tmp = src;
    src = dst;
    dst = tmp;
  }
  return src;
}

// Largest balanced prefix index of the sorted moves s[0..B)
// (uncoarsen.hpp:239-288, find_mv_wgt_sequence + find_balance_sequence):
// D[p][j] = the weight moved into part p minus the weight moved out of it by
// moves 0..j; index j is balanced when every part with D[p][j] > 0 keeps
// (float)(pw[p] + D[p][j]) <= MAXW.  Each move is two events (part, index,
// +-w).  Sorted by (part, index), a segmented scan gives D after each event,
// and D holds until the part's next event; an event that breaks the cap marks
// that index range in a difference array.  The result is the largest
// unmarked index, 0 if every index is marked (move 0 is applied regardless,
// as in the reference: its -1 case is dead code, uncoarsen.hpp:481-488).
// Block-wide; t is a second buffer of kSortMax keys; s is overwritten.  The
// moves' source parts are read from srcp (the level's parts, or the
// candidates' parts taken before any move of the round was applied).
__device__ i32 refine_balanced_pos(const LevelArgs& a, u64* s, u64* t, i32 B, u32* s_warp, const i32* srcp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const i32 E = 2 * B;
  i32 P = 32;
  while (P < E) P <<= 1;
  for (i32 m = threadIdx.x; m < B; m += blockDim.x) {
    const i32 v = (i32)(u32)s[m];
    const i32 src = ldc(srcp + v), dst = ldc(a.target + v);
    const u32 w = (u32)a.vwgt[v];
    t[2 * m] = ((u64)(u32)dst << 43) | ((u64)m << 32) | w;
    t[2 * m + 1] = ((u64)(u32)src << 43) | ((u64)m << 32) | (u32)(0u - w);
  }
  for (i32 i = E + threadIdx.x; i < P; i += blockDim.x) t[i] = ~0ull;
  __syncthreads();
  u64* ev = block_merge_sort(t, s, P);
  i32* diff = reinterpret_cast<i32*>(ev == t ? s : t);   // B + 1 counters
  for (i32 j = threadIdx.x; j <= B; j += blockDim.x) diff[j] = 0;
  // segmented inclusive scan of the deltas, R consecutive events per thread
  constexpr i32 kMaxR = kSortMax / kLevelThreads;
  const i32 R = P > (i32)blockDim.x ? P / (i32)blockDim.x : 1;
  const i32 i0 = threadIdx.x * R;
  i32 val[kMaxR];
  u32 head_seen = 0;
  i32 acc = 0;
#pragma unroll
  for (i32 r = 0; r < kMaxR; ++r) {
    val[r] = 0;
    const i32 i = i0 + r;
    if (r < R && i < E) {
      const u64 e = ev[i];
      const bool head = i == 0 || (ev[i - 1] >> 43) != (e >> 43);
      const i32 d = (i32)(u32)e;
      acc = head ? d : acc + d;
      head_seen |= head ? (1u << r) : 0u;
      val[r] = acc;
    }
  }
  // exclusive scan over threads of (has head, running sum) pairs:
  // (f1, v1) + (f2, v2) = (f1 | f2, f2 ? v2 : v1 + v2)
  u32 f = head_seen ? 1u : 0u;
  i32 v = acc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 fo = __shfl_up_sync(kFullMask, f, o);
    const i32 vo = __shfl_up_sync(kFullMask, v, o);
    if (lane >= o) {
      if (!f) v += vo;
      f |= fo;
    }
  }
  u32 fe = __shfl_up_sync(kFullMask, f, 1);
  i32 ve = __shfl_up_sync(kFullMask, v, 1);
  if (lane == 0) {
    fe = 0;
    ve = 0;
  }
  if (lane == 31) {
    s_warp[wid] = (u32)v;
    s_warp[16 + wid] = f;
  }
  __syncthreads();
  if (wid == 0) {
    u32 wf = lane < nw ? s_warp[16 + lane] : 0u;
    i32 wv = lane < nw ? (i32)s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 fo = __shfl_up_sync(kFullMask, wf, o);
      const i32 vo = __shfl_up_sync(kFullMask, wv, o);
      if (lane >= o) {
        if (!wf) wv += vo;
        wf |= fo;
      }
    }
    // exclusive prefix of each warp
    u32 pf = __shfl_up_sync(kFullMask, wf, 1);
    i32 pv = __shfl_up_sync(kFullMask, wv, 1);
    if (lane == 0) {
      pf = 0;
      pv = 0;
    }
    __syncwarp();
    if (lane < nw) {
      s_warp[lane] = (u32)pv;
      s_warp[16 + lane] = pf;
    }
  }
  __syncthreads();
  {
    const u32 pf = s_warp[16 + wid];
    const i32 pv = (i32)s_warp[wid];
    const i32 carry = fe ? ve : pv + ve;   // running sum entering this thread
    (void)pf;
    const float maxw_plain = a.maxw;
#pragma unroll
    for (i32 r = 0; r < kMaxR; ++r) {
      const i32 i = i0 + r;
      if (r < R && i < E) {
        const bool before_head = (head_seen & ((2u << r) - 1u)) == 0;
        const i32 D = before_head ? val[r] + carry : val[r];
        const u64 e = ev[i];
        const u32 p = (u32)(e >> 43);
        if (D > 0 && __uint2float_rn((u32)D + ldc(a.pw + p)) > (a.batch ? __ldg(a.pmaxw + p) : maxw_plain)) {
          const i32 m = (i32)((e >> 32) & 0x7FFu);
          const i32 end = (i + 1 < E && (ev[i + 1] >> 43) == (e >> 43)) ? (i32)((ev[i + 1] >> 32) & 0x7FFu) : B;
          atomicAdd(&diff[m], 1);
          atomicAdd(&diff[end], -1);
        }
      }
    }
  }
  __syncthreads();
  // marks per index = prefix of diff; the largest index with none
  const i32 R2 = (B + (i32)blockDim.x - 1) / (i32)blockDim.x;
  const i32 j0 = threadIdx.x * R2;
  i32 loc = 0;
  for (i32 j = j0; j < j0 + R2 && j < B; ++j) loc += diff[j];
  u32 tot;
  i32 run = (i32)block_exscan_u32((u32)loc, s_warp, tot);
  i32 best = -1;
  for (i32 j = j0; j < j0 + R2 && j < B; ++j) {
    run += diff[j];
    if (run == 0) best = j;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const i32 y = __shfl_xor_sync(kFullMask, best, o);
    best = best > y ? best : y;
  }
  __syncthreads();
  if (lane == 0) s_warp[wid] = (u32)best;
  __syncthreads();
  i32 pos = -1;
  for (i32 w = 0; w < nw; ++w) pos = pos > (i32)s_warp[w] ? pos : (i32)s_warp[w];
  __syncthreads();
  return pos < 0 ? 0 : pos;
}

// Sort one candidate set cands[0..cnt) into s by (gain desc, id asc) and keep
// the first B = min(cnt, cap) (uncoarsen.hpp:471-476 with
// move_request.hpp:36-41); more than kSortMax candidates are streamed
// through shared memory keeping the running top `cap`.  Block-wide.
__device__ i32 select_sort(const LevelArgs& a, const u64* cands, i32 cnt, u64* s, i32* greedy) {
  const i32 cap = a.move_cap;
  const i32 B = cnt < cap ? cnt : cap;
  if (cnt <= kSortMax) {
    i32 P = 32;
    while (P < cnt) P <<= 1;
    for (i32 i = threadIdx.x; i < P; i += blockDim.x) s[i] = i < cnt ? ldc(cands + i) : ~0ull;
    __syncthreads();
    // the greedy region is free until the greedy pass and holds kSortMax keys
    u64* t = reinterpret_cast<u64*>(greedy);
    if (block_merge_sort(s, t, P) == t) {
      for (i32 i = threadIdx.x; i < B; i += blockDim.x) s[i] = t[i];
      __syncthreads();
    }
  } else {
    // More than kSortMax candidates: narrow a key threshold T with
    // B <= #(keys <= T) <= kSortMax by histogram passes over the keys, then
    // sort the keys <= T.  Keys are distinct (one per vertex), so the first B
    // of that sort are the first B of all.
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    u32* hist = reinterpret_cast<u32*>(greedy);   // kSelBins counters (free until the sort below)
    __shared__ u64 s_mn[32], s_mx[32];
    __shared__ u64 s_lo, s_hi, s_T;
    __shared__ u32 s_warp[33];
    __shared__ i32 s_below, s_cum, s_bin, s_fill;
    u64 mn = ~0ull, mx = 0;
    for (i32 i = threadIdx.x; i < cnt; i += blockDim.x) {
      const u64 k = ldc(cands + i);
      mn = k < mn ? k : mn;
      mx = k > mx ? k : mx;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const u64 y = __shfl_xor_sync(kFullMask, mn, o), z = __shfl_xor_sync(kFullMask, mx, o);
      mn = y < mn ? y : mn;
      mx = z > mx ? z : mx;
    }
    if (lane == 0) {
      s_mn[wid] = mn;
      s_mx[wid] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < nw; ++w) {
        mn = s_mn[w] < mn ? s_mn[w] : mn;
        mx = s_mx[w] > mx ? s_mx[w] : mx;
      }
      s_lo = mn;
      s_hi = mx;
      s_below = 0;
      s_T = mx;
    }
    __syncthreads();
    // every pass leaves one bin of the last: at least 11 bits fewer to
    // resolve, so 6 passes reach single keys
    for (i32 pass = 0; pass < 8; ++pass) {
      const u64 lo = s_lo, hi = s_hi;
      const i32 below = s_below;
      if (threadIdx.x == 0) {
        s_bin = 0;
        s_cum = below;
      }
      i32 sft = 0;
      while (((hi - lo) >> sft) >= (u64)kSelBins) ++sft;
      for (i32 b = threadIdx.x; b < kSelBins; b += blockDim.x) hist[b] = 0;
      __syncthreads();
      for (i32 base = 0; base < cnt; base += blockDim.x) {   // warp-uniform trip count
        const i32 i = base + threadIdx.x;
        u32 bin = 0xffffffffu;
        if (i < cnt) {
          const u64 k = ldc(cands + i);
          if (k >= lo && k <= hi) bin = (u32)((k - lo) >> sft);
        }
        const u32 same = __match_any_sync(kFullMask, bin);   // lanes of one bin add once
        if (bin != 0xffffffffu && lane == __ffs(same) - 1) atomicAdd(&hist[bin], (u32)__popc(same));
      }
      __syncthreads();
      // first bin where below + (inclusive count) reaches B
      constexpr i32 kPer = kSelBins / kLevelThreads;
      const i32 b0 = threadIdx.x * kPer;
      u32 loc = 0;
      for (i32 j = 0; j < kPer; ++j) loc += hist[b0 + j];
      u32 tot;
      u32 run = (u32)below + block_exscan_u32(loc, s_warp, tot);
      for (i32 j = 0; j < kPer; ++j) {
        const u32 h = hist[b0 + j];
        if (run < (u32)B && run + h >= (u32)B) {   // exactly one bin
          s_bin = b0 + j;
          s_cum = (i32)run;
        }
        run += h;
      }
      __syncthreads();
      const i32 b = s_bin, cum = s_cum;
      const u32 hb = hist[b];
      const bool last = (u64)b == ((hi - lo) >> sft);
      const u64 top = last ? hi : lo + ((u64)(b + 1) << sft) - 1;   // no overflow below the last bin
      __syncthreads();
      if ((i64)cum + hb <= (i64)kSortMax) {
        if (threadIdx.x == 0) s_T = top;
        __syncthreads();
        break;
      }
      if (threadIdx.x == 0) {
        s_lo = lo + ((u64)b << sft);
        s_hi = top;
        s_below = cum;
        s_T = top;
      }
      __syncthreads();
    }
    // keep the keys <= T
    if (threadIdx.x == 0) s_fill = 0;
    __syncthreads();
    const u64 T = s_T;
    for (i32 base = 0; base < cnt; base += blockDim.x) {
      const i32 i = base + threadIdx.x;
      u64 k = 0;
      bool keep = false;
      if (i < cnt) {
        k = ldc(cands + i);
        keep = k <= T;
      }
      const u32 m = __ballot_sync(kFullMask, keep);
      i32 at = 0;
      if (lane == 0 && m) at = atomicAdd(&s_fill, __popc(m));
      at = __shfl_sync(kFullMask, at, 0);
      const i32 pos = at + __popc(m & ((1u << lane) - 1));
      if (keep && pos < kSortMax) s[pos] = k;   // the threshold keeps at most kSortMax keys
    }
    __syncthreads();
    const i32 nk = s_fill < kSortMax ? s_fill : kSortMax;
    i32 P = 32;
    while (P < nk) P <<= 1;
    for (i32 i = nk + threadIdx.x; i < P; i += blockDim.x) s[i] = ~0ull;
    __syncthreads();
    u64* t = reinterpret_cast<u64*>(greedy);
    if (block_merge_sort(s, t, P) == t) {
      for (i32 i = threadIdx.x; i < B; i += blockDim.x) s[i] = t[i];
      __syncthreads();
    }
  }
  return B;
}

// Balance rounds: greedy pass in sorted order over s[0..B): take a move while
// its source is still overweight and its destination stays within the cap,
// skip the others.  Sources and destinations of one round are disjoint (a
// destination had room, a source did not), so one running weight per part
// suffices.  The kept moves are compacted to the front of s; returns their
// number.  Parts of the candidate set are [pb, pb + k).
__device__ i32 select_greedy(const LevelArgs& a, u64* s, i32* greedy, i32 B, i32 pb, i32 k) {
  __shared__ i32 s_nsel;
  i32* mv_src = greedy;
  i32* mv_des = mv_src + kMaxMoveCap;
  u32* mv_w = reinterpret_cast<u32*>(mv_des + kMaxMoveCap);
  u32* rem = (k <= kGreedySmemParts ? mv_w + kMaxMoveCap : a.brem + pb) - pb;
  for (i32 t = threadIdx.x; t < B; t += blockDim.x) {
    const i32 v = (i32)(u32)s[t];
    mv_src[t] = ldc(a.part + v);
    mv_des[t] = ldc(a.btarget + v);
    mv_w[t] = (u32)a.vwgt[v];
  }
  for (i32 q = threadIdx.x; q < k; q += blockDim.x) rem[pb + q] = ldc(a.pw + pb + q);
  __syncthreads();
  if (threadIdx.x == 0) {
    i32 nsel = 0;
    for (i32 t = 0; t < B; ++t) {
      const u32 w = mv_w[t];
      const i32 sp = mv_src[t], dp = mv_des[t];
      if (over_cap(rem[sp], bcap_of(a, sp)) && !over_cap(rem[dp] + w, bcap_of(a, dp))) {
        rem[sp] -= w;
        rem[dp] += w;
        s[nsel++] = s[t];
      }
    }
    s_nsel = nsel;
  }
  __syncthreads();
  const i32 nsel = s_nsel;
  __syncthreads();
  return nsel;
}

// Plain level, balance rounds: block 0 sorts the candidates and keeps the
// greedy selection.  Resets the per-round counters.
__device__ void ph_bal_select(const LevelArgs& a, u64* s, i32* greedy) {
  if (blockIdx.x != 0) return;
  RoundState* st = a.st;
  const i32 cnt = ldc(&st->ccount);
  if (cnt == 0) {
    if (threadIdx.x == 0) st->bdone = 1;
    return;
  }
  const i32 B = select_sort(a, a.cands, cnt, s, greedy);
  const i32 nsel = select_greedy(a, s, greedy, B, 0, a.k);
  for (i32 i = threadIdx.x; i < nsel; i += blockDim.x) a.top[i] = s[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    st->firstbad = nsel;   // moves 0..nsel-1 of top are applied
    st->ccount = 0;
    st->ucount = 0;
  }
}

// Batched level: CTA b selects for graphs b, b + grid, ... from their own
// candidate buckets and appends the moves it keeps to the flat list
// top[0..mcount).  A graph with candidates raises anyf[r % 3]; block 0
// clears anyf[(r + 1) % 3], last read two barriers ago.
__device__ void ph_select_batch(const LevelArgs& a, u64* s, i32* greedy, u32* s_warp, bool balance_mode, i64 r) {
  __shared__ i32 s_cnt, s_base;
  RoundState* st = a.st;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.anyf[(r + 1) % 3] = 0;
    st->ucount = 0;
  }
  for (i32 g = blockIdx.x; g < a.G; g += gridDim.x) {
    if (threadIdx.x == 0) {
      s_cnt = ldc(a.gcc + g);
      a.gcc[g] = 0;
    }
    __syncthreads();
    const i32 cnt = s_cnt;
    __syncthreads();
    if (cnt == 0) continue;   // block-uniform
    if (threadIdx.x == 0) atomicExch(a.anyf + r % 3, 1);
    u64* cg = a.cands + __ldg(a.gvbase + g);
    const i32 B = select_sort(a, cg, cnt, s, greedy);
    i32 keep;
    if (!balance_mode) {
      // the check below overwrites s: park the sorted moves in the bucket
      for (i32 i = threadIdx.x; i < B; i += blockDim.x) cg[i] = s[i];
      keep = refine_balanced_pos(a, s, reinterpret_cast<u64*>(greedy), B, s_warp, a.part) + 1;
    } else {
      keep = select_greedy(a, s, greedy, B, __ldg(a.gpbase + g), __ldg(a.gk + g));
      for (i32 i = threadIdx.x; i < keep; i += blockDim.x) cg[i] = s[i];
    }
    if (threadIdx.x == 0) s_base = atomicAdd(a.mcount, keep);
    __syncthreads();
    for (i32 i = threadIdx.x; i < keep; i += blockDim.x) a.top[s_base + i] = cg[i];
    __syncthreads();
  }
}


// One move, by one warp: v goes to its target; v and its neighbours are
// flagged for the gain update and appended to U (uncoarsen.hpp:290-323).
// The part-weight change goes to pwc: pw itself, or the round's delta array
// when other CTAs may still read pw in the same phase.
__device__ __forceinline__ void apply_move(const LevelArgs& a, UStage& S, u64 key, u32* pwc,
                                           unsigned long long* s_gsum) {
  const int lane = threadIdx.x & 31;
  const i32 v = (i32)(u32)key;
  const i32 s = ldc(a.part + v), d = ldc(a.target + v);
  const i32 beg = a.xadj[v], end = a.xadj[v + 1];   // issued beside the loads above
  if (lane == 0) {
    const u32 w = (u32)a.vwgt[v];
    atomicAdd(&pwc[d], w);
    atomicSub(&pwc[s], w);
    a.part[v] = d;
    atomicAdd(s_gsum, (unsigned long long)(i64)key_gain(key));
    if (atomicExch(&a.updflag[v], 1) == 0) ustage_push(S, v, a.U, &a.st->ucount);
  }
  for (i32 e = beg + lane; e < end; e += 32) {
    const i32 u = a.adjncy[e];
    if (atomicExch(&a.updflag[u], 1) == 0) ustage_push(S, u, a.U, &a.st->ucount);
  }
}

// Batched level: apply every graph's kept moves, top[0..mcount).  One warp
// per move.
__device__ void ph_apply_refine(const LevelArgs& a, UStage& S) {
  RoundState* st = a.st;
  const i32 pos = ldc(a.mcount) - 1;
  const i64 warp = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const i64 nwarps = ((i64)gridDim.x * blockDim.x) >> 5;
  __shared__ unsigned long long s_gsum;
  if (threadIdx.x == 0) {
    s_gsum = 0;
    S.cnt = 0;
  }
  __syncthreads();
  if (warp == 0 && (threadIdx.x & 31) == 0) {
    st->rounds += 1;
    st->moves += pos + 1;
  }
  for (i64 j = warp; j <= pos; j += nwarps) apply_move(a, S, ldc(a.top + j), a.pw, &s_gsum);
  ustage_flush(S, a.U, &st->ucount);
  if (threadIdx.x == 0 && s_gsum) atomicAdd((unsigned long long*)&st->gain_sum, s_gsum);
}

// Block-wide min (or max) of one u64 per thread; every thread gets the result.
template <bool kMax>
__device__ __forceinline__ u64 block_reduce_u64(u64 x, u64* s_tmp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const u64 y = __shfl_xor_sync(kFullMask, x, o);
    x = kMax ? (y > x ? y : x) : (y < x ? y : x);
  }
  __syncthreads();
  if (lane == 0) s_tmp[wid] = x;
  __syncthreads();
  u64 r = s_tmp[0];
  for (int w = 1; w < nw; ++w) r = kMax ? (s_tmp[w] > r ? s_tmp[w] : r) : (s_tmp[w] < r ? s_tmp[w] : r);
  return r;
}

constexpr i32 kRiskEvents = 1024;   // event limit of the at-risk balance check
constexpr i32 kRiskParts = 1024;    // part limit of that check (k)
constexpr i32 kRiskCands = 1024;    // candidate limit of that check

// The balance check of a round whose candidates are all kept (cnt <= cap),
// without sorting the candidates.  Only parts flagged in risk can be over
// MAXW at any index (a part's running change D never exceeds its inflow
// bound), so only the moves into or out of those parts matter.
//  * Last index: the reference applies moves 0..pos for the LARGEST balanced
//    index pos (Q11), so when the last index is balanced every candidate
//    moves.  A flagged part's change at the last index is its net change
//    over all candidates (pnet).
//  * Otherwise each move into or out of a flagged part is an event (part,
//    key, +-w), the events are grouped by part (a counting sort), and a
//    part's D after one of its events is the sum of its events with keys up
//    to that key, which holds until the part's next event; an event with
//    D > 0 and (float)(pw + D) > MAXW marks the key range [key, next key of
//    the part) -- the index ranges the reference's table marks
//    (uncoarsen.hpp:239-288), in key order.  Every candidate key is tested
//    against the marked ranges, and the moves with key <= K* apply, K* = the
//    largest unmarked key, or the smallest key if all are marked (prefix 0
//    always counts as balanced, :481-488).
// All global loads come first and at once, from two halves of the CTA: warps
// 0-7 fetch the candidate list entries (key, source, destination, weight,
// written beside each other by the candidates phase), warps 8-15 every
// part's flag, net change and weight.  Everything after one block barrier is
// shared memory.  Returns false (block-uniform) when the last index is not
// balanced and k > kRiskParts, cnt > kRiskCands or the events exceed
// kRiskEvents; the caller then runs the check over all parts.
__device__ bool refine_check_risk(const LevelArgs& a, i32 cnt, u64* s, i32* greedy, u64* keep, u64* s_tmp,
                                  u32* s_warp, u64* kstar, i32* napplied) {
  __shared__ i32 s_ne, s_nbad, s_lastbad;
  constexpr i32 kHalf = kLevelThreads / 2;
  constexpr i32 kPerThread = kRiskCands / kHalf;   // candidates per loading thread
  static_assert(kRiskCands % kHalf == 0, "candidates split evenly over the loading threads");
  u64* ev_key = s + kMaxMoveCap;      // [kRiskEvents] events as found
  u64* gk = ev_key + kRiskEvents;     // [kRiskEvents] grouped by part
  u64* bad_lo = keep;                 // [kRiskEvents] marked key ranges [lo, hi)
  u64* bad_hi = keep + kRiskEvents;   // [kRiskEvents]
  i32* ev_b = greedy;                 // [kRiskEvents] part of each event
  i32* ev_d = ev_b + kRiskEvents;     // [kRiskEvents] weight change
  i32* gb = ev_d + kRiskEvents;       // grouped: part
  i32* gd = gb + kRiskEvents;         // grouped: weight change
  i32* bcnt = gd + kRiskEvents;       // [kRiskParts] events per part
  i32* boff = bcnt + kRiskParts;      // [kRiskParts] first grouped slot
  i32* bfill = boff + kRiskParts;     // [kRiskParts]
  i32* rpw = bfill + kRiskParts;      // [kRiskParts] part weight before the round
  i32* rflag = rpw + kRiskParts;      // [kRiskParts] part flagged in risk
  static_assert(4 * kRiskEvents + 5 * kRiskParts <= kGreedyWords, "check arrays fit the greedy region");
  static_assert(kMaxMoveCap + 2 * kRiskEvents <= kSortMax, "event keys fit the sort buffer");
  static_assert(kRiskCands <= kMaxMoveCap, "candidate keys fit the sort buffer");
  const i32 k = a.k;
  const bool small = k <= kRiskParts && cnt <= kRiskCands;   // block-uniform
  if (threadIdx.x == 0) {
    s_ne = 0;
    s_nbad = 0;
    s_lastbad = 0;
  }
  if (small)
    for (i32 b = threadIdx.x; b < k; b += blockDim.x) {
      bcnt[b] = 0;
      bfill[b] = 0;
    }
  __syncthreads();
  u64 key[kPerThread];
  i32 src[kPerThread], dst[kPerThread], w[kPerThread];
  if (threadIdx.x < kHalf) {
    if (small) {
#pragma unroll
      for (i32 q = 0; q < kPerThread; ++q) {
        const i32 i = threadIdx.x + q * kHalf;
        key[q] = ~0ull;
        src[q] = dst[q] = w[q] = 0;
        if (i < cnt) {
          key[q] = ldc(a.cands + i);
          const u64 inf = ldc(a.cinfo + i);
          w[q] = ldc(a.cw + i);
          src[q] = (i32)(u32)(inf >> 32);
          dst[q] = (i32)(u32)inf;
        }
      }
    }
  } else {
    bool bad = false;
    for (i32 p = threadIdx.x - kHalf; p < k; p += kHalf) {
      const u32 f = ldc(a.risk + p);
      const i32 d = ldc(a.pnet + p);
      const u32 pw = ldc(a.pw + p);
      if (small) {
        rflag[p] = (i32)f;
        rpw[p] = (i32)pw;
      }
      if (f && d > 0 && __uint2float_rn((u32)d + pw) > a.maxw) bad = true;
    }
    if (bad) s_lastbad = 1;
  }
  __syncthreads();
  if (!s_lastbad) {   // block-uniform: the last index is balanced, every candidate moves
    *kstar = ~0ull;
    *napplied = cnt;
    return true;
  }
  if (!small) return false;
  u64 kmin = ~0ull;
  if (threadIdx.x < kHalf) {
#pragma unroll
    for (i32 q = 0; q < kPerThread; ++q) {
      const i32 i = threadIdx.x + q * kHalf;
      if (i >= cnt) continue;
      s[i] = key[q];
      kmin = key[q] < kmin ? key[q] : kmin;
      if (rflag[src[q]]) {
        const i32 e = atomicAdd(&s_ne, 1);
        if (e < kRiskEvents) {
          ev_key[e] = key[q];
          ev_b[e] = src[q];
          ev_d[e] = -w[q];
          atomicAdd(&bcnt[src[q]], 1);
        }
      }
      if (rflag[dst[q]]) {
        const i32 e = atomicAdd(&s_ne, 1);
        if (e < kRiskEvents) {
          ev_key[e] = key[q];
          ev_b[e] = dst[q];
          ev_d[e] = w[q];
          atomicAdd(&bcnt[dst[q]], 1);
        }
      }
    }
  }
  __syncthreads();
  trace_mark(a, 29);
  const i32 ne = s_ne;
  if (ne > kRiskEvents) return false;   // block-uniform
  {   // first grouped slot of each part: exclusive scan, two parts per thread
    const i32 b0 = 2 * threadIdx.x;
    const u32 c0 = b0 < k ? (u32)bcnt[b0] : 0u, c1 = b0 + 1 < k ? (u32)bcnt[b0 + 1] : 0u;
    u32 tot;
    const u32 ex = block_exscan_u32(c0 + c1, s_warp, tot);
    if (b0 < k) boff[b0] = (i32)ex;
    if (b0 + 1 < k) boff[b0 + 1] = (i32)(ex + c0);
  }
  __syncthreads();
  for (i32 e = threadIdx.x; e < ne; e += blockDim.x) {
    const i32 b = ev_b[e];
    const i32 at = boff[b] + atomicAdd(&bfill[b], 1);
    gk[at] = ev_key[e];
    gd[at] = ev_d[e];
    gb[at] = b;
  }
  __syncthreads();
  // marked key ranges
  for (i32 j = threadIdx.x; j < ne; j += blockDim.x) {
    const i32 b = gb[j];
    const u64 kj = gk[j];
    i32 D = 0;
    u64 knext = ~0ull;
    for (i32 f = boff[b], fe = boff[b] + bcnt[b]; f < fe; ++f) {
      const u64 kf = gk[f];
      if (kf <= kj) D += gd[f];
      else knext = kf < knext ? kf : knext;
    }
    if (D > 0 && __uint2float_rn((u32)D + (u32)rpw[b]) > a.maxw) {
      const i32 at = atomicAdd(&s_nbad, 1);
      bad_lo[at] = kj;
      bad_hi[at] = knext;
    }
  }
  kmin = block_reduce_u64<false>(kmin, s_tmp);   // (its barriers publish the ranges)
  trace_mark(a, 30);
  const i32 nbad = s_nbad;
  // the largest candidate key in no marked range
  u64 best = 0;
  bool any = false;
  for (i32 i = threadIdx.x; i < cnt; i += blockDim.x) {
    const u64 kk = s[i];
    bool marked = false;
    for (i32 r = 0; r < nbad && !marked; ++r) marked = bad_lo[r] <= kk && kk < bad_hi[r];
    if (!marked) {
      best = kk > best ? kk : best;
      any = true;
    }
  }
  const u64 top = block_reduce_u64<true>(any ? best + 1 : 0, s_tmp);   // +1: 0 means none
  const u64 K = top ? top - 1 : kmin;
  u32 c = 0;
  for (i32 i = threadIdx.x; i < cnt; i += blockDim.x) c += s[i] <= K;
  u32 tot;
  (void)block_exscan_u32(c, s_warp, tot);
  *kstar = K;
  *napplied = (i32)tot;
  return true;
}

// Plain level: select and apply in one phase.  The kept moves are the first
// B = min(cnt, cap) candidates by (gain desc, id asc) (uncoarsen.hpp:471-476,
// move_request.hpp:36-41), and moves 0..pos are applied, pos = the largest
// balanced index (uncoarsen.hpp:239-288; prefix 0 always counts as
// balanced, :481-488).
//  * cnt <= cap and no part's inflow bound passes MAXW (see ph_candidates):
//    every index is balanced, all candidates move, and their order does not
//    matter: no sort, no check.
//  * cnt <= cap otherwise: the check over the flagged parts alone, in key
//    order (refine_threshold); the moves with key <= K* apply.
//  * cnt > cap, or too many events for that check: every CTA that owns a
//    move index below B sorts the candidates itself (all get the same order)
//    and runs the check over all parts (refine_balanced_pos).
// Every check reads the source parts from msrc and pw as it was before the
// round: the moves of this phase add their weights to pwd, which the gain
// update folds into pw.  Move j is applied by global warp j (mod the warp
// count), so a CTA owns an index below B iff blockIdx.x * warps_per_cta < B.
// Returns (thread 0) the CTA's appends to U.  cnt: the round's candidates.
__device__ u32 ph_refine_apply(const LevelArgs& a, u64* s, i32* greedy, u64* keep, u32* s_warp, u64* s_tmp,
                               UStage& S, i32 cnt) {
  RoundState* st = a.st;
  const i32 B = cnt < a.move_cap ? cnt : a.move_cap;
  const i32 nw = blockDim.x >> 5;
  const i64 warp = (i64)blockIdx.x * nw + (threadIdx.x >> 5);
  const i64 nwarps = (i64)gridDim.x * nw;
  if ((i64)blockIdx.x * nw >= B) return 0;   // block-uniform: no move index of this CTA is kept
  // the warp's first candidate, loaded beside the check flag (used when every
  // candidate applies)
  const u64 key0 = warp < cnt ? ldc(a.cands + warp) : 0ull;
  const bool check = ldc(&st->needcheck) != 0;
  __shared__ unsigned long long s_gsum;
  if (threadIdx.x == 0) {
    s_gsum = 0;
    S.cnt = 0;
  }
  u64 kstar = ~0ull;   // cnt <= cap: the moves with key <= kstar apply
  i32 napplied = B;
  bool sorted = false;
  i32 pos = B - 1;     // sorted: moves 0..pos of keep apply
  if (check) {
    bool done = false;
    if (cnt <= a.move_cap) done = refine_check_risk(a, cnt, s, greedy, keep, s_tmp, s_warp, &kstar, &napplied);
    trace_mark(a, 25);
    if (!done) {
      select_sort(a, a.cands, cnt, s, greedy);   // s[0..B) sorted (ends with a block barrier)
      for (i32 i = threadIdx.x; i < B; i += blockDim.x) keep[i] = s[i];
      __syncthreads();
      pos = refine_balanced_pos(a, s, reinterpret_cast<u64*>(greedy), B, s_warp, a.msrc);
      napplied = pos + 1;
      sorted = true;
      trace_mark(a, 26);
    }
  } else if (cnt > a.move_cap) {
    select_sort(a, a.cands, cnt, s, greedy);   // the first cap candidates, all balanced
    for (i32 i = threadIdx.x; i < B; i += blockDim.x) keep[i] = s[i];
    sorted = true;
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->rounds += 1;
    st->moves += napplied;
    st->cand_sum += cnt;
  }
  if (sorted) {
    for (i64 j = warp; j <= pos; j += nwarps) apply_move(a, S, keep[j], a.pwd, &s_gsum);
  } else {
    for (i64 j = warp; j < cnt; j += nwarps) {
      const u64 key = j == warp ? key0 : ldc(a.cands + j);
      if (key <= kstar) apply_move(a, S, key, a.pwd, &s_gsum);   // warp-uniform
    }
  }
  ustage_flush(S, a.U, &st->ucount);
  if (threadIdx.x == 0 && s_gsum) atomicAdd((unsigned long long*)&st->gain_sum, s_gsum);
  return (u32)S.cnt;
}

// Plain level, after the moves of a round: their part-weight changes join pw,
// the inflow bounds and the per-round counters start again from zero.  Runs
// beside the gain update, which reads none of these.
__device__ void ph_fold(const LevelArgs& a) {
  const i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < a.k; p += stride) {
    const u32 d = ldc(a.pwd + p);
    if (d) {
      a.pw[p] = ldc(a.pw + p) + d;
      a.pwd[p] = 0;
    }
    if (ldc(a.pin + p)) a.pin[p] = 0;
    if (ldc(a.risk + p)) a.risk[p] = 0;
    if (ldc(a.pnet + p)) a.pnet[p] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.st->ccount = 0;
    a.st->needcheck = 0;
  }
}

// ---------------------------------------------------------------------------
// Balance rounds (default mode; the reference has none -- an overweight part
// is only reported, cuda_check.hpp:105-113).
//   prep      lightest part (ties: smaller id), new round epoch, stop when no
//             part is overweight                                  (block 0)
//   filter    boundary vertices of overweight parts -> list
//   eval      per listed vertex (one warp): best neighbouring part with room
//             by signed gain ed_q - id (ties: smaller q), else the lightest
//             part if it has room; marks candidates
//   emit      candidates without a smaller-id candidate neighbour -> keys
//   select    sort by (gain desc, id asc), cap, then a greedy pass in that
//             order keeps each move whose source is still overweight and
//             whose destination stays within the cap          (block 0)
//   apply     the kept moves, flag U; then the gain update
// ---------------------------------------------------------------------------
__device__ void ph_bal_prep(const LevelArgs& a, u64* s_tmp) {
  if (blockIdx.x != 0) return;
  u64 best = ~0ull;
  u32 heavy = 0;
  for (i32 p = threadIdx.x; p < a.k; p += blockDim.x) {
    const u32 w = ldc(a.pw + p);
    const u64 key = ((u64)w << 32) | (u32)p;
    best = key < best ? key : best;
    heavy = w > heavy ? w : heavy;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const u64 y = __shfl_xor_sync(kFullMask, best, o);
    best = y < best ? y : best;
    const u32 z = __shfl_xor_sync(kFullMask, heavy, o);
    heavy = z > heavy ? z : heavy;
  }
  if ((threadIdx.x & 31) == 0) s_tmp[threadIdx.x >> 5] = best;
  __shared__ u32 s_heavy[32];
  if ((threadIdx.x & 31) == 0) s_heavy[threadIdx.x >> 5] = heavy;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      best = s_tmp[w] < best ? s_tmp[w] : best;
      heavy = s_heavy[w] > heavy ? s_heavy[w] : heavy;
    }
    a.st->light = (i32)(u32)best;
    a.st->epoch = ++(*a.epoch);
    a.st->lcount = 0;
    if (!over_cap(heavy, a.bcap)) a.st->bdone = 1;   // no part is overweight
  }
  __syncthreads();
}

// Batched level: CTA b finds the lightest part of graphs b, b + grid, ...;
// a balance-active graph with an overweight part raises anyf[r % 3] (block 0
// clears anyf[(r + 1) % 3]).  Block 0 opens the round's epoch.
__device__ void ph_bal_prep_batch(const LevelArgs& a, u64* s_tmp, i64 r) {
  __shared__ u32 s_over[32];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.st->epoch = ++(*a.epoch);
    a.st->lcount = 0;
    a.anyf[(r + 1) % 3] = 0;
  }
  for (i32 g = blockIdx.x; g < a.G; g += gridDim.x) {
    const i32 pb = __ldg(a.gpbase + g), k = __ldg(a.gk + g);
    u64 best = ~0ull;
    u32 over = 0;
    for (i32 p = pb + threadIdx.x; p < pb + k; p += blockDim.x) {
      const u32 w = ldc(a.pw + p);
      const u64 key = ((u64)w << 32) | (u32)p;
      best = key < best ? key : best;
      over |= over_cap(w, __ldg(a.pbcap + p)) ? 1u : 0u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const u64 y = __shfl_xor_sync(kFullMask, best, o);
      best = y < best ? y : best;
      over |= __shfl_xor_sync(kFullMask, over, o);
    }
    if ((threadIdx.x & 31) == 0) {
      s_tmp[threadIdx.x >> 5] = best;
      s_over[threadIdx.x >> 5] = over;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        best = s_tmp[w] < best ? s_tmp[w] : best;
        over |= s_over[w];
      }
      a.glight[g] = (i32)(u32)best;
      if (over && ((__ldg(a.gflags + g) >> 1) & 1)) atomicExch(a.anyf + r % 3, 1);
    }
    __syncthreads();
  }
}

// Boundary vertices of overweight parts -> blist.
__device__ void ph_bal_filter(const LevelArgs& a) {
  if (a.batch && blockIdx.x == 0 && threadIdx.x == 0) *a.mcount = 0;
  const int lane = threadIdx.x & 31;
  const i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 base = (i64)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < a.n; base += stride) {
    const i64 v = base + lane;
    bool want = false;
    if (v < a.n && ldc(a.bnd + v) && graph_flag(a, (i32)v, 1)) {
      const i32 p = ldc(a.part + v);
      want = over_cap(ldc(a.pw + p), bcap_of(a, p));
    }
    warp_append(want, (i32)v, a.blist, &a.st->lcount);
  }
}

__device__ void ph_bal_eval(const LevelArgs& a, u32* acc_all) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (wid >= a.acc_warps) return;
  u32* acc = acc_all + (size_t)wid * a.kacc;
  RoundState* st = a.st;
  const u32 ep = ldc(&st->epoch);
  const i32 light_plain = a.batch ? 0 : ldc(&st->light);
  const i32 nl = ldc(&st->lcount);
  const i64 nw = (i64)gridDim.x * a.acc_warps;
  for (i64 i = (i64)blockIdx.x * a.acc_warps + wid; i < nl; i += nw) {
    const i32 v = ldc(a.blist + i);
    const i32 p = ldc(a.part + v);
    const u32 w = (u32)a.vwgt[v];
    const i32 pb = part_base_of(a, v);
    u32* accb = acc - pb;   // rows are indexed by the graph's own part ids
    const i32 light = a.batch ? ldc(a.glight + __ldg(a.gid + v)) : light_plain;
    const i32 beg = a.xadj[v], end = a.xadj[v + 1];
    for (i32 e = beg + lane; e < end; e += 32) atomicAdd(&accb[ldc(a.part + a.adjncy[e])], (u32)a.adjwgt[e]);
    __syncwarp();
    const u32 id = accb[p];
    u64 best = 0;
    for (i32 e = beg + lane; e < end; e += 32) {
      const i32 q = ldc(a.part + a.adjncy[e]);
      if (q == p || over_cap(ldc(a.pw + q) + w, bcap_of(a, q))) continue;
      const i32 g = (i32)(accb[q] - id);
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
    } else if (light != p && !over_cap(ldc(a.pw + light) + w, bcap_of(a, light))) {
      q_best = light;
      g_best = (i32)(accb[light] - id);
    }
    if (lane == 0 && q_best >= 0) {
      a.bmark[v] = ep;
      a.btarget[v] = q_best;
      a.bgain[v] = g_best;
    }
    __syncwarp();
    for (i32 e = beg + lane; e < end; e += 32) accb[ldc(a.part + a.adjncy[e])] = 0;
    __syncwarp();
  }
}

__device__ void ph_bal_emit(const LevelArgs& a) {
  RoundState* st = a.st;
  const int lane = threadIdx.x & 31;
  const i32 nl = ldc(&st->lcount);
  const u32 ep = ldc(&st->epoch);
  const i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 base = (i64)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < nl; base += stride) {
    const i64 i = base + lane;
    bool emit = false;
    i32 v = 0, g = 0;
    if (i < nl) {
      v = ldc(a.blist + i);
      emit = ldc(a.bmark + v) == ep;
      g = emit ? ldc(a.bgain + v) : 0;
      for (i32 e = a.xadj[v]; emit && e < a.xadj[v + 1]; ++e) {
        const i32 u = a.adjncy[e];
        if (u < v && ldc(a.bmark + u) == ep) { emit = false; break; }
      }
    }
    if (a.batch) {   // graph buckets, as in ph_candidates
      if (emit) {
        const i32 gv = __ldg(a.gid + v);
        a.cands[__ldg(a.gvbase + gv) + atomicAdd(a.gcc + gv, 1)] = move_key(g, v);
      }
    } else {
      warp_append64(emit, move_key(g, v), a.cands, &st->ccount);
    }
  }
}

__device__ void ph_apply_balance(const LevelArgs& a, UStage& S) {
  RoundState* st = a.st;
  const i32 pos = (a.batch ? ldc(a.mcount) : ldc(&st->firstbad)) - 1;
  const int lane = threadIdx.x & 31;
  const i64 warp = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const i64 nwarps = ((i64)gridDim.x * blockDim.x) >> 5;
  if (threadIdx.x == 0) S.cnt = 0;
  __syncthreads();
  if (warp == 0 && lane == 0) {
    st->brounds += 1;
    st->bmoves += pos + 1;
  }
  for (i64 j = warp; j <= pos; j += nwarps) {
    const i32 v = (i32)(u32)ldc(a.top + j);
    const i32 s = ldc(a.part + v), d = ldc(a.btarget + v);
    if (lane == 0) {
      const u32 w = (u32)a.vwgt[v];
      atomicAdd(&a.pw[d], w);
      atomicSub(&a.pw[s], w);
      a.part[v] = d;
      if (atomicExch(&a.updflag[v], 1) == 0) ustage_push(S, v, a.U, &st->ucount);
    }
    const i32 beg = a.xadj[v], end = a.xadj[v + 1];
    for (i32 e = beg + lane; e < end; e += 32) {
      const i32 u = a.adjncy[e];
      if (atomicExch(&a.updflag[u], 1) == 0) ustage_push(S, u, a.U, &st->ucount);
    }
  }
  ustage_flush(S, a.U, &st->ucount);
}

// ---------------------------------------------------------------------------
// The level kernel.
// ---------------------------------------------------------------------------
// Resident level-kernel CTAs per SM the register budget is sized for.
#ifndef GKW_LEVEL_MIN_BLOCKS
#define GKW_LEVEL_MIN_BLOCKS 2
#endif
__global__ void __launch_bounds__(kLevelThreads, GKW_LEVEL_MIN_BLOCKS) k_level(LevelArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  u64* s_sort = reinterpret_cast<u64*>(smem_raw);                  // kSortMax u64
  i32* greedy = reinterpret_cast<i32*>(smem_raw + kSortMax * 8);   // kGreedyWords
  u64* s_keep = reinterpret_cast<u64*>(greedy + kGreedyWords);    // kMaxMoveCap u64: sorted moves
  u32* acc_all = reinterpret_cast<u32*>(s_keep + kMaxMoveCap);     // acc_warps * k u32
  __shared__ u32 s_warp[33];
  __shared__ u64 s_tmp[32];
  __shared__ i32 s_flag;
  __shared__ i32 s_cnt, s_base;
  __shared__ UStage s_ustage;
  {
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (wid < a.acc_warps)
      for (i32 q = lane; q < a.kacc; q += 32) acc_all[(size_t)wid * a.kacc + q] = 0;
  }
  __syncthreads();
  RoundState* st = a.st;
  // batched levels: the rotating flag use counter (uniform over the grid)
  i64 fr = 0;
  // the counting barriers' words start at zero: block 0 clears them before
  // its first grid barrier, which every CTA passes before the first of them
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.cbar->w[0] = 0;
    a.cbar->w[1] = 0;
    a.cbar->w[2] = 0;
  }
  trace_mark(a, 0);
  if (a.flags & LF_PROJECT) {
    ph_project(a, s_ustage);
    if (!grid_barrier(a.bar, a.err, &s_flag)) return;
    trace_mark(a, 1);
  }
  if (a.flags & LF_LISTS) {
    ph_lists(a);
    if (!grid_barrier(a.bar, a.err, &s_flag)) return;
    trace_mark(a, 2);
  }
  if (a.flags & LF_UPDATE) ph_update_first(a, acc_all, reinterpret_cast<u32*>(smem_raw), s_ustage);
  if (a.flags & LF_BALANCE) {
    if (a.batch) ph_bal_prep_batch(a, s_tmp, fr);
    else ph_bal_prep(a, s_tmp);
  }
  if (a.flags & (LF_UPDATE | LF_BALANCE)) {
    if (!grid_barrier(a.bar, a.err, &s_flag)) return;
    trace_mark(a, 3);
  }
  if (a.flags & LF_BALANCE) {
    for (i64 r = 0;; ++r) {
      if (r > a.max_rounds) {   // uniform: every CTA counts the same rounds
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(a.err, 2);
        return;
      }
      // nothing overweight (prep) or no candidate (select)
      if (a.batch ? ldc(a.anyf + fr % 3) == 0 : ldc(&st->bdone) != 0) break;
      ++fr;
      ph_bal_filter(a);
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
      trace_mark(a, 9);
      ph_bal_eval(a, acc_all);
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
      trace_mark(a, 10);
      ph_bal_emit(a);
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
      trace_mark(a, 11);
      if (a.batch) ph_select_batch(a, s_sort, greedy, s_warp, true, fr);
      else ph_bal_select(a, s_sort, greedy);
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
      trace_mark(a, 12);
      if (a.batch ? ldc(a.anyf + fr % 3) == 0 : ldc(&st->bdone) != 0) break;
      ++fr;
      ph_apply_balance(a, s_ustage);
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
      trace_mark(a, 14);
      ph_update(a, acc_all, true, s_ustage);
      if (a.batch) ph_bal_prep_batch(a, s_tmp, fr);
      else ph_bal_prep(a, s_tmp);
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
      trace_mark(a, 15);
    }
  }
  if (a.flags & LF_REFINE) {
    // plain levels: the round's list lengths ride on the barriers
    // (grid_barrier_count); P only grows within a level.  A launch without an
    // earlier phase passes one grid barrier first, which orders block 0's
    // clearing of the counting words before every CTA's first use.
    if (!(a.flags & (LF_PROJECT | LF_LISTS | LF_UPDATE | LF_BALANCE)))
      if (!grid_barrier(a.bar, a.err, &s_flag)) return;
    __shared__ i32 s_total;
    u32 cbk = 0;
    i32 nP = a.batch ? -1 : ldc(&st->pcount[0]);
    for (i64 r = 0;; ++r) {
      if (r > a.max_rounds) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(a.err, 3);
        return;
      }
      const u32 my_cands = ph_candidates(a, &s_cnt, &s_base, reinterpret_cast<u32*>(greedy), nP);
      if (a.batch) {
        if (!grid_barrier(a.bar, a.err, &s_flag)) return;
        trace_mark(a, 20);
        ++fr;
        ph_select_batch(a, s_sort, greedy, s_warp, false, fr);
        if (!grid_barrier(a.bar, a.err, &s_flag)) return;
        trace_mark(a, 21);
        if (ldc(a.anyf + fr % 3) == 0) break;
        ph_apply_refine(a, s_ustage);
        if (!grid_barrier(a.bar, a.err, &s_flag)) return;
        trace_mark(a, 23);
        ph_update(a, acc_all, true, s_ustage);
        if (!grid_barrier(a.bar, a.err, &s_flag)) return;
        trace_mark(a, 24);
        continue;
      }
      i32 nC, nU, nPadd;
      if (!grid_barrier_count(a.cbar, cbk++, a.err, &s_flag, &s_total, my_cands, &nC)) return;
      if (nC < 0) nC = ldc(&st->ccount);
      trace_mark(a, 20);
      if (nC == 0) break;   // every CTA has the same count
      const u32 my_u = ph_refine_apply(a, s_sort, greedy, s_keep, s_warp, s_tmp, s_ustage, nC);
      if (!grid_barrier_count(a.cbar, cbk++, a.err, &s_flag, &s_total, my_u, &nU)) return;
      trace_mark(a, 23);
      const u32 my_p = ph_update(a, acc_all, true, s_ustage, nU);
      ph_fold(a);
      if (!grid_barrier_count(a.cbar, cbk++, a.err, &s_flag, &s_total, my_p, &nPadd)) return;
      nP = nPadd < 0 ? ldc(&st->pcount[0]) : nP + nPadd;
      trace_mark(a, 24);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    LevelStatsDev* o = a.stat_slot;
    o->rounds = ldc(&st->rounds);
    o->moves = ldc(&st->moves);
    o->gain_sum = ldc(&st->gain_sum);
    o->brounds = ldc(&st->brounds);
    o->bmoves = ldc(&st->bmoves);
    o->rows = (i64)ldc(&st->rows);
    o->cand_sum = ldc(&st->cand_sum);
    o->err = *(volatile i32*)a.err;
  }
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

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static void ctx_common(Handle& h, Pool& P, RefineCtx* c, size_t n) {
  c->updflag = P.alloc_n<i32>(n);
  c->inP = P.alloc_n<i32>(n);
  c->U = P.alloc_n<i32>(n);
  c->P[0] = P.alloc_n<i32>(n);
  c->P[1] = P.alloc_n<i32>(n);
  c->cands = P.alloc_n<u64>(n);
  // a batch keeps up to move_cap moves per graph in one round; every vertex
  // is a candidate at most once per round, so n entries always suffice
  const bool batched = c->kacc > 0 && c->kacc < c->k;
  c->top = P.alloc_n<u64>(batched ? std::max<size_t>(n, kMaxMoveCap) : kMaxMoveCap);
  c->pw = P.alloc_n<u32>(c->k);
  c->pwd = P.alloc_n<u32>(c->k);
  c->pin = P.alloc_n<u32>(c->k);
  c->msrc = P.alloc_n<i32>(n);
  c->cinfo = P.alloc_n<u64>(n);
  c->cw = P.alloc_n<i32>(n);
  c->risk = P.alloc_n<u32>(c->k);
  c->pnet = P.alloc_n<i32>(c->k);
  c->st = P.alloc_n<RoundState>(1);
  c->bmark = P.alloc_n<u32>(n);
  c->btarget = P.alloc_n<i32>(n);
  c->bgain = P.alloc_n<i32>(n);
  c->blist = P.alloc_n<i32>(n);
  c->brem = P.alloc_n<u32>(c->k);
  c->epoch = P.alloc_n<u32>(1);
  c->bar = P.alloc_n<GridBarrier>(1);
  c->cbar = P.alloc_n<CountBarrier>(1);
  c->err = P.alloc_n<i32>(1);
  c->stats = P.alloc_n<LevelStatsDev>(kStatSlots);
  if (const char* t = getenv("GKW_TRACE"); t && *t == '1') {
    c->trace = P.alloc_n<u64>((size_t)kStatSlots * kTraceCap);
    c->trace_n = P.alloc_n<i32>(kStatSlots);
    GKW_CUDA(cudaMemsetAsync(c->trace_n, 0, sizeof(i32) * kStatSlots, h.stream));
  }
  GKW_CUDA(cudaMemsetAsync(c->bmark, 0, sizeof(u32) * n, h.stream));
  GKW_CUDA(cudaMemsetAsync(c->pwd, 0, sizeof(u32) * c->k, h.stream));   // kept at zero between rounds
  GKW_CUDA(cudaMemsetAsync(c->pin, 0, sizeof(u32) * c->k, h.stream));
  GKW_CUDA(cudaMemsetAsync(c->risk, 0, sizeof(u32) * c->k, h.stream));
  GKW_CUDA(cudaMemsetAsync(c->pnet, 0, sizeof(i32) * c->k, h.stream));
  GKW_CUDA(cudaMemsetAsync(c->epoch, 0, sizeof(u32), h.stream));
  GKW_CUDA(cudaMemsetAsync(c->bar, 0, sizeof(GridBarrier), h.stream));
  GKW_CUDA(cudaMemsetAsync(c->err, 0, sizeof(i32), h.stream));
  GKW_CUDA(cudaMemsetAsync(c->stats, 0, sizeof(LevelStatsDev) * kStatSlots, h.stream));
  // per-warp part-connection rows: as many warps as fit beside the sort buffer
  const size_t budget = 120 * 1024;
  if (c->kacc <= 0) c->kacc = c->k;
  const i32 w = (i32)std::min<size_t>(kLevelThreads / 32, budget / (4 * (size_t)c->kacc));
  c->acc_warps = std::max(1, w);
  c->smem = (size_t)kSortMax * 8 + (size_t)kGreedyWords * 4 + (size_t)kMaxMoveCap * 8 +
            (size_t)c->acc_warps * c->kacc * 4;
  // one value for every handle of the process (handles of a server launch
  // this kernel concurrently with different sizes): the device's opt-in limit
  // less the kernel's static shared memory
  cudaFuncAttributes fa;
  GKW_CUDA(cudaFuncGetAttributes(&fa, k_level));
  const int max_dyn = h.smem_optin - (int)fa.sharedSizeBytes;
  GKW_REQUIRE(c->smem <= (size_t)max_dyn, GKW_E_UNSUPPORTED, "level kernel needs too much shared memory");
  GKW_CUDA(cudaFuncSetAttribute(k_level, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn));
  int bps = 0;
  GKW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_level, kLevelThreads, c->smem));
  GKW_REQUIRE(bps >= 1, GKW_E_UNSUPPORTED, "level kernel does not fit on an SM");
  c->grid = h.sm_count * std::min(bps, 2);
}

RefineCtx* refine_create(Handle& h, i32 n_max, i32 k, i32 move_cap, i32 kacc) {
  GKW_REQUIRE(move_cap >= 1 && move_cap <= kMaxMoveCap, GKW_E_UNSUPPORTED, "move_cap must be in [1, 2048]");
  if (kacc <= 0) kacc = k;
  GKW_REQUIRE(kacc >= 1 && kacc <= 40000, GKW_E_UNSUPPORTED, "k must be in [1, 40000]");
  GKW_REQUIRE(k >= kacc && k < (1 << 21), GKW_E_UNSUPPORTED, "too many parts");
  RefineCtx* c = new RefineCtx();
  c->n_max = n_max;
  c->k = k;
  c->kacc = kacc;
  c->cap = move_cap;
  const size_t n = std::max(n_max, 1);
  Pool& P = h.hier;
  c->part[0] = P.alloc_n<i32>(n);
  c->part[1] = P.alloc_n<i32>(n);
  c->bnd[0] = P.alloc_n<i32>(n);
  c->bnd[1] = P.alloc_n<i32>(n);
  c->gain = P.alloc_n<i32>(n);
  c->target = P.alloc_n<i32>(n);
  ctx_common(h, P, c, n);
  return c;
}

// A context over caller-owned state arrays (per-phase entry points).
RefineCtx* refine_create_ext(Handle& h, i32 n, i32 k, i32 move_cap, i32* part, i32* bnd, i32* gain,
                             i32* target) {
  GKW_REQUIRE(move_cap >= 1 && move_cap <= kMaxMoveCap, GKW_E_UNSUPPORTED, "move_cap must be in [1, 2048]");
  GKW_REQUIRE(k >= 1 && k <= 40000, GKW_E_UNSUPPORTED, "k must be in [1, 40000]");
  RefineCtx* c = new RefineCtx();
  c->n_max = n;
  c->k = k;
  c->cap = move_cap;
  c->part[0] = part;
  c->bnd[0] = bnd;
  c->gain = gain;
  c->target = target;
  ctx_common(h, h.scratch, c, std::max(n, 1));
  return c;
}

void refine_destroy(RefineCtx* c) { delete c; }
i32* refine_part(RefineCtx* c) { return c->part[c->cur]; }
i32* refine_boundary(RefineCtx* c) { return c->bnd[c->cur]; }
i32* refine_gain(RefineCtx* c) { return c->gain; }
i32* refine_target(RefineCtx* c) { return c->target; }
u32* refine_pw(RefineCtx* c) { return c->pw; }

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
  GKW_CUDA(cudaMemsetAsync(c->updflag, 0, sizeof(i32) * g.n, h.stream));
  GKW_CUDA(cudaMemsetAsync(c->inP, 0, sizeof(i32) * g.n, h.stream));
  GKW_CUDA(cudaMemsetAsync(c->gain, 0, sizeof(i32) * g.n, h.stream));
}

void refine_init_union(Handle& h, RefineCtx* c, const DevGraph& cu, const i32* part, i32* bnd_out) {
  c->cur = 0;
  GKW_CUDA(cudaMemsetAsync(c->pw, 0, sizeof(u32) * c->k, h.stream));
  if (cu.n == 0) return;
  launch(k_boundary_pw, ceil_div(cu.n, 256), 256, 0, h.stream, cu.n, cu.xadj, cu.adjncy, cu.vwgt, part, bnd_out,
         c->pw);
  GKW_CHECK_LAUNCH();
}

void level_run(Handle& h, RefineCtx* c, const DevGraph& g, const LevelJob& j, i32 slot) {
  GKW_REQUIRE(j.move_cap >= 1 && j.move_cap <= c->cap, GKW_E_INVALID, "move_cap out of range");
  GKW_REQUIRE(slot >= 0 && slot < kStatSlots, GKW_E_INTERNAL, "stats slot out of range");
  GKW_CUDA(cudaMemsetAsync(c->st, 0, sizeof(RoundState), h.stream));
  // barrier words start from zero for every launch; an error of an earlier
  // level stays in c->err, so every later level leaves at its first barrier
  GKW_CUDA(cudaMemsetAsync(c->bar, 0, sizeof(GridBarrier), h.stream));
  LevelArgs a;
  memset(&a, 0, sizeof(a));
  a.n = g.n;
  a.k = c->k;
  {   // first gain pass: lane groups on short rows, when their connection rows
      // fit in the sort and greedy buffers
    const size_t room = ((size_t)kSortMax * 8 + (size_t)kGreedyWords * 4) / 4;
    const double avg = g.n ? (double)g.m / g.n : 0.0;
    const size_t kr = (size_t)std::max(c->kacc, 1);
    a.upd_lanes = (avg <= 8.0 && (kLevelThreads / 8) * kr <= room)    ? 8
                  : (avg <= 16.0 && (kLevelThreads / 16) * kr <= room) ? 16
                                                                       : 32;
  }
  a.xadj = g.xadj;
  a.adjncy = g.adjncy;
  a.adjwgt = g.adjwgt;
  a.vwgt = g.vwgt;
  a.maxw = j.maxw;
  a.bcap = j.bcap;
  a.move_cap = j.move_cap;
  a.max_rounds = 4 * (i64)g.n + 64;
  i32 flags = 0;
  const i32 src = c->cur;
  i32 dst = c->cur;
  if (j.cmap) {
    flags |= LF_PROJECT | LF_UPDATE;
    dst = c->cur ^ 1;
    a.cmap = j.cmap;
    a.part_c = c->part[src];
    a.bnd_c = c->bnd[src];
  }
  if (j.lists) {
    flags |= LF_LISTS | LF_UPDATE;
    a.updated_in = j.updated;
  }
  if (j.balance) flags |= LF_BALANCE;
  if (j.refine) flags |= LF_REFINE;
  a.flags = flags;
  a.part = c->part[dst];
  a.bnd = c->bnd[dst];
  a.gain = c->gain;
  a.target = c->target;
  a.updflag = c->updflag;
  a.inP = c->inP;
  a.U = c->U;
  a.P0 = c->P[0];
  a.P1 = c->P[1];
  a.cands = c->cands;
  a.top = c->top;
  a.pw = c->pw;
  a.pwd = c->pwd;
  a.pin = c->pin;
  a.msrc = c->msrc;
  a.cinfo = c->cinfo;
  a.cw = c->cw;
  a.risk = c->risk;
  a.pnet = c->pnet;
  a.st = c->st;
  a.bmark = c->bmark;
  a.btarget = c->btarget;
  a.bgain = c->bgain;
  a.blist = c->blist;
  a.brem = c->brem;
  a.epoch = c->epoch;
  a.bar = c->bar;
  a.cbar = c->cbar;
  a.err = c->err;
  a.stat_slot = c->stats + slot;
  a.acc_warps = c->acc_warps;
  a.kacc = c->kacc;
  if (j.batch) {
    a.batch = 1;
    a.G = j.batch->G;
    a.gid = j.batch->gid;
    a.gvbase = j.batch->gvbase;
    a.gpbase = j.batch->gpbase;
    a.gk = j.batch->gk;
    a.gflags = j.batch->gflags;
    a.pmaxw = j.batch->pmaxw;
    a.pbcap = j.batch->pbcap;
    a.gcc = j.batch->gcc;
    a.glight = j.batch->glight;
    a.mcount = j.batch->mcount;
    a.anyf = j.batch->anyf;
    a.part_init = j.batch->part_init;
    a.bnd_init = j.batch->bnd_init;
  }
  if (c->trace) {
    a.trace = c->trace + (size_t)slot * kTraceCap;
    a.trace_cap = kTraceCap;
    a.trace_n = c->trace_n + slot;
  }
  i32 grid = (i32)ceil_div(std::max(g.n, 1), std::max(h.tuning.level_verts_per_cta, 32));
  grid = std::max(grid, std::max(h.tuning.level_min_ctas, c->kacc / 4));   // large k: few gain-update warps per CTA
  grid = std::min(grid, c->grid);
  grid = coop_grid(h, (const void*)k_level, grid, kLevelThreads, c->smem);
  void* args[] = {&a};
  if (j.ev_start) GKW_CUDA(cudaEventRecord(j.ev_start, h.stream));
  launch_coop(h, (const void*)k_level, grid, kLevelThreads, c->smem, args);
  if (j.ev_end) GKW_CUDA(cudaEventRecord(j.ev_end, h.stream));
  c->cur = dst;
}

std::vector<RefineLevelStats> level_stats(Handle& h, RefineCtx* c, i32 nslots) {
  GKW_REQUIRE(nslots >= 0 && nslots <= kStatSlots, GKW_E_INTERNAL, "stats slot out of range");
  std::vector<LevelStatsDev> d((size_t)std::max(nslots, 1));
  if (nslots) {
    GKW_CUDA(cudaMemcpyAsync(d.data(), c->stats, sizeof(LevelStatsDev) * nslots, cudaMemcpyDeviceToHost,
                             h.stream));
  }
  GKW_CUDA(cudaMemcpyAsync(h.h_pinned, c->err, sizeof(i32), cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  const i32 err = *(i32*)h.h_pinned;
  if (err == 1) throw Error{GKW_E_INTERNAL, "level kernel: grid barrier timed out"};
  if (err == 2) throw Error{GKW_E_INTERNAL, "balancing did not terminate"};
  if (err == 3) throw Error{GKW_E_INTERNAL, "refinement did not terminate"};
  if (c->trace && nslots) {
    std::vector<i32> tn(nslots);
    std::vector<u64> tr((size_t)nslots * kTraceCap);
    GKW_CUDA(cudaMemcpyAsync(tn.data(), c->trace_n, sizeof(i32) * nslots, cudaMemcpyDeviceToHost, h.stream));
    GKW_CUDA(cudaMemcpyAsync(tr.data(), c->trace, sizeof(u64) * tr.size(), cudaMemcpyDeviceToHost, h.stream));
    GKW_CUDA(cudaStreamSynchronize(h.stream));
    for (i32 s = 0; s < nslots; ++s) {
      if (tn[s] < 2) continue;
      double acc[32] = {0};
      i32 cnt[32] = {0};
      const u64* t = tr.data() + (size_t)s * kTraceCap;
      for (i32 i = 1; i < tn[s]; ++i) {
        const u32 ph = (u32)(t[i] >> 56);
        const double dt = (double)((t[i] & 0x00ffffffffffffffull) - (t[i - 1] & 0x00ffffffffffffffull));
        if (ph < 32) { acc[ph] += dt; cnt[ph] += 1; }
      }
      const double tot = (double)((t[tn[s] - 1] & 0x00ffffffffffffffull) - (t[0] & 0x00ffffffffffffffull));
      fprintf(stderr, "[gkw trace] level slot %d: %.1f us total; candidates/round %.0f;", s, tot / 1e3,
              d[s].rounds ? (double)d[s].cand_sum / d[s].rounds : 0.0);
      for (i32 p = 0; p < 32; ++p)
        if (cnt[p]) fprintf(stderr, " ph%d x%d %.2fus", p, cnt[p], acc[p] / cnt[p] / 1e3);
      fprintf(stderr, "\n");
    }
    GKW_CUDA(cudaMemsetAsync(c->trace_n, 0, sizeof(i32) * kStatSlots, h.stream));
  }
  std::vector<RefineLevelStats> out((size_t)nslots);
  for (i32 i = 0; i < nslots; ++i) {
    out[i].rounds = d[i].rounds;
    out[i].moves = d[i].moves;
    out[i].gain_sum = d[i].gain_sum;
    out[i].brounds = d[i].brounds;
    out[i].bmoves = d[i].bmoves;
    out[i].rows = d[i].rows;
  }
  return out;
}

// ---------------------------------------------------------------------------
// Metrics: exact weighted cut over u < v (uncoarsen.hpp:398-424) and part
// weights (cuda_check.hpp:61-73); part weights are summed per CTA in shared
// memory first.
// ---------------------------------------------------------------------------
__global__ void k_cut_pw(i32 n, const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                         const i32* __restrict__ adjwgt, const i32* __restrict__ vwgt,
                         const i32* __restrict__ part, i32 k, unsigned long long* __restrict__ cut,
                         unsigned long long* __restrict__ pw, i32* __restrict__ bad) {
  extern __shared__ unsigned long long s_pw[];
  const bool local = k <= 4096;
  if (local) {
    for (i32 p = threadIdx.x; p < k; p += blockDim.x) s_pw[p] = 0;
    __syncthreads();
  }
  u64 c = 0;
  for (i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (i64)gridDim.x * blockDim.x) {
    const i32 p = part[v];
    if ((u32)p >= (u32)k) {
      atomicOr(bad, 1);
      continue;
    }
    for (i32 e = xadj[v]; e < xadj[v + 1]; ++e) {
      const i32 u = adjncy[e];
      if (v < u && part[u] != p) c += (u32)adjwgt[e];
    }
    if (local) atomicAdd(&s_pw[p], (unsigned long long)(u32)vwgt[v]);
    else atomicAdd(&pw[p], (unsigned long long)(u32)vwgt[v]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFullMask, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(cut, (unsigned long long)c);
  if (local) {
    __syncthreads();
    for (i32 p = threadIdx.x; p < k; p += blockDim.x)
      if (s_pw[p]) atomicAdd(&pw[p], s_pw[p]);
  }
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

void launch_cut_pw(cudaStream_t stream, i32 sm_count, const DevGraph& g, const i32* part, i32 k, i64* d_acc) {
  if (g.n == 0) return;
  const size_t sm = k <= 4096 ? sizeof(unsigned long long) * k : 0;
  const u32 grid = std::max<u32>(1, std::min<u32>(ceil_div(g.n, 256), (u32)sm_count * 8));
  launch(k_cut_pw, grid, 256, sm, stream, g.n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, part, k,
         (unsigned long long*)d_acc, (unsigned long long*)(d_acc + 2), (i32*)(d_acc + 1));
  GKW_CHECK_LAUNCH();
}

void compute_cut_pw(Handle& h, const DevGraph& g, const i32* part, i32 k, i64* d_cut, i64* d_pw) {
  GKW_REQUIRE(d_pw == d_cut + 2, GKW_E_INTERNAL, "cut accumulators must be contiguous");
  GKW_CUDA(cudaMemsetAsync(d_cut, 0, sizeof(i64) * (k + 2), h.stream));   // [0] cut, [1] bad-part flag, pw
  launch_cut_pw(h.stream, h.sm_count, g, part, k, d_cut);
}

}  // namespace gkw
