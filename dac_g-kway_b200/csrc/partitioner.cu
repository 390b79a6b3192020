// The multilevel driver and the C ABI.
//
// graph_partitioner() of the reference (gkway/graph_partitioner.hpp:222-365)
// runs coarsening (:14-123), the initial partition (:125-131) and the
// uncoarsening loop (:133-220); partition_impl below does the same on
// device-resident levels kept in the handle's hierarchy pool.
#include <algorithm>
#include <cstring>
#include <exception>
#include <functional>
#include <new>

#include "gkw_internal.cuh"

namespace gkw {

// ---------------------------------------------------------------------------
// Input validation on the device: xadj monotone from 0 to nnz, neighbour ids
// in range and not the vertex itself, weights >= 0.  Also sums vertex weights.
// flags[0] bit0 bad xadj, bit1 bad id, bit2 self loop, bit3 negative weight.
// ---------------------------------------------------------------------------
// flags[1] receives the longest row.  Rows are checked by G lanes each (G
// from the average row length); rows longer than kValidateLong are left to
// k_validate_long, one CTA each, so that a hub row does not hold a lane for
// thousands of loads.
constexpr i32 kValidateLong = 512;

__device__ __forceinline__ i32 validate_entries(i32 v, i32 n, i32 b, i32 e, i32 first, i32 step,
                                                const i32* __restrict__ adjncy, const i32* __restrict__ adjwgt) {
  i32 f = 0;
  for (i32 j = b + first; j < e; j += step) {
    const i32 u = adjncy[j];
    if (u < 0 || u >= n) f |= 2;
    else if (u == v) f |= 4;
    if (adjwgt[j] < 0) f |= 8;
  }
  return f;
}

template <int G>
__global__ void k_validate(i32 n, i64 m, const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                           const i32* __restrict__ adjwgt, const i32* __restrict__ vwgt,
                           i32* __restrict__ flags, unsigned long long* __restrict__ wsum, i32* __restrict__ longlist,
                           i32* __restrict__ longcnt) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 v = t / G;
  const int sub = threadIdx.x & (G - 1);
  i32 f = 0, deg = 0;
  u64 w = 0;
  if (v < n) {
    const i32 b = xadj[v], e = xadj[v + 1];
    if (e < b || b < 0 || (i64)e > m) f |= 1;
    if (v == 0 && b != 0) f |= 1;
    if (v == n - 1 && (i64)e != m) f |= 1;
    if (sub == 0) {
      if (vwgt[v] < 0) f |= 8;
      w = (u32)vwgt[v];
    }
    if (!(f & 1)) {
      deg = e - b;
      if (deg > kValidateLong) {
        if (sub == 0) longlist[atomicAdd(longcnt, 1)] = (i32)v;
      } else {
        f |= validate_entries((i32)v, n, b, e, sub, G, adjncy, adjwgt);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    f |= __shfl_xor_sync(0xffffffffu, f, o);
    w += __shfl_xor_sync(0xffffffffu, w, o);
    const i32 d = __shfl_xor_sync(0xffffffffu, deg, o);
    deg = d > deg ? d : deg;
  }
  // one set of global atomics per CTA: per-warp atomics on these three words
  // serialised (131k warps on a million-vertex graph, ~0.1 ms)
  __shared__ i32 s_f[32], s_d[32];
  __shared__ unsigned long long s_w[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) {
    s_f[wid] = f;
    s_d[wid] = deg;
    s_w[wid] = w;
  }
  __syncthreads();
  if (wid == 0) {
    f = lane < nw ? s_f[lane] : 0;
    deg = lane < nw ? s_d[lane] : 0;
    w = lane < nw ? s_w[lane] : 0;
    for (int o = 16; o > 0; o >>= 1) {
      f |= __shfl_xor_sync(0xffffffffu, f, o);
      w += __shfl_xor_sync(0xffffffffu, w, o);
      const i32 d = __shfl_xor_sync(0xffffffffu, deg, o);
      deg = d > deg ? d : deg;
    }
    if (lane == 0) {
      if (f) atomicOr(flags, f);
      if (w) atomicAdd(wsum, (unsigned long long)w);
      if (deg) atomicMax(flags + 1, deg);
    }
  }
}

__global__ void k_validate_long(i32 n, const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                                const i32* __restrict__ adjwgt, i32* __restrict__ flags,
                                const i32* __restrict__ longlist, const i32* __restrict__ longcnt) {
  const i32 nl = *longcnt;
  for (i32 r = blockIdx.x; r < nl; r += gridDim.x) {
    const i32 v = longlist[r];
    i32 f = validate_entries(v, n, xadj[v], xadj[v + 1], threadIdx.x, blockDim.x, adjncy, adjwgt);
    for (int o = 16; o > 0; o >>= 1) f |= __shfl_xor_sync(0xffffffffu, f, o);
    if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
  }
}

__global__ void k_fill_i32(i32* p, i64 n, i32 v) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

__global__ void k_sub_i32(i32* p, i64 n, i32 v) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] -= v;
}

// returns total vertex weight (the longest row in *maxdeg); throws on malformed input
i64 validate(Handle& h, const DevGraph& g, i64* maxdeg) {
  Pool::Mark mk = h.scratch.mark();
  i32* flags = h.scratch.alloc_n<i32>(4);   // [0] error bits, [1] longest row, [2] long rows
  unsigned long long* ws = h.scratch.alloc_n<unsigned long long>(1);
  i32* longlist = h.scratch.alloc_n<i32>(std::max(g.n, 1));
  GKW_CUDA(cudaMemsetAsync(flags, 0, sizeof(i32) * 4, h.stream));
  GKW_CUDA(cudaMemsetAsync(ws, 0, sizeof(u64), h.stream));
  if (g.n > 0) {
    const double avg = (double)g.m / g.n;
    auto go = [&](auto kern, int G) {
      launch(kern, ceil_div((u64)g.n * G, 256), 256, 0, h.stream, g.n, g.m, g.xadj, g.adjncy, g.adjwgt, g.vwgt,
             flags, ws, longlist, flags + 2);
    };
    if (avg <= 6.5) go(k_validate<4>, 4);
    else if (avg <= 14) go(k_validate<8>, 8);
    else go(k_validate<16>, 16);
    launch(k_validate_long, (u32)h.sm_count * 2, 256, 0, h.stream, g.n, g.xadj, g.adjncy, g.adjwgt, flags,
           (const i32*)longlist, (const i32*)(flags + 2));
    GKW_CHECK_LAUNCH();
  }
  GKW_CUDA(cudaMemcpyAsync(h.h_pinned, flags, sizeof(i32) * 2, cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaMemcpyAsync(h.h_pinned + 1, ws, sizeof(u64), cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  const i32 f = (i32)(h.h_pinned[0] & 0xffffffff);
  if (maxdeg) *maxdeg = (i32)((u64)h.h_pinned[0] >> 32);
  const i64 W = h.h_pinned[1];
  h.scratch.release(mk);
  if (f & 1) throw Error{GKW_E_INVALID, "malformed xadj (must rise from 0 to nnz)"};
  if (f & 2) throw Error{GKW_E_INVALID, "neighbour id out of range"};
  if (f & 4) throw Error{GKW_E_INVALID, "self loop in the graph"};
  if (f & 8) throw Error{GKW_E_INVALID, "negative weight"};
  return W;
}

// GKW_CHECK=1: validate every stage's output on the device before the next
// stage reads it (coarse CSR, cmap range, part ids), so that a stage that
// produced bad indices is reported by name instead of feeding them on.
static bool stage_checks() {
  static const bool on = [] {
    const char* e = getenv("GKW_CHECK");
    return e && *e == '1';
  }();
  return on;
}

static void check_stage(const char* what, i32 level, const std::function<void()>& f) {
  try {
    f();
  } catch (const Error& e) {
    throw Error{GKW_E_INTERNAL, std::string("stage check after ") + what + " (level " + std::to_string(level) +
                                    "): " + e.msg};
  }
}

// Milliseconds between two recorded events; -1 (and no pending CUDA error
// left behind) if either was never recorded.
static double elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float t = 0;
  if (cudaEventElapsedTime(&t, a, b) != cudaSuccess) {
    cudaGetLastError();
    return -1.0;
  }
  return t;
}

void ensure_timer_events(Handle& h) {
  if (h.tev_ready) return;
  for (cudaEvent_t& e : h.tev) GKW_CUDA(cudaEventCreate(&e));
  h.tev_ready = true;
}

// Initial partition of the coarsest graph cg into cpart: the device GGGP, or
// the caller's callback (the reference calls host METIS here,
// metis_partition.hpp:46-47).
static void initial_partition(Handle& h, const DevGraph& cg, i32 k, const gkw_options& opt, i32* cpart) {
  if (opt.init_method == GKW_INIT_CALLBACK) {
    std::vector<i32> hx(cg.n + 1), ha(cg.m), hw(cg.m), hv(cg.n), hp(cg.n);
    GKW_CUDA(cudaMemcpyAsync(hx.data(), cg.xadj, sizeof(i32) * (cg.n + 1), cudaMemcpyDeviceToHost, h.stream));
    if (cg.m) {
      GKW_CUDA(cudaMemcpyAsync(ha.data(), cg.adjncy, sizeof(i32) * cg.m, cudaMemcpyDeviceToHost, h.stream));
      GKW_CUDA(cudaMemcpyAsync(hw.data(), cg.adjwgt, sizeof(i32) * cg.m, cudaMemcpyDeviceToHost, h.stream));
    }
    if (cg.n) GKW_CUDA(cudaMemcpyAsync(hv.data(), cg.vwgt, sizeof(i32) * cg.n, cudaMemcpyDeviceToHost, h.stream));
    GKW_CUDA(cudaStreamSynchronize(h.stream));
    const i32 rcb = opt.init_fn(opt.init_user, cg.n, hx.data(), ha.data(), hw.data(), hv.data(), k, hp.data());
    if (rcb != 0) throw Error{GKW_E_INIT, "initial-partition callback returned " + std::to_string(rcb)};
    for (i32 v = 0; v < cg.n; ++v)
      if (hp[v] < 0 || hp[v] >= k) throw Error{GKW_E_INIT, "initial-partition callback gave a part out of range"};
    if (cg.n) GKW_CUDA(cudaMemcpyAsync(cpart, hp.data(), sizeof(i32) * cg.n, cudaMemcpyHostToDevice, h.stream));
    GKW_CUDA(cudaStreamSynchronize(h.stream));
  } else {
    device_init_partition(h, cg, k, opt.eps, opt.seed, std::max(1, std::min(8, opt.init_trials)), cpart);
  }
}

static void check_options(const gkw_options& opt) {
  GKW_REQUIRE(opt.group_cap >= 1, GKW_E_INVALID, "group_cap must be >= 1");
  GKW_REQUIRE(opt.threshold_factor >= 0, GKW_E_INVALID, "threshold_factor must be >= 0");
  GKW_REQUIRE(opt.init_method == GKW_INIT_DEVICE || (opt.init_method == GKW_INIT_CALLBACK && opt.init_fn),
              GKW_E_INVALID, "init_method CALLBACK needs init_fn");
}

void partition_impl(Handle& h, const DevGraph& g0, i32 k, const gkw_options& opt, i32* d_part_out,
                           i64* cut_out, gkw_stats* stats) {
  GKW_REQUIRE(k >= 1, GKW_E_INVALID, "k must be >= 1");
  GKW_REQUIRE(g0.n >= 0 && g0.m >= 0 && g0.m < ((i64)1 << 31), GKW_E_UNSUPPORTED,
              "graphs need n >= 0 and nnz < 2^31");
  check_options(opt);
  ensure_timer_events(h);
  cudaEvent_t* ev = h.tev;              // phase marks
  cudaEvent_t* lev = h.tev + 5;         // level kernel of slot s: lev[2s], lev[2s+1]
  GKW_CUDA(cudaEventRecord(ev[0], h.stream));
  i64 maxdeg0 = -1;
  const i64 W = validate(h, g0, &maxdeg0);
  // the reference's MAX_PARTITION_WGT, or the default mode's strict cap
  const float maxw = opt.enforce_balance ? balance_cap(W, k, opt.eps) : max_part_weight(W, k, opt.eps);
  const i64 threshold = (i64)opt.threshold_factor * k;

  // ---- coarsening (graph_partitioner.hpp:66-105) ----
  std::vector<Level> lv(1);
  lv[0].g = g0;
  lv[0].g.maxdeg = maxdeg0;
  std::vector<i32> uf_rounds;
  while ((i64)lv.back().g.n > threshold && (i32)lv.size() < kMaxLevels) {
    CoarsenOut co;
    coarsen_level(h, lv.back().g, opt.group_cap, co);
    if (co.nc == lv.back().g.n || co.nc < k + 1) break;   // level discarded (:93-96)
    // default mode: no coarse vertex may outweigh coarse_vertex_frac of a part
    // (a whole component merged into one vertex cannot be balanced later)
    if (opt.enforce_balance && opt.coarse_vertex_frac > 0 &&
        (double)co.max_cvw > opt.coarse_vertex_frac * (double)W / (double)k)
      break;
    lv.back().cmap = co.cmap;
    if (stage_checks()) {
      const i32 L = (i32)lv.size() - 1;
      check_stage("grouping", L, [&] { check_parts(h, lv.back().g.n, co.cmap, co.nc); });
      DevGraph cgc;
      cgc.n = co.nc;
      cgc.m = co.mc;
      cgc.xadj = co.cxadj;
      cgc.adjncy = co.cadjncy;
      cgc.adjwgt = co.cadjwgt;
      cgc.vwgt = co.cvwgt;
      check_stage("contraction", L, [&] { validate(h, cgc); });
    }
    Level nl;
    nl.g.n = co.nc;
    nl.g.m = co.mc;
    nl.g.xadj = co.cxadj;
    nl.g.adjncy = co.cadjncy;
    nl.g.adjwgt = co.cadjwgt;
    nl.g.vwgt = co.cvwgt;
    nl.g.maxdeg = co.maxdeg;
    uf_rounds.push_back(co.uf_rounds);
    lv.push_back(nl);
  }
  GKW_CUDA(cudaEventRecord(ev[1], h.stream));

  // ---- initial partition of the coarsest level ----
  const DevGraph& cg = lv.back().g;
  RefineCtx* rc = refine_create(h, std::max(g0.n, 1), k, opt.move_cap);
  struct CtxGuard {
    RefineCtx* c;
    ~CtxGuard() { refine_destroy(c); }
  } cguard{rc};
  i32* cpart = refine_part(rc);
  initial_partition(h, cg, k, opt, cpart);
  if (stage_checks()) check_stage("initial partition", (i32)lv.size() - 1, [&] { check_parts(h, cg.n, cpart, k); });
  refine_init_coarsest(h, rc, cg, cpart);
  i64* d_metrics = h.hier.alloc_n<i64>(k + 2);   // [0] cut, [1] bad-part flag, [2..k+2) part weights
  i64* d_init = h.hier.alloc_n<i64>(k + 2);      // the same for the initial partition
  if (stats)   // cut of the initial partition itself (before any balance move), read at the end
    compute_cut_pw(h, cg, refine_part(rc), k, d_init, d_init + 2);
  const i32 nl = (i32)lv.size();
  // default mode: balance rounds at every level but the balance_skip_levels
  // coarsest ones (the finest level always)
  auto balances = [&](i32 L) {
    return opt.enforce_balance && (L == 0 || L < nl - std::max(0, opt.balance_skip_levels));
  };
  if (balances(nl - 1)) {
    LevelJob j;
    j.balance = true;
    j.bcap = maxw;
    j.move_cap = opt.move_cap;
    j.ev_start = lev[2 * (nl - 1)];
    j.ev_end = lev[2 * (nl - 1) + 1];
    level_run(h, rc, cg, j, nl - 1);
  }
  GKW_CUDA(cudaEventRecord(ev[2], h.stream));

  // ---- uncoarsening (graph_partitioner.hpp:174-192): one launch per level ----
  for (i32 L = nl - 2; L >= 0; --L) {
    LevelJob j;
    j.cmap = lv[L].cmap;
    j.balance = balances(L);
    j.bcap = maxw;
    j.refine = true;
    j.maxw = maxw;
    j.move_cap = opt.move_cap;
    j.ev_start = lev[2 * L];
    j.ev_end = lev[2 * L + 1];
    level_run(h, rc, lv[L].g, j, L);
    if (stage_checks()) check_stage("refinement", L, [&] { check_parts(h, lv[L].g.n, refine_part(rc), k); });
  }
  GKW_CUDA(cudaEventRecord(ev[3], h.stream));
  // ---- output and final metrics (graph_partitioner.hpp:194-202) ----
  if (g0.n) {
    GKW_CUDA(cudaMemcpyAsync(d_part_out, refine_part(rc), sizeof(i32) * g0.n, cudaMemcpyDeviceToDevice,
                             h.stream));
  }
  compute_cut_pw(h, g0, d_part_out, k, d_metrics, d_metrics + 2);
  std::vector<i64> hm(k + 2);
  GKW_CUDA(cudaMemcpyAsync(hm.data(), d_metrics, sizeof(i64) * (k + 2), cudaMemcpyDeviceToHost, h.stream));
  i64 init_cut = 0;
  if (stats) GKW_CUDA(cudaMemcpyAsync(&init_cut, d_init, sizeof(i64), cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaEventRecord(ev[4], h.stream));
  // one host sync for the statistics, the error words and the metrics above
  std::vector<RefineLevelStats> rs = level_stats(h, rc, nl);
  GKW_REQUIRE(hm[1] == 0, GKW_E_INTERNAL, "partition produced a part id out of range");
  if (cut_out) *cut_out = hm[0];
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->n_levels = (i32)lv.size();
    for (size_t i = 0; i < lv.size(); ++i) {
      stats->level_n[i] = lv[i].g.n;
      stats->level_m[i] = lv[i].g.m;
    }
    for (size_t i = 0; i < uf_rounds.size(); ++i) stats->uf_rounds[i] = uf_rounds[i];
    for (size_t i = 0; i + 1 < lv.size(); ++i) {
      stats->refine_rounds[i] = rs[i].rounds;
      stats->refine_moves[i] = rs[i].moves;
    }
    for (size_t i = 0; i < lv.size(); ++i) {
      stats->balance_rounds[i] = rs[i].brounds;
      stats->balance_moves[i] = rs[i].bmoves;
      stats->round_entries[i] = rs[i].rows;
      // the coarsest level has a launch only when it runs balance rounds
      const bool ran = (i + 1 < lv.size()) || balances(nl - 1);
      stats->ms_level[i] = ran ? elapsed_ms(lev[2 * i], lev[2 * i + 1]) : -1.0;
    }
    stats->init_cut = init_cut;
    stats->cut = hm[0];
    i64 mx = 0;
    for (i32 p = 0; p < k; ++p) mx = std::max(mx, hm[2 + p]);
    stats->max_part_weight = mx;
    stats->maxw = maxw;
    stats->ms_coarsen = elapsed_ms(ev[0], ev[1]);
    stats->ms_init = elapsed_ms(ev[1], ev[2]);
    stats->ms_refine = elapsed_ms(ev[2], ev[3]);
    stats->ms_total = elapsed_ms(ev[0], ev[4]);
  }
}

// One graph partitioned for several k over one hierarchy.  Matching,
// union-find, grouping and contraction do not depend on k; only where the
// coarsening stops does (the threshold threshold_factor * k,
// graph_partitioner.hpp:22; the discard rule nc < k + 1, :93-96; the default
// mode's coarse-vertex cap).  The levels are built while some k still
// coarsens, and each k runs the initial partition and the uncoarsening of
// partition_impl on its own prefix of them, so its result is the one
// partition_impl gives alone.  d_parts holds nk rows of g0.n part ids.
void partition_multi_impl(Handle& h, const DevGraph& g0, i32 nk, const i32* ks, const gkw_options& opt,
                          i32* d_parts, i64* cuts_out) {
  GKW_REQUIRE(nk >= 0 && (nk == 0 || ks != nullptr), GKW_E_INVALID, "ks is NULL");
  for (i32 q = 0; q < nk; ++q) GKW_REQUIRE(ks[q] >= 1, GKW_E_INVALID, "k must be >= 1");
  GKW_REQUIRE(g0.n >= 0 && g0.m >= 0 && g0.m < ((i64)1 << 31), GKW_E_UNSUPPORTED,
              "graphs need n >= 0 and nnz < 2^31");
  check_options(opt);
  i64 maxdeg0 = -1;
  const i64 W = validate(h, g0, &maxdeg0);
  std::vector<Level> lv(1);
  lv[0].g = g0;
  lv[0].g.maxdeg = maxdeg0;
  std::vector<i32> Lk(nk, -1);   // coarsest level of each k
  for (;;) {
    const i32 l = (i32)lv.size() - 1;
    const i64 nl = lv.back().g.n;
    bool any = false;
    for (i32 q = 0; q < nk; ++q) {
      if (Lk[q] < 0 && (nl <= (i64)opt.threshold_factor * ks[q] || (i32)lv.size() >= kMaxLevels)) Lk[q] = l;
      any |= Lk[q] < 0;
    }
    if (!any) break;
    CoarsenOut co;
    coarsen_level(h, lv.back().g, opt.group_cap, co);
    bool cont = false;
    for (i32 q = 0; q < nk; ++q) {
      if (Lk[q] >= 0) continue;
      bool stop = co.nc == nl || co.nc < ks[q] + 1;   // level discarded for this k
      if (opt.enforce_balance && opt.coarse_vertex_frac > 0 &&
          (double)co.max_cvw > opt.coarse_vertex_frac * (double)W / (double)ks[q])
        stop = true;
      if (stop) Lk[q] = l;
      else cont = true;
    }
    if (!cont) break;
    lv.back().cmap = co.cmap;
    Level nx;
    nx.g.n = co.nc;
    nx.g.m = co.mc;
    nx.g.xadj = co.cxadj;
    nx.g.adjncy = co.cadjncy;
    nx.g.adjwgt = co.cadjwgt;
    nx.g.vwgt = co.cvwgt;
    nx.g.maxdeg = co.maxdeg;
    lv.push_back(nx);
  }
  for (i32 q = 0; q < nk; ++q) {
    const i32 k = ks[q];
    const float maxw = opt.enforce_balance ? balance_cap(W, k, opt.eps) : max_part_weight(W, k, opt.eps);
    const i32 nl = Lk[q] + 1;
    const DevGraph& cg = lv[nl - 1].g;
    const Pool::Mark mk = h.hier.mark();   // this k's state, released before the next k
    RefineCtx* rc = refine_create(h, std::max(g0.n, 1), k, opt.move_cap);
    struct CtxGuard {
      RefineCtx* c;
      ~CtxGuard() { refine_destroy(c); }
    } cguard{rc};
    i32* cpart = refine_part(rc);
    initial_partition(h, cg, k, opt, cpart);
    refine_init_coarsest(h, rc, cg, cpart);
    auto balances = [&](i32 L) {
      return opt.enforce_balance && (L == 0 || L < nl - std::max(0, opt.balance_skip_levels));
    };
    if (balances(nl - 1)) {
      LevelJob j;
      j.balance = true;
      j.bcap = maxw;
      j.move_cap = opt.move_cap;
      level_run(h, rc, cg, j, nl - 1);
    }
    for (i32 L = nl - 2; L >= 0; --L) {
      LevelJob j;
      j.cmap = lv[L].cmap;
      j.balance = balances(L);
      j.bcap = maxw;
      j.refine = true;
      j.maxw = maxw;
      j.move_cap = opt.move_cap;
      level_run(h, rc, lv[L].g, j, L);
    }
    i32* out = d_parts + (size_t)q * g0.n;
    if (g0.n) {
      GKW_CUDA(cudaMemcpyAsync(out, refine_part(rc), sizeof(i32) * g0.n, cudaMemcpyDeviceToDevice, h.stream));
    }
    i64* d_metrics = h.hier.alloc_n<i64>(k + 2);
    compute_cut_pw(h, g0, out, k, d_metrics, d_metrics + 2);
    i64 hm[2] = {0, 0};
    GKW_CUDA(cudaMemcpyAsync(hm, d_metrics, sizeof(i64) * 2, cudaMemcpyDeviceToHost, h.stream));
    level_stats(h, rc, nl);   // one sync; error words of the level kernels
    GKW_REQUIRE(hm[1] == 0, GKW_E_INTERNAL, "partition produced a part id out of range");
    if (cuts_out) cuts_out[q] = hm[0];
    h.hier.release(mk);
  }
}

// The autotuner (gkw_autotune).  Launch shapes never change a result, only
// its time, so each candidate is timed on a full partition of the caller's
// graph:
//   * match lanes: one partition during which every level's match is also
//     run with 4, 8, 16 and 32 lanes per vertex (best of three launches each,
//     CUDA events); each average-degree bucket met keeps the lane count with
//     the least summed time;
//   * level-kernel density: vertices per CTA in {256, 512, 1024, 2048} x
//     minimum CTAs in {16, 32, 64}, best of two partitions each by the
//     refinement phase's event time;
//   * coarsening: per-phase kernels on every level, or one fused launch per
//     level for levels of at most 80k or 300k vertices, best of two
//     partitions each by the coarsening phase's event time.
void autotune(Handle& h, const DevGraph& g, i32 k, const gkw_options& opt) {
  i32* part = nullptr;
  GKW_CUDA(cudaMalloc((void**)&part, sizeof(i32) * std::max(g.n, 1)));
  struct Free {
    i32* p;
    ~Free() { cudaFree(p); }
  } fr{part};
  auto run = [&](gkw_stats* st) {
    h.hier.reset();
    h.scratch.reset();
    i64 cut = 0;
    partition_impl(h, g, k, opt, part, &cut, st);
  };
  gkw_stats st;
  run(&st);   // warm
  memset(h.tune_match_ms, 0, sizeof(h.tune_match_ms));
  h.tune_collect = true;
  try {
    run(&st);
  } catch (...) {
    h.tune_collect = false;
    throw;
  }
  h.tune_collect = false;
  const i32 lanes[kMatchLaneChoices] = {2, 4, 8, 16, 32};
  for (i32 b = 0; b < 4; ++b) {
    i32 best = -1;
    for (i32 q = 0; q < kMatchLaneChoices; ++q)
      if (h.tune_match_ms[b][q] > 0 && (best < 0 || h.tune_match_ms[b][q] < h.tune_match_ms[b][best])) best = q;
    if (best >= 0) h.tuning.match_lanes[b] = lanes[best];
  }
  gkw_tuning best = h.tuning;
  double best_ms = 1e300;
  for (i32 vpc : {256, 512, 1024, 2048}) {
    for (i32 minc : {16, 32, 64}) {
      h.tuning.level_verts_per_cta = vpc;
      h.tuning.level_min_ctas = minc;
      double t = 1e300;
      for (int rep = 0; rep < 2; ++rep) {
        run(&st);
        t = std::min(t, st.ms_refine);
      }
      if (t < best_ms) {
        best_ms = t;
        best = h.tuning;
      }
    }
  }
  h.tuning = best;
  // coarsening: the per-phase kernels, or one fused launch for the levels of
  // at most 80k / 300k vertices, by the coarsening phase's event time
  best_ms = 1e300;
  for (i32 fmax : {0, 80000, 300000}) {
    h.tuning.coarsen_fused_max_n = fmax;
    h.tuning.coarsen_verts_per_cta = 256;
    double t = 1e300;
    for (int rep = 0; rep < 2; ++rep) {
      run(&st);
      t = std::min(t, st.ms_coarsen);
    }
    if (t < best_ms) {
      best_ms = t;
      best = h.tuning;
    }
  }
  h.tuning = best;
}

// Copies a host CSR into the handle's hierarchy pool (unit weights where the
// arrays are NULL).  The host arrays may be a slice of a larger concatenated
// CSR: xadj values are then offset by xadj[0] and neighbour ids by vbase, and
// both are rebased on the device.
DevGraph upload_host_graph(Handle& hh, const DevGraph& hg, i64 vbase) {
  GKW_REQUIRE(hg.n >= 0 && hg.m >= 0, GKW_E_INVALID, "negative size");
  GKW_REQUIRE(vbase >= 0 && vbase < ((i64)1 << 31), GKW_E_UNSUPPORTED, "vertex offset out of range");
  const i64 n = hg.n, m = hg.m;
  i32* x = hh.hier.alloc_n<i32>(n + 1);
  i32* a = hh.hier.alloc_n<i32>(std::max<i64>(m, 1));
  i32* w = hh.hier.alloc_n<i32>(std::max<i64>(m, 1));
  i32* vw = hh.hier.alloc_n<i32>(std::max<i64>(n, 1));
  GKW_CUDA(cudaMemcpyAsync(x, hg.xadj, sizeof(i32) * (n + 1), cudaMemcpyHostToDevice, hh.stream));
  const i32 ebase = hg.xadj[0];
  if (ebase != 0) {
    launch(k_sub_i32, ceil_div(n + 1, 256), 256, 0, hh.stream, x, n + 1, ebase);
    GKW_CHECK_LAUNCH();
  }
  if (m) {
    GKW_CUDA(cudaMemcpyAsync(a, hg.adjncy, sizeof(i32) * m, cudaMemcpyHostToDevice, hh.stream));
    if (vbase != 0) {
      launch(k_sub_i32, ceil_div(m, 256), 256, 0, hh.stream, a, m, (i32)vbase);
      GKW_CHECK_LAUNCH();
    }
    if (hg.adjwgt) GKW_CUDA(cudaMemcpyAsync(w, hg.adjwgt, sizeof(i32) * m, cudaMemcpyHostToDevice, hh.stream));
    else launch(k_fill_i32, ceil_div(m, 256), 256, 0, hh.stream, w, m, 1);
  }
  if (n) {
    if (hg.vwgt) GKW_CUDA(cudaMemcpyAsync(vw, hg.vwgt, sizeof(i32) * n, cudaMemcpyHostToDevice, hh.stream));
    else launch(k_fill_i32, ceil_div(n, 256), 256, 0, hh.stream, vw, n, 1);
  }
  GKW_CHECK_LAUNCH();
  DevGraph g;
  g.n = hg.n;
  g.m = m;
  g.xadj = x;
  g.adjncy = a;
  g.adjwgt = w;
  g.vwgt = vw;
  return g;
}

// Partition of a graph held in host memory: copy it into the handle's pool,
// partition, copy the part ids back.  The host arrays may be a slice of a
// larger concatenated CSR: `xadj` values are then offset by xadj[0] and
// neighbour ids by `vbase`, and both are rebased on the device.
void partition_host(Handle& hh, const DevGraph& hg, i64 vbase, i32 k, const gkw_options& o, i32* part_out,
                    i64* cut_out, gkw_stats* stats) {
  GKW_REQUIRE(hg.n == 0 || part_out != nullptr, GKW_E_INVALID, "part_out is NULL");
  hh.hier.reset();
  hh.scratch.reset();
  const DevGraph g = upload_host_graph(hh, hg, vbase);
  i32* part = hh.hier.alloc_n<i32>(std::max<i64>(hg.n, 1));
  partition_impl(hh, g, k, o, part, cut_out, stats);
  if (hg.n) GKW_CUDA(cudaMemcpyAsync(part_out, part, sizeof(i32) * hg.n, cudaMemcpyDeviceToHost, hh.stream));
  GKW_CUDA(cudaStreamSynchronize(hh.stream));
}

// Several k over one hierarchy, host arrays in and out (nk rows of n ids).
void partition_multi_host(Handle& hh, const DevGraph& hg, i32 nk, const i32* ks, const gkw_options& o,
                          i32* parts_out, i64* cuts_out) {
  GKW_REQUIRE(hg.n == 0 || nk == 0 || parts_out != nullptr, GKW_E_INVALID, "parts_out is NULL");
  hh.hier.reset();
  hh.scratch.reset();
  const DevGraph g = upload_host_graph(hh, hg, 0);
  i32* parts = hh.hier.alloc_n<i32>(std::max<i64>((i64)hg.n * std::max(nk, 1), 1));
  partition_multi_impl(hh, g, nk, ks, o, parts, cuts_out);
  if (hg.n && nk)
    GKW_CUDA(cudaMemcpyAsync(parts_out, parts, sizeof(i32) * (size_t)hg.n * nk, cudaMemcpyDeviceToHost, hh.stream));
  GKW_CUDA(cudaStreamSynchronize(hh.stream));
}

}  // namespace gkw
