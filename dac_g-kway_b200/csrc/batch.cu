// Batched partitioning of many independent graphs as one disjoint union.
//
// Every step of the pipeline is a rule on a vertex's own neighbourhood, on its
// union-find component, or on one graph's parts, so it can run over the union
// of many graphs at once and give each graph exactly its lone result:
//
//   * coarsening: matching, union-find labels (max id of the component, hop
//     distance from it), the (root, dist, id) group order and the contraction
//     never mix graphs, and the coarse ids of a graph stay one contiguous,
//     identically ordered block.  A graph that has stopped coarsening is
//     frozen (no vertex takes a partner) and passes to the next level as an
//     identical copy.  The stop rules are checked per graph; when a graph's
//     new level must be discarded (no progress, fewer than k + 1 vertices, a
//     vertex heavier than the coarse-vertex cap), the level is built again
//     with that graph frozen.
//   * initial partition: GGGP on the deepest level with global part ids
//     (graph g owns [pbase[g], pbase[g] + k[g])); seeds use the graph's own
//     part ids.
//   * uncoarsening: one level-kernel launch per union level; a graph refines
//     (and balances) only below its own coarsest level, and its candidate
//     order, move cap, balanced prefix and end of rounds are its own
//     (refine.cu, batched levels).
//
// The whole batch costs the launches and host round trips of one partition
// instead of one partition per graph.
#include <algorithm>
#include <cstring>
#include <vector>

#include "gkw_internal.cuh"

namespace gkw {

namespace {

__global__ void k_fill_one(i32* p, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = 1;
}

__global__ void k_fill_gid(i32 n, const i32* __restrict__ gvbase, i32 G, i32* __restrict__ gid) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  i32 lo = 0, hi = G;   // last g with gvbase[g] <= v
  while (hi - lo > 1) {
    const i32 mid = (lo + hi) >> 1;
    if (gvbase[mid] <= v) lo = mid;
    else hi = mid;
  }
  gid[v] = lo;
}

__global__ void k_graph_weight(i32 n, const i32* __restrict__ gid, const i32* __restrict__ vwgt,
                               unsigned long long* __restrict__ W) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) atomicAdd(W + gid[v], (unsigned long long)(u32)vwgt[v]);
}

__global__ void k_cross_edges(i32 n, const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                              const i32* __restrict__ gid, i32* __restrict__ bad) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 g = gid[v];
  for (i32 e = xadj[v]; e < xadj[v + 1]; ++e)
    if (gid[adjncy[e]] != g) { atomicExch(bad, 1); return; }
}

__global__ void k_coarse_range(i32 n, const i32* __restrict__ gid, const i32* __restrict__ cmap,
                               i32* __restrict__ cmin, i32* __restrict__ cmax) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) {
    atomicMin(cmin + gid[v], cmap[v]);
    atomicMax(cmax + gid[v], cmap[v]);
  }
}

__global__ void k_graph_maxw(i32 n, const i32* __restrict__ gid, const i32* __restrict__ vwgt, i32* __restrict__ mx) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) atomicMax(mx + gid[v], vwgt[v]);
}

__global__ void k_local_parts(i32 n, const i32* __restrict__ gid, const i32* __restrict__ gpbase,
                              const i32* __restrict__ part, i32* __restrict__ out) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) out[v] = part[v] - gpbase[gid[v]];
}

__global__ void k_graph_cut(i32 n, const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                            const i32* __restrict__ adjwgt, const i32* __restrict__ gid,
                            const i32* __restrict__ part, unsigned long long* __restrict__ cut) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 p = part[v];
  u64 c = 0;
  for (i32 e = xadj[v]; e < xadj[v + 1]; ++e) {
    const i32 u = adjncy[e];
    if (u > v && part[u] != p) c += (u32)adjwgt[e];
  }
  if (c) atomicAdd(cut + gid[v], (unsigned long long)c);
}

// A graph frozen at the input level is carried to level 1 by the contraction,
// which sorts each row; the lone partition of that graph works on the input
// rows in their own order, so copy them verbatim over the contracted block.
// A row whose length changed (duplicate edges merged) sets *bad.
__global__ void k_copy_frozen(i32 n, const i32* __restrict__ gid, const i32* __restrict__ frozen,
                              const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                              const i32* __restrict__ adjwgt, const i32* __restrict__ cmap,
                              const i32* __restrict__ cxadj, i32* __restrict__ cadjncy, i32* __restrict__ cadjwgt,
                              i32* __restrict__ bad) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n || !frozen[gid[v]]) return;
  const i32 c = cmap[v], e0 = xadj[v], len = xadj[v + 1] - e0, c0 = cxadj[c];
  if (cxadj[c + 1] - c0 != len) {
    atomicExch(bad, 1);
    return;
  }
  for (i32 t = 0; t < len; ++t) {
    cadjncy[c0 + t] = cmap[adjncy[e0 + t]];
    cadjwgt[c0 + t] = adjwgt[e0 + t];
  }
}

template <class T>
T* to_dev(Handle& h, const std::vector<T>& v) {
  T* d = h.hier.alloc_n<T>(std::max<size_t>(v.size(), 1));
  if (!v.empty()) GKW_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, h.stream));
  return d;
}

template <class T>
std::vector<T> to_host(Handle& h, const T* d, size_t n) {
  std::vector<T> v(n);
  if (n) GKW_CUDA(cudaMemcpyAsync(v.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  return v;
}

struct ULevel {
  DevGraph g;
  i32* cmap = nullptr;             // to the next level
  i32* gid = nullptr;              // [n]
  std::vector<i32> gv;             // [G + 1] vertex offsets (host)
  i32* gv_d = nullptr;             // [G + 1] (device)
};

}  // namespace

bool partition_batch_union(Handle& hh, const DevGraph& hg, i32 G, const i32* graph_ptr, const i32* ks,
                           const gkw_options& o, i32* part_out, i64* cuts_out) {
  GKW_REQUIRE(o.init_method == GKW_INIT_DEVICE, GKW_E_INVALID, "batched union needs the device initial partition");
  hh.hier.reset();
  hh.scratch.reset();
  const i64 n = hg.n, m = hg.m;
  // ---- input ----
  i32* x = hh.hier.alloc_n<i32>(n + 1);
  i32* a = hh.hier.alloc_n<i32>(std::max<i64>(m, 1));
  i32* w = hh.hier.alloc_n<i32>(std::max<i64>(m, 1));
  i32* vw = hh.hier.alloc_n<i32>(std::max<i64>(n, 1));
  GKW_CUDA(cudaMemcpyAsync(x, hg.xadj, sizeof(i32) * (n + 1), cudaMemcpyHostToDevice, hh.stream));
  if (m) {
    GKW_CUDA(cudaMemcpyAsync(a, hg.adjncy, sizeof(i32) * m, cudaMemcpyHostToDevice, hh.stream));
    if (hg.adjwgt) GKW_CUDA(cudaMemcpyAsync(w, hg.adjwgt, sizeof(i32) * m, cudaMemcpyHostToDevice, hh.stream));
    else launch(k_fill_one, ceil_div(m, 256), 256, 0, hh.stream, w, m);
  }
  if (n) {
    if (hg.vwgt) GKW_CUDA(cudaMemcpyAsync(vw, hg.vwgt, sizeof(i32) * n, cudaMemcpyHostToDevice, hh.stream));
    else launch(k_fill_one, ceil_div(n, 256), 256, 0, hh.stream, vw, n);
  }
  GKW_CHECK_LAUNCH();
  DevGraph g0;
  g0.n = (i32)n;
  g0.m = m;
  g0.xadj = x;
  g0.adjncy = a;
  g0.adjwgt = w;
  g0.vwgt = vw;
  validate(hh, g0);

  // ---- graph tables ----
  std::vector<i32> kv(ks, ks + G), pb(G), part_base;
  i32 K = 0, kmax = 1, depth = 0;
  for (i32 i = 0; i < G; ++i) {
    pb[i] = K;
    GKW_REQUIRE(kv[i] >= 1 && (i64)K + kv[i] < (1 << 21), GKW_E_UNSUPPORTED, "too many parts in the batch");
    for (i32 q = 0; q < kv[i]; ++q) part_base.push_back(K);
    K += kv[i];
    kmax = std::max(kmax, kv[i]);
    i32 d = 0;
    while ((1 << d) < kv[i]) ++d;
    depth = std::max(depth, d);
  }
  if (G == 0 || n == 0) {
    if (cuts_out)
      for (i32 i = 0; i < G; ++i) cuts_out[i] = 0;
    return true;
  }
  i32* gk_d = to_dev(hh, kv);
  i32* gpb_d = to_dev(hh, pb);
  i32* pbase_d = to_dev(hh, part_base);
  std::vector<ULevel> lv(1);
  lv[0].g = g0;
  lv[0].gv.assign(graph_ptr, graph_ptr + G + 1);
  lv[0].gv_d = to_dev(hh, lv[0].gv);
  lv[0].gid = hh.hier.alloc_n<i32>(n);
  launch(k_fill_gid, ceil_div(n, 256), 256, 0, hh.stream, (i32)n, lv[0].gv_d, G, lv[0].gid);
  GKW_CHECK_LAUNCH();
  {
    i32* bad = hh.scratch.alloc_n<i32>(1);
    GKW_CUDA(cudaMemsetAsync(bad, 0, sizeof(i32), hh.stream));
    launch(k_cross_edges, ceil_div(n, 256), 256, 0, hh.stream, (i32)n, x, a, lv[0].gid, bad);
    GKW_CHECK_LAUNCH();
    if (to_host(hh, bad, 1)[0]) return false;   // an edge joins two graphs: not a batch of independent graphs
  }
  std::vector<u64> Wg;
  {
    unsigned long long* Wd = hh.scratch.alloc_n<unsigned long long>(G);
    GKW_CUDA(cudaMemsetAsync(Wd, 0, sizeof(u64) * G, hh.stream));
    launch(k_graph_weight, ceil_div(n, 256), 256, 0, hh.stream, (i32)n, lv[0].gid, vw, Wd);
    GKW_CHECK_LAUNCH();
    auto t = to_host(hh, Wd, G);
    Wg.assign(t.begin(), t.end());
  }
  // caps per part: the default mode's strict cap, or the reference's MAXW
  std::vector<float> pmaxw(K), pbcap(K);
  for (i32 i = 0; i < G; ++i) {
    const float mw = o.enforce_balance ? balance_cap((i64)Wg[i], kv[i], o.eps) : max_part_weight((i64)Wg[i], kv[i], o.eps);
    for (i32 q = 0; q < kv[i]; ++q) {
      pmaxw[pb[i] + q] = mw;
      pbcap[pb[i] + q] = mw;
    }
  }
  float* pmaxw_d = to_dev(hh, pmaxw);
  float* pbcap_d = to_dev(hh, pbcap);

  // ---- coarsening ----
  std::vector<i32> Lg(G, -1);   // coarsest level of each graph (-1: still coarsening)
  auto n_of = [&](const ULevel& L, i32 i) { return L.gv[i + 1] - L.gv[i]; };
  i32* frozen_d = hh.hier.alloc_n<i32>(G);
  for (;;) {
    ULevel& cur = lv.back();
    const i32 l = (i32)lv.size() - 1;
    bool any = false;
    for (i32 i = 0; i < G; ++i) {
      if (Lg[i] < 0 && (i64)n_of(cur, i) <= (i64)o.threshold_factor * kv[i]) Lg[i] = l;
      any |= Lg[i] < 0;
    }
    if (!any || (i32)lv.size() >= kMaxLevels) break;
    std::vector<i32> frozen(G);
    bool redo = true;
    CoarsenOut co;
    ULevel nx;
    while (redo) {
      for (i32 i = 0; i < G; ++i) frozen[i] = Lg[i] >= 0 ? 1 : 0;
      GKW_CUDA(cudaMemcpyAsync(frozen_d, frozen.data(), sizeof(i32) * G, cudaMemcpyHostToDevice, hh.stream));
      const Pool::Mark mk = hh.hier.mark();
      const Pool::Mark mks = hh.scratch.mark();
      co = CoarsenOut();
      coarsen_level(hh, cur.g, o.group_cap, co, cur.gid, frozen_d);
      // coarse ids of a graph form one contiguous block
      i32* cmin = hh.scratch.alloc_n<i32>(G);
      i32* cmax = hh.scratch.alloc_n<i32>(G);
      std::vector<i32> init_min(G, INT32_MAX), init_max(G, -1);
      GKW_CUDA(cudaMemcpyAsync(cmin, init_min.data(), sizeof(i32) * G, cudaMemcpyHostToDevice, hh.stream));
      GKW_CUDA(cudaMemcpyAsync(cmax, init_max.data(), sizeof(i32) * G, cudaMemcpyHostToDevice, hh.stream));
      launch(k_coarse_range, ceil_div(cur.g.n, 256), 256, 0, hh.stream, cur.g.n, cur.gid, co.cmap, cmin, cmax);
      GKW_CHECK_LAUNCH();
      const std::vector<i32> hmin = to_host(hh, cmin, G), hmax = to_host(hh, cmax, G);
      nx = ULevel();
      nx.gv.assign(G + 1, 0);
      i32 run = 0;
      for (i32 i = 0; i < G; ++i) {
        nx.gv[i] = run;
        if (n_of(cur, i) > 0) {
          GKW_REQUIRE(hmin[i] == run && hmax[i] >= hmin[i], GKW_E_INTERNAL, "batched coarsening mixed graphs");
          run = hmax[i] + 1;
        }
      }
      nx.gv[G] = run;
      GKW_REQUIRE(run == co.nc, GKW_E_INTERNAL, "batched coarsening lost vertices");
      nx.gv_d = to_dev(hh, nx.gv);
      nx.gid = hh.hier.alloc_n<i32>(std::max(co.nc, 1));
      if (co.nc) launch(k_fill_gid, ceil_div(co.nc, 256), 256, 0, hh.stream, co.nc, nx.gv_d, G, nx.gid);
      i32* mx = hh.scratch.alloc_n<i32>(G);
      GKW_CUDA(cudaMemsetAsync(mx, 0, sizeof(i32) * G, hh.stream));
      if (co.nc) launch(k_graph_maxw, ceil_div(co.nc, 256), 256, 0, hh.stream, co.nc, nx.gid, co.cvwgt, mx);
      GKW_CHECK_LAUNCH();
      const std::vector<i32> hmx = to_host(hh, mx, G);
      // the discard rules of each coarsening graph (graph_partitioner.hpp:93-96,
      // and the default mode's coarse-vertex stop)
      redo = false;
      for (i32 i = 0; i < G; ++i) {
        if (Lg[i] >= 0) continue;
        const i32 nn = n_of(cur, i), nc = nx.gv[i + 1] - nx.gv[i];
        bool stop = nc == nn || nc < kv[i] + 1;
        if (o.enforce_balance && o.coarse_vertex_frac > 0 &&
            (double)hmx[i] > o.coarse_vertex_frac * (double)Wg[i] / (double)kv[i])
          stop = true;
        if (stop) {
          Lg[i] = l;
          redo = true;
        }
      }
      hh.scratch.release(mks);
      if (redo) hh.hier.release(mk);   // build the level again with those graphs frozen
    }
    bool still = false, any_frozen = false;
    for (i32 i = 0; i < G; ++i) {
      still |= Lg[i] < 0;
      any_frozen |= Lg[i] >= 0 && n_of(cur, i) > 0;
    }
    if (!still) break;   // every graph stopped at this level: the coarse level is not needed
    if (l == 0 && any_frozen) {
      i32* bad = hh.scratch.alloc_n<i32>(1);
      GKW_CUDA(cudaMemsetAsync(bad, 0, sizeof(i32), hh.stream));
      launch(k_copy_frozen, ceil_div(cur.g.n, 256), 256, 0, hh.stream, cur.g.n, cur.gid, frozen_d, cur.g.xadj,
             cur.g.adjncy, cur.g.adjwgt, co.cmap, co.cxadj, co.cadjncy, co.cadjwgt, bad);
      GKW_CHECK_LAUNCH();
      if (to_host(hh, bad, 1)[0]) return false;   // duplicate edges: partition graph by graph
    }
    cur.cmap = co.cmap;
    nx.g.n = co.nc;
    nx.g.m = co.mc;
    nx.g.xadj = co.cxadj;
    nx.g.adjncy = co.cadjncy;
    nx.g.adjwgt = co.cadjwgt;
    nx.g.vwgt = co.cvwgt;
    lv.push_back(std::move(nx));
  }
  const i32 D = (i32)lv.size() - 1;
  for (i32 i = 0; i < G; ++i)
    if (Lg[i] < 0) Lg[i] = D;   // level cap reached

  // ---- initial partition on the deepest level ----
  const ULevel& deep = lv[D];
  RefineCtx* rc = refine_create(hh, std::max((i32)n, 1), K, o.move_cap, kmax);
  struct CtxGuard {
    RefineCtx* c;
    ~CtxGuard() { refine_destroy(c); }
  } cguard{rc};
  i32* cpart = refine_part(rc);
  std::vector<i32> pv0(K), pv1(K);
  for (i32 i = 0; i < G; ++i)
    for (i32 q = 0; q < kv[i]; ++q) {
      pv0[pb[i] + q] = deep.gv[i];
      pv1[pb[i] + q] = deep.gv[i + 1];
    }
  GggpBatch gb;
  gb.part_v0 = to_dev(hh, pv0);
  gb.part_v1 = to_dev(hh, pv1);
  gb.gid = deep.gid;
  gb.gpbase = gpb_d;
  gb.gk = gk_d;
  gb.part_base = pbase_d;
  gb.depth = depth;
  device_init_partition(hh, deep.g, K, o.eps, o.seed, std::max(1, std::min(8, o.init_trials)), cpart, &gb);
  refine_init_coarsest(hh, rc, deep.g, cpart);

  // per-round batch state
  i32* gcc = hh.hier.alloc_n<i32>(G);
  i32* glight = hh.hier.alloc_n<i32>(G);
  i32* mcount = hh.hier.alloc_n<i32>(1);
  i32* anyf = hh.hier.alloc_n<i32>(3);
  std::vector<i32*> gflags_d(lv.size());
  auto level_job = [&](i32 L, const std::vector<i32>& flags, BatchLevel& bl) {
    gflags_d[L] = to_dev(hh, flags);
    bl.G = G;
    bl.gid = lv[L].gid;
    bl.gvbase = lv[L].gv_d;
    bl.gpbase = gpb_d;
    bl.gk = gk_d;
    bl.gflags = gflags_d[L];
    bl.pmaxw = pmaxw_d;
    bl.pbcap = pbcap_d;
    bl.gcc = gcc;
    bl.glight = glight;
    bl.mcount = mcount;
    bl.anyf = anyf;
    GKW_CUDA(cudaMemsetAsync(gcc, 0, sizeof(i32) * G, hh.stream));
    GKW_CUDA(cudaMemsetAsync(mcount, 0, sizeof(i32), hh.stream));
    GKW_CUDA(cudaMemsetAsync(anyf, 0, sizeof(i32) * 3, hh.stream));
  };
  // default mode: balance rounds at every level of a graph but its
  // balance_skip_levels coarsest ones, and always at its input level
  // (partitioner.cu).  A graph's coarsest level is identical to the deepest
  // union level, where its coarsest balance runs.
  auto balances = [&](i32 i, i32 L) {
    return o.enforce_balance && (L == 0 || L < Lg[i] + 1 - std::max(0, o.balance_skip_levels));
  };
  {
    std::vector<i32> flags(G, 0);
    bool anyb = false;
    for (i32 i = 0; i < G; ++i)
      if (balances(i, Lg[i])) {
        flags[i] = 2;
        anyb = true;
      }
    if (anyb) {
      BatchLevel bl;
      level_job(D, flags, bl);
      LevelJob j;
      j.balance = true;
      j.move_cap = o.move_cap;
      j.batch = &bl;
      level_run(hh, rc, deep.g, j, D);
    }
  }
  // ---- uncoarsening ----
  for (i32 L = D - 1; L >= 0; --L) {
    std::vector<i32> flags(G, 0);
    bool anyr = false, anyb = false;
    for (i32 i = 0; i < G; ++i)
      if (L < Lg[i]) {
        flags[i] = balances(i, L) ? 3 : 1;
        anyr = true;
        anyb |= flags[i] == 3;
      }
    BatchLevel bl;
    level_job(L, flags, bl);
    LevelJob j;
    j.cmap = lv[L].cmap;
    j.balance = anyb;
    j.refine = anyr;
    j.move_cap = o.move_cap;
    j.batch = &bl;
    level_run(hh, rc, lv[L].g, j, L);
  }
  level_stats(hh, rc, (i32)lv.size());   // error words of the level kernels

  // ---- output: each graph's own part ids and cut ----
  const i32* part = refine_part(rc);
  i32* loc = hh.hier.alloc_n<i32>(n);
  launch(k_local_parts, ceil_div(n, 256), 256, 0, hh.stream, (i32)n, lv[0].gid, gpb_d, part, loc);
  unsigned long long* cut = hh.scratch.alloc_n<unsigned long long>(G);
  GKW_CUDA(cudaMemsetAsync(cut, 0, sizeof(u64) * G, hh.stream));
  launch(k_graph_cut, ceil_div(n, 256), 256, 0, hh.stream, (i32)n, x, a, w, lv[0].gid, part, cut);
  GKW_CHECK_LAUNCH();
  GKW_CUDA(cudaMemcpyAsync(part_out, loc, sizeof(i32) * n, cudaMemcpyDeviceToHost, hh.stream));
  const std::vector<unsigned long long> hc = to_host(hh, cut, G);
  if (cuts_out)
    for (i32 i = 0; i < G; ++i) cuts_out[i] = (i64)hc[i];
  return true;
}

}  // namespace gkw
