// Batched partitioning of many independent graphs as one disjoint union.
//
// Every step of the pipeline is a rule on a vertex's own neighbourhood, on its
// union-find component, or on one graph's parts, so it can run over the union
// of many graphs at once and give each graph exactly its lone result:
//
//   * coarsening: matching, union-find labels (max id of the component, hop
//     distance from it), the (root, dist, id) group order and the contraction
//     never mix graphs, and the coarse ids of a graph stay one contiguous,
//     identically ordered block.  The stop rules are checked per graph.  A
//     union level holds only the graphs still present at that depth: a graph
//     that stops at level l is left out of level l + 1 (its block is dropped
//     by a gather), so the union's work is the sum of the lone runs' work.
//   * initial partition: the coarsest level of every graph, wherever it is in
//     the union's hierarchy, is gathered into one coarsest union, partitioned
//     by GGGP with global part ids (graph g owns [pbase[g], pbase[g] + k[g]));
//     seeds use the graph's own part ids.
//   * uncoarsening: one level-kernel launch per union level.  A graph whose
//     coarsest level this is enters there: its vertices take their initial
//     part (cmap < 0 points into the coarsest union) and run the balance
//     rounds of a coarsest level; the other graphs project, refine and
//     balance.  Candidate order, move cap, balanced prefix and end of rounds
//     are per graph (refine.cu, batched levels).
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

// Per graph: range of its coarse ids and its heaviest coarse vertex.
__global__ void k_coarse_stats(i32 n, const i32* __restrict__ gid, const i32* __restrict__ cmap,
                               const i32* __restrict__ cvwgt, i32* __restrict__ cmin, i32* __restrict__ cmax,
                               i32* __restrict__ mx) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 g = gid[v], c = cmap[v];
  atomicMin(cmin + g, c);
  atomicMax(cmax + g, c);
  atomicMax(mx + g, cvwgt[c]);
}

// out[g] = xadj[gv[g]] for g in [0, G]: the edge offset of each graph's block.
__global__ void k_edge_bounds(i32 G, const i32* __restrict__ gv, const i32* __restrict__ xadj, i32* __restrict__ out) {
  const i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (g <= G) out[g] = xadj[gv[g]];
}

// Gather of whole graph blocks: vertex v of graph g (dv[g] >= 0) goes to
// dv[g] + (v - sgv[g]), its row to de[g] + (xadj[v] - xadj[sgv[g]]), its
// neighbour ids shifted by dv[g] - sgv[g].  Rows keep their order.
__global__ void k_gather_blocks(i32 n, const i32* __restrict__ gid, const i32* __restrict__ sgv,
                                const i32* __restrict__ dv, const i32* __restrict__ de,
                                const i32* __restrict__ xadj, const i32* __restrict__ adjncy,
                                const i32* __restrict__ adjwgt, const i32* __restrict__ vwgt,
                                i32* __restrict__ oxadj, i32* __restrict__ oadjncy, i32* __restrict__ oadjwgt,
                                i32* __restrict__ ovwgt) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 g = gid[v], d = dv[g];
  if (d < 0) return;
  const i32 s0 = sgv[g], shift = d - s0;
  const i32 nv = (i32)v + shift;
  const i32 e0 = xadj[v], e1 = xadj[v + 1];
  const i32 o = e0 - xadj[s0] + de[g];
  oxadj[nv] = o;
  ovwgt[nv] = vwgt[v];
  for (i32 e = e0; e < e1; ++e) {
    oadjncy[o + (e - e0)] = adjncy[e] + shift;
    oadjwgt[o + (e - e0)] = adjwgt[e];
  }
}

__global__ void k_set_i32(i32* p, i32 v) { *p = v; }

// cmap of a union level: vertices of graphs that continue (sd[g] is the
// offset from this level's block to the coarsened source block, cd[g] from
// the coarse block to the next level's block; kept[g]) take their coarse id
// in the next level.
__global__ void k_compose_cmap(i32 n, const i32* __restrict__ gid, const i32* __restrict__ kept,
                               const i32* __restrict__ sd, const i32* __restrict__ cd,
                               const i32* __restrict__ scmap, i32* __restrict__ cmap) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 g = gid[v];
  if (kept[g]) cmap[v] = scmap[(i32)v + sd[g]] + cd[g];
}

// Vertices of graphs whose coarsest level this is (cu[g] >= 0): cmap < 0
// names the vertex's place in the coarsest union, -(1 + index).
__global__ void k_enter_cmap(i32 n, const i32* __restrict__ gid, const i32* __restrict__ gv,
                             const i32* __restrict__ cu, i32* __restrict__ cmap) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 g = gid[v], c = cu[g];
  if (c >= 0) cmap[v] = -1 - ((i32)v - gv[g] + c);
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

// One level of the union: the graphs present at this depth, each a block.
struct ULevel {
  DevGraph g;
  i32* cmap = nullptr;   // to the next level (continuing graphs) or into the coarsest union
  i32* gid = nullptr;    // [n]
  std::vector<i32> gv;   // [G + 1] vertex offsets (host; empty block: graph absent)
  std::vector<i32> ge;   // [G + 1] edge offsets (host)
  i32* gv_d = nullptr;   // [G + 1] (device)
  i32 n_of(i32 i) const { return gv[i + 1] - gv[i]; }
};

// Fills gv_d, gid and ge of a level whose g and gv are set.
void finish_level(Handle& hh, ULevel& L, i32 G) {
  L.gv_d = to_dev(hh, L.gv);
  L.gid = hh.hier.alloc_n<i32>(std::max(L.g.n, 1));
  if (L.g.n) launch(k_fill_gid, ceil_div(L.g.n, 256), 256, 0, hh.stream, L.g.n, L.gv_d, G, L.gid);
  i32* eb = hh.scratch.alloc_n<i32>(G + 1);
  launch(k_edge_bounds, ceil_div(G + 1, 256), 256, 0, hh.stream, G, L.gv_d, L.g.xadj, eb);
  GKW_CHECK_LAUNCH();
  L.ge = to_host(hh, eb, G + 1);
}

// Gathers the blocks of src whose dst_v[g] >= 0 into dst arrays at the given
// vertex / edge offsets.
void gather_blocks(Handle& hh, const ULevel& src, const std::vector<i32>& dst_v, const std::vector<i32>& dst_e,
                   i32* ox, i32* oa, i32* ow, i32* ovw) {
  if (src.g.n == 0) return;
  i32* dv = to_dev(hh, dst_v);
  i32* de = to_dev(hh, dst_e);
  launch(k_gather_blocks, ceil_div(src.g.n, 256), 256, 0, hh.stream, src.g.n, src.gid, src.gv_d, dv, de, src.g.xadj,
         src.g.adjncy, src.g.adjwgt, src.g.vwgt, ox, oa, ow, ovw);
  GKW_CHECK_LAUNCH();
}

// The union of src's graphs with keep[g], block order kept.
ULevel compact(Handle& hh, const ULevel& src, const std::vector<char>& keep, i32 G) {
  ULevel d;
  d.gv.assign(G + 1, 0);
  std::vector<i32> dv(G, -1), de(G, 0);
  i64 nv = 0, ne = 0;
  for (i32 i = 0; i < G; ++i) {
    d.gv[i] = (i32)nv;
    if (keep[i]) {
      dv[i] = (i32)nv;
      de[i] = (i32)ne;
      nv += src.n_of(i);
      ne += src.ge[i + 1] - src.ge[i];
    }
  }
  d.gv[G] = (i32)nv;
  i32* x = hh.hier.alloc_n<i32>(nv + 1);
  i32* a = hh.hier.alloc_n<i32>(std::max<i64>(ne, 1));
  i32* w = hh.hier.alloc_n<i32>(std::max<i64>(ne, 1));
  i32* vw = hh.hier.alloc_n<i32>(std::max<i64>(nv, 1));
  gather_blocks(hh, src, dv, de, x, a, w, vw);
  launch(k_set_i32, 1, 1, 0, hh.stream, x + nv, (i32)ne);
  GKW_CHECK_LAUNCH();
  d.g.n = (i32)nv;
  d.g.m = ne;
  d.g.xadj = x;
  d.g.adjncy = a;
  d.g.adjwgt = w;
  d.g.vwgt = vw;
  finish_level(hh, d, G);
  return d;
}

}  // namespace

bool partition_batch_union(Handle& hh, const DevGraph& hg, i32 G, const i32* graph_ptr, const i32* ks,
                           const gkw_options& o, i32* part_out, i64* cuts_out, i32* levels_out) {
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
    for (i32 i = 0; i < G; ++i) {
      if (cuts_out) cuts_out[i] = 0;
      if (levels_out) levels_out[i] = 1;
    }
    return true;
  }
  i32* gk_d = to_dev(hh, kv);
  i32* gpb_d = to_dev(hh, pb);
  i32* pbase_d = to_dev(hh, part_base);
  std::vector<ULevel> lv(1);
  lv[0].g = g0;
  lv[0].gv.assign(graph_ptr, graph_ptr + G + 1);
  finish_level(hh, lv[0], G);
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

  // ---- coarsening (graph_partitioner.hpp:66-105, per graph) ----
  std::vector<i32> Lg(G, -1);   // coarsest level of each graph (-1: still coarsening)
  for (;;) {
    const i32 l = (i32)lv.size() - 1;
    bool any = false;
    for (i32 i = 0; i < G; ++i) {
      if (Lg[i] < 0 && (i64)lv[l].n_of(i) <= (i64)o.threshold_factor * kv[i]) Lg[i] = l;
      any |= Lg[i] < 0;
    }
    if (!any) break;
    if ((i32)lv.size() >= kMaxLevels) {
      for (i32 i = 0; i < G; ++i)
        if (Lg[i] < 0) Lg[i] = l;
      break;
    }
    // the source of this step: the graphs still coarsening
    std::vector<char> keepS(G);
    bool all = true;
    for (i32 i = 0; i < G; ++i) {
      keepS[i] = Lg[i] < 0;
      all &= keepS[i] || lv[l].n_of(i) == 0;
    }
    ULevel S_own;
    if (!all) S_own = compact(hh, lv[l], keepS, G);
    const ULevel& S = all ? lv[l] : S_own;
    CoarsenOut co;
    coarsen_level(hh, S.g, o.group_cap, co);
    // per graph: its block of coarse ids and its heaviest coarse vertex
    std::vector<i32> init3(3 * (size_t)G);
    for (i32 i = 0; i < G; ++i) {
      init3[i] = INT32_MAX;
      init3[G + i] = -1;
      init3[2 * G + i] = 0;
    }
    i32* st3 = to_dev(hh, init3);
    if (S.g.n)
      launch(k_coarse_stats, ceil_div(S.g.n, 256), 256, 0, hh.stream, S.g.n, S.gid, co.cmap, co.cvwgt, st3, st3 + G,
             st3 + 2 * G);
    GKW_CHECK_LAUNCH();
    const std::vector<i32> h3 = to_host(hh, st3, 3 * (size_t)G);
    ULevel C;
    C.gv.assign(G + 1, 0);
    i32 run = 0;
    for (i32 i = 0; i < G; ++i) {
      C.gv[i] = run;
      if (S.n_of(i) > 0) {
        GKW_REQUIRE(h3[i] == run && h3[G + i] >= h3[i], GKW_E_INTERNAL, "batched coarsening mixed graphs");
        run = h3[G + i] + 1;
      }
    }
    C.gv[G] = run;
    GKW_REQUIRE(run == co.nc, GKW_E_INTERNAL, "batched coarsening lost vertices");
    // the discard rules of each coarsening graph (graph_partitioner.hpp:93-96),
    // and the default mode's coarse-vertex stop
    std::vector<char> keepC(G, 0);
    bool allC = true, anyC = false;
    for (i32 i = 0; i < G; ++i) {
      if (!keepS[i]) continue;
      const i32 nn = S.n_of(i), nc = C.n_of(i);
      bool stop = nc == nn || nc < kv[i] + 1;
      if (o.enforce_balance && o.coarse_vertex_frac > 0 &&
          (double)h3[2 * G + i] > o.coarse_vertex_frac * (double)Wg[i] / (double)kv[i])
        stop = true;
      if (stop) Lg[i] = l;
      keepC[i] = !stop;
      allC &= !stop || nc == 0;
      anyC |= !stop;
    }
    if (!anyC) break;   // every graph stopped at this level: the coarse level is not needed
    C.g.n = co.nc;
    C.g.m = co.mc;
    C.g.xadj = co.cxadj;
    C.g.adjncy = co.cadjncy;
    C.g.adjwgt = co.cadjwgt;
    C.g.vwgt = co.cvwgt;
    finish_level(hh, C, G);
    const std::vector<i32> cgv = C.gv;   // coarse blocks before the stopped graphs are dropped
    ULevel next = allC ? std::move(C) : compact(hh, C, keepC, G);
    // cmap of this level for the graphs that continue
    ULevel& cur = lv[l];
    cur.cmap = hh.hier.alloc_n<i32>(std::max(cur.g.n, 1));
    std::vector<i32> kept(G), sd(G), cd(G);
    for (i32 i = 0; i < G; ++i) {
      kept[i] = keepC[i];
      sd[i] = S.gv[i] - cur.gv[i];
      cd[i] = next.gv[i] - cgv[i];
    }
    i32* kd = to_dev(hh, kept);
    i32* sdd = to_dev(hh, sd);
    i32* cdd = to_dev(hh, cd);
    launch(k_compose_cmap, ceil_div(cur.g.n, 256), 256, 0, hh.stream, cur.g.n, cur.gid, kd, sdd, cdd, co.cmap,
           cur.cmap);
    GKW_CHECK_LAUNCH();
    lv.push_back(std::move(next));
  }
  const i32 D = (i32)lv.size() - 1;
  for (i32 i = 0; i < G; ++i)
    if (Lg[i] < 0) Lg[i] = D;

  // ---- the coarsest union: each graph's coarsest level, in graph order ----
  std::vector<i32> cu_gv(G + 1, 0), cu_ge(G + 1, 0);
  {
    i64 rn = 0, re = 0;
    for (i32 i = 0; i < G; ++i) {
      cu_gv[i] = (i32)rn;
      cu_ge[i] = (i32)re;
      const ULevel& L = lv[Lg[i]];
      rn += L.n_of(i);
      re += L.ge[i + 1] - L.ge[i];
    }
    cu_gv[G] = (i32)rn;
    cu_ge[G] = (i32)re;
  }
  ULevel cu;
  cu.gv = cu_gv;
  {
    const i32 ncu = cu_gv[G], mcu = cu_ge[G];
    i32* cx = hh.hier.alloc_n<i32>(ncu + 1);
    i32* ca = hh.hier.alloc_n<i32>(std::max(mcu, 1));
    i32* cw = hh.hier.alloc_n<i32>(std::max(mcu, 1));
    i32* cvw = hh.hier.alloc_n<i32>(std::max(ncu, 1));
    for (i32 l = 0; l <= D; ++l) {
      std::vector<i32> dv(G, -1), de(G, 0), cuv(G, -1);
      bool anyl = false;
      for (i32 i = 0; i < G; ++i)
        if (Lg[i] == l) {
          dv[i] = cu_gv[i];
          de[i] = cu_ge[i];
          cuv[i] = cu_gv[i];
          anyl = true;
        }
      if (!anyl) continue;
      gather_blocks(hh, lv[l], dv, de, cx, ca, cw, cvw);
      // cmap of the entering vertices: their place in the coarsest union
      if (!lv[l].cmap) lv[l].cmap = hh.hier.alloc_n<i32>(std::max(lv[l].g.n, 1));
      i32* cud = to_dev(hh, cuv);
      launch(k_enter_cmap, ceil_div(std::max(lv[l].g.n, 1), 256), 256, 0, hh.stream, lv[l].g.n, lv[l].gid,
             lv[l].gv_d, cud, lv[l].cmap);
      GKW_CHECK_LAUNCH();
    }
    launch(k_set_i32, 1, 1, 0, hh.stream, cx + ncu, mcu);
    GKW_CHECK_LAUNCH();
    cu.g.n = ncu;
    cu.g.m = mcu;
    cu.g.xadj = cx;
    cu.g.adjncy = ca;
    cu.g.adjwgt = cw;
    cu.g.vwgt = cvw;
    cu.gv_d = to_dev(hh, cu.gv);
    cu.gid = hh.hier.alloc_n<i32>(std::max(ncu, 1));
    if (ncu) launch(k_fill_gid, ceil_div(ncu, 256), 256, 0, hh.stream, ncu, cu.gv_d, G, cu.gid);
    GKW_CHECK_LAUNCH();
  }

  // ---- initial partition of the coarsest union ----
  RefineCtx* rc = refine_create(hh, std::max((i32)n, 1), K, o.move_cap, kmax);
  struct CtxGuard {
    RefineCtx* c;
    ~CtxGuard() { refine_destroy(c); }
  } cguard{rc};
  i32* part_cu = hh.hier.alloc_n<i32>(std::max(cu.g.n, 1));
  i32* bnd_cu = hh.hier.alloc_n<i32>(std::max(cu.g.n, 1));
  {
    std::vector<i32> pv0(K), pv1(K);
    for (i32 i = 0; i < G; ++i)
      for (i32 q = 0; q < kv[i]; ++q) {
        pv0[pb[i] + q] = cu_gv[i];
        pv1[pb[i] + q] = cu_gv[i + 1];
      }
    GggpBatch gb;
    gb.part_v0 = to_dev(hh, pv0);
    gb.part_v1 = to_dev(hh, pv1);
    gb.gid = cu.gid;
    gb.gpbase = gpb_d;
    gb.gk = gk_d;
    gb.part_base = pbase_d;
    gb.depth = depth;
    device_init_partition(hh, cu.g, K, o.eps, o.seed, std::max(1, std::min(8, o.init_trials)), part_cu, &gb);
  }
  refine_init_union(hh, rc, cu.g, part_cu, bnd_cu);   // boundary of the initial parts, part weights

  // per-round batch state
  i32* gcc = hh.hier.alloc_n<i32>(G);
  i32* glight = hh.hier.alloc_n<i32>(G);
  i32* mcount = hh.hier.alloc_n<i32>(1);
  i32* anyf = hh.hier.alloc_n<i32>(3);
  // default mode: balance rounds at every level of a graph but its
  // balance_skip_levels coarsest ones, and always at its input level
  // (partitioner.cu)
  auto balances = [&](i32 i, i32 L) {
    return o.enforce_balance && (L == 0 || L < Lg[i] + 1 - std::max(0, o.balance_skip_levels));
  };
  // ---- uncoarsening: one level-kernel launch per union level ----
  for (i32 L = D; L >= 0; --L) {
    std::vector<i32> flags(G, 0);
    bool anyr = false, anyb = false;
    for (i32 i = 0; i < G; ++i) {
      if (Lg[i] < L || lv[L].n_of(i) == 0) continue;   // not present at this level
      const i32 bal = balances(i, L) ? 2 : 0;
      if (Lg[i] == L) {
        flags[i] = 4 | bal;   // enters: initial parts, the coarsest level's balance rounds
      } else {
        flags[i] = 1 | bal;
        anyr = true;
      }
      anyb |= bal != 0;
    }
    BatchLevel bl;
    bl.G = G;
    bl.gid = lv[L].gid;
    bl.gvbase = lv[L].gv_d;
    bl.gpbase = gpb_d;
    bl.gk = gk_d;
    bl.gflags = to_dev(hh, flags);
    bl.pmaxw = pmaxw_d;
    bl.pbcap = pbcap_d;
    bl.gcc = gcc;
    bl.glight = glight;
    bl.mcount = mcount;
    bl.anyf = anyf;
    bl.part_init = part_cu;
    bl.bnd_init = bnd_cu;
    GKW_CUDA(cudaMemsetAsync(gcc, 0, sizeof(i32) * G, hh.stream));
    GKW_CUDA(cudaMemsetAsync(mcount, 0, sizeof(i32), hh.stream));
    GKW_CUDA(cudaMemsetAsync(anyf, 0, sizeof(i32) * 3, hh.stream));
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
  for (i32 i = 0; i < G; ++i) {
    if (cuts_out) cuts_out[i] = (i64)hc[i];
    if (levels_out) levels_out[i] = Lg[i] + 1;
  }
  return true;
}

}  // namespace gkw
