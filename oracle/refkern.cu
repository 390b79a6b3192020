// Reference-kernel checker (test infrastructure only; nothing in the product
// links it).
//
// Runs the reference's own CUDA kernels -- copied unchanged out of
// gkway/coarsen.hpp and gkway/uncoarsen.hpp into _ref/refkern_src.cuh by
// refkern_extract.py at build time -- on small graphs, so that the tests can
// compare the oracle's restatement of each rule with the reference's code:
//
//   rk_match            matching_with_score            coarsen.hpp:39-78
//   rk_union_find       init_group_id + HEC_union_find loop   :351-359, 80-118, 461-469
//   rk_group_map        count_coarsen_group, init_group_ptr, breakdown_large_group,
//                       count_num_coarsen_vertex, construct_cmap   :361-406, 120-155, 408-421, 471-481
//   rk_coarse_vwgt      cal_coarsen_vwgt               :157-171
//   rk_contract         construct_tmp_adjp, copied_adjncy, HEC_remove_duplicate_edge,
//                       construct_coarsen_graph        :173-349
//   rk_expand           expand_partition               uncoarsen.hpp:325-356
//   rk_update_vertex_info  update_vertex_info + calculate_gain   :82-109, 175-237
//   rk_refine           one level's refinement loop    :427-506, with find_mv_wgt_sequence,
//                       find_balance_sequence, apply_sequence_move (:239-323) and
//                       update_vertex_info on the device
//   rk_partition        the whole of graph_partitioner() (graph_partitioner.hpp:14-220)
//   rk_cutsize          calculate_cutsize              uncoarsen.hpp:398-424
//
// What runs on the host instead, and why:
//   * ModernGPU (scans, mergesort, segmented sort; not vendored in the
//     reference tree): its calls compute plain inclusive/exclusive sums and
//     ascending sorts (coarsen.hpp:325,338,342,412,415,476; uncoarsen.hpp:472),
//     done here with the standard library; the mergesort of group keys is taken
//     as stable.
//   * The per-part row scan `scan<<<k, 1024>>>` (uncoarsen.hpp:37-80) and
//     create_independent_move_buffer (:111-173) are not run: both leave a
//     kernel early and then wait at a block or warp barrier with the exited
//     threads in its mask.  Their rules (an inclusive sum per part row; the
//     candidate test) are applied on the host.
//   * HEC_union_find is launched with a block size that divides n, so that no
//     thread leaves before its __syncthreads.  Its labels (high bits) are
//     schedule-independent; its low bits depend on the schedule.  rk_partition
//     takes the union-find from a callback (the oracle's canonical schedule)
//     so that a whole run is deterministic.
//   * update_vertex_info keeps k counters per thread in a 12000-word shared
//     array with 128 threads per block (uncoarsen.hpp:192, :379-383): k must be
//     at most 93, as in the reference.
// Host arrays are 0-based int32 at this boundary (the kernels see 1-based ids).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "declarations.h"
#include "gkway/move_request.hpp"
#include "refkern_src.cuh"

namespace {

typedef unsigned u32;
typedef unsigned long long u64;

struct RkError {
  int code;
};

inline void ck(cudaError_t e) {
  if (e != cudaSuccess) throw RkError{(int)e};
}

template <class T>
struct Dev {
  T* p = nullptr;
  size_t n = 0;
  explicit Dev(size_t count) : n(count) { ck(cudaMalloc((void**)&p, sizeof(T) * std::max<size_t>(count, 1))); }
  Dev(const Dev&) = delete;
  Dev& operator=(const Dev&) = delete;
  ~Dev() { cudaFree(p); }
  void put(const T* h, size_t count) {
    if (count) ck(cudaMemcpy(p, h, sizeof(T) * count, cudaMemcpyHostToDevice));
  }
  void put(const std::vector<T>& h) { put(h.data(), h.size()); }
  void get(T* h, size_t count) const {
    if (count) ck(cudaMemcpy(h, p, sizeof(T) * count, cudaMemcpyDeviceToHost));
  }
  std::vector<T> get(size_t count) const {
    std::vector<T> h(count);
    get(h.data(), count);
    return h;
  }
  void zero(size_t count) {
    if (count) ck(cudaMemset(p, 0, sizeof(T) * count));
  }
};

constexpr u32 kThreads = THREAD_PER_BLOCK;   // 512, the reference's launch width
inline u32 blocks(u64 n) { return (u32)std::max<u64>(1, (n + kThreads - 1) / kThreads); }

inline void sync_check() {
  ck(cudaGetLastError());
  ck(cudaDeviceSynchronize());
}

void set_consts(u32 k, float maxw, u32 group_cap) {
  ck(cudaMemcpyToSymbol(D_NUM_PARTITIONS, &k, sizeof(u32)));
  ck(cudaMemcpyToSymbol(D_MAX_PARTITION_WGT, &maxw, sizeof(float)));
  ck(cudaMemcpyToSymbol(D_MAX_COARSEN_GROUP, &group_cap, sizeof(u32)));
}

// One level's CSR on the device in the reference's layout (1-based ids).
struct DevCsr {
  int n;
  Dev<u32> adjp, adjncy, adjwgt, vwgt;
  DevCsr(int n_, const int* xadj, const int* adjncy0, const int* adjwgt_, const int* vwgt_)
      : n(n_), adjp(n_ + 1), adjncy(xadj[n_]), adjwgt(xadj[n_]), vwgt(n_) {
    const int m = xadj[n];
    adjp.put(reinterpret_cast<const u32*>(xadj), n + 1);
    std::vector<u32> a(m);
    for (int e = 0; e < m; ++e) a[e] = (u32)adjncy0[e] + 1;
    adjncy.put(a);
    adjwgt.put(reinterpret_cast<const u32*>(adjwgt_), m);
    if (vwgt_) vwgt.put(reinterpret_cast<const u32*>(vwgt_), n);
  }
};

// Largest block size <= 512 that divides n: HEC_union_find returns for
// gid >= n before a __syncthreads, so every launched thread must be in range.
u32 exact_block(u32 n) {
  for (u32 b = std::min<u32>(n, 512); b > 1; --b)
    if (n % b == 0) return b;
  return 1;
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const RkError& e) {
    cudaGetLastError();
    return e.code ? e.code : -1;
  }
}

// Group order and coarse ids from union-find keys (high 32 bits: 1-based
// label, low 32 bits: iteration), coarsen.hpp:408-421 then 471-481.
int group_map_dev(int n, const std::vector<u64>& keys, int group_cap, Dev<u32>& cmap) {
  Dev<u64> group(n);
  Dev<u32> vid(n), head(n), ptr((size_t)n + 1);
  std::vector<u32> hv(n);
  std::iota(hv.begin(), hv.end(), 1u);
  group.put(keys);
  vid.put(hv);
  gk::count_coarsen_group<<<blocks(n), kThreads>>>(group.p, vid.p, head.p, n);
  sync_check();
  std::vector<u32> h = head.get(n);   // exclusive scan (coarsen.hpp:412)
  u32 roots = 0;
  for (int i = 0; i < n; ++i) {
    const u32 x = h[i];
    h[i] = roots;
    roots += x;
  }
  head.put(h);
  // stable sort of (key, vertex id) by key (coarsen.hpp:415)
  std::vector<u64> hk = keys;
  std::vector<u32> order(n);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](u32 a, u32 b) { return hk[a] < hk[b]; });
  std::vector<u64> sk(n);
  for (int i = 0; i < n; ++i) {
    sk[i] = hk[order[i]];
    hv[i] = order[i] + 1;
  }
  group.put(sk);
  vid.put(hv);
  gk::init_group_ptr<<<blocks(n), kThreads>>>(group.p, vid.p, head.p, ptr.p, roots, n);
  gk::breakdown_large_group<<<blocks(n), kThreads>>>(group.p, head.p, vid.p, ptr.p, n);
  sync_check();
  head.zero(n);
  gk::count_num_coarsen_vertex<<<blocks(n), kThreads>>>(group.p, vid.p, head.p, n);
  sync_check();
  h = head.get(n);   // inclusive scan (coarsen.hpp:476)
  for (int i = 1; i < n; ++i) h[i] += h[i - 1];
  const int nc = n ? (int)h[n - 1] : 0;
  head.put(h);
  gk::construct_cmap<<<blocks(n), kThreads>>>(head.p, vid.p, cmap.p, n);
  sync_check();
  return nc;
}

// Contraction (coarsen.hpp:302-349); cmap 1-based on the device.  Returns m_c.
u32 contract_dev(const DevCsr& g, u32 m, const Dev<u32>& cmap, u32 nc, Dev<u32>& cadjp, Dev<u32>& cadjncy,
                 Dev<u32>& cadjwgt) {
  const u32 n = (u32)g.n;
  Dev<u32> tmp_adjp((size_t)nc + 1), tmp_adjncy(m), tmp_adjwgt(m);
  tmp_adjp.zero((size_t)nc + 1);
  gk::construct_tmp_adjp<<<blocks(n), kThreads>>>(g.adjp.p, tmp_adjp.p, cmap.p, n);
  sync_check();
  std::vector<u32> tp = tmp_adjp.get((size_t)nc + 1);   // inclusive scan (:325)
  for (u32 i = 1; i <= nc; ++i) tp[i] += tp[i - 1];
  tmp_adjp.put(tp);
  cadjp.put(tp);   // running write positions of copied_adjncy (:331)
  gk::copied_adjncy<<<blocks(n), kThreads>>>(g.adjp.p, cadjp.p, tmp_adjp.p, g.adjncy.p, tmp_adjncy.p, g.adjwgt.p,
                                             tmp_adjwgt.p, cmap.p, n);
  sync_check();
  // segmented sort by neighbour id (:338); equal ids are summed next, so
  // their order within a segment does not matter
  std::vector<u32> ta = tmp_adjncy.get(m), tw = tmp_adjwgt.get(m);
  std::vector<std::pair<u32, u32>> seg;
  for (u32 c = 0; c < nc; ++c) {
    seg.clear();
    for (u32 e = tp[c]; e < tp[c + 1]; ++e) seg.emplace_back(ta[e], tw[e]);
    std::sort(seg.begin(), seg.end(), [](const std::pair<u32, u32>& a, const std::pair<u32, u32>& b) {
      return a.first < b.first;
    });
    for (u32 e = tp[c]; e < tp[c + 1]; ++e) {
      ta[e] = seg[e - tp[c]].first;
      tw[e] = seg[e - tp[c]].second;
    }
  }
  tmp_adjncy.put(ta);
  tmp_adjwgt.put(tw);
  cadjp.zero((size_t)nc + 1);
  gk::HEC_remove_duplicate_edge<<<blocks(n), kThreads>>>(g.adjwgt.p, tmp_adjp.p, tmp_adjncy.p, tmp_adjwgt.p,
                                                         cadjp.p, nc);
  sync_check();
  std::vector<u32> cp = cadjp.get((size_t)nc + 1);   // inclusive scan (:342)
  for (u32 i = 1; i <= nc; ++i) cp[i] += cp[i - 1];
  cadjp.put(cp);
  const u32 mc = cp[nc];
  gk::construct_coarsen_graph<<<blocks(n), kThreads>>>(cadjncy.p, cadjwgt.p, tmp_adjncy.p, tmp_adjwgt.p, cadjp.p,
                                                       tmp_adjp.p, nc);
  sync_check();
  return mc;
}

// uncoarsen.hpp:10-21 on the host (the candidate rule below needs it)
inline bool host_valid_move(u32 dest_w, u32 vw, float maxw) { return !((float)(dest_w + vw) > maxw); }

void update_dev(const DevCsr& g, Dev<u32>& part, Dev<u32>& bnd, Dev<int>& gain, Dev<u32>& target,
                Dev<u32>& updated) {
  const u32 per = 128;   // MAX_VERTEX_PER_BLOCK (uncoarsen.hpp:379, 496)
  gk::update_vertex_info<<<(g.n + per - 1) / per, per>>>(part.p, bnd.p, gain.p, target.p, g.adjncy.p, g.adjwgt.p,
                                                         g.adjp.p, updated.p, g.n);
  sync_check();
}

// The refinement loop of one level (uncoarsen.hpp:427-506) on device state.
int refine_dev(const DevCsr& g, int k, float maxw, int move_cap, Dev<u32>& part, Dev<u32>& bnd, Dev<int>& gain,
               Dev<u32>& target, Dev<u32>& updated, Dev<u32>& pw, long long* moves, long long* gain_sum) {
  const int n = g.n;
  const std::vector<u32> hx = g.adjp.get((size_t)n + 1);
  const std::vector<u32> ha = g.adjncy.get(hx[n]);
  const std::vector<u32> hvw = g.vwgt.get(n);
  Dev<mvRequest> buf(move_cap);
  Dev<int> delta((size_t)k * move_cap), op(1);
  Dev<u32> seq(move_cap), cutsize(1);
  cutsize.zero(1);
  int rounds = 0;
  for (long long guard = 0;; ++guard) {
    if (guard > 4ll * n + 64) throw RkError{-2};
    // create_independent_move_buffer (:111-173), on the host
    const std::vector<u32> hp = part.get(n), hb = bnd.get(n), ht = target.get(n), hpw = pw.get(k);
    const std::vector<int> hg = gain.get(n);
    updated.zero(n);   // :133 clears every vertex's flag
    std::vector<mvRequest> mv;
    for (int v = 0; v < n; ++v) {
      if (!hb[v] || hg[v] <= 0 || !host_valid_move(hpw[ht[v]], hvw[v], maxw)) continue;
      bool yield = false;
      for (u32 e = hx[v]; e < hx[v + 1] && !yield; ++e) {
        const u32 u = ha[e] - 1;
        if (hg[u] > 0 && host_valid_move(hpw[ht[u]], hvw[u], maxw) && (u32)v > u) yield = true;
      }
      if (yield) continue;
      mvRequest r;
      r.vertex_id = (u32)v + 1;
      r.source_partition = hp[v];
      r.des_partition = ht[v];
      r.gain = hg[v];
      mv.push_back(r);
    }
    if (mv.empty()) break;   // :466-468
    // mergesort with mvRequest::operator< (move_request.hpp:36-41), a total order
    std::sort(mv.begin(), mv.end(), [](mvRequest a, mvRequest b) { return a < b; });
    const u32 B = (u32)std::min<size_t>(mv.size(), (size_t)move_cap);   // :474-475
    buf.put(mv.data(), B);
    delta.zero((size_t)k * B);
    gk::find_mv_wgt_sequence<<<blocks(B), kThreads>>>(buf.p, delta.p, g.vwgt.p, B);
    sync_check();
    std::vector<int> hd = delta.get((size_t)k * B);   // scan<<<k, 1024>>> (:477): inclusive per part row
    for (int p = 0; p < k; ++p)
      for (u32 j = 1; j < B; ++j) hd[(size_t)p * B + j] += hd[(size_t)p * B + j - 1];
    delta.put(hd);
    op.zero(1);
    gk::find_balance_sequence<<<blocks(B), kThreads>>>(buf.p, delta.p, pw.p, seq.p, op.p, B);
    sync_check();
    int pos = 0;
    op.get(&pos, 1);
    gk::apply_sequence_move<<<blocks(B), kThreads>>>(buf.p, delta.p, part.p, pw.p, updated.p, g.vwgt.p, g.adjp.p,
                                                    g.adjncy.p, cutsize.p, op.p, B);
    sync_check();
    for (int j = 0; j <= pos; ++j) *gain_sum += mv[j].gain;
    *moves += pos + 1;
    ++rounds;
    update_dev(g, part, bnd, gain, target, updated);   // :494-498
  }
  return rounds;
}

}  // namespace

extern "C" {

typedef int (*rk_init_fn)(void* user, int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                          int k, int* part);
typedef int (*rk_uf_fn)(int n, const int* cand, int* root, int* dist);

int rk_device_count() {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return c;
}

int rk_match(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt, int* cand) {
  return guarded([&] {
    DevCsr g(n, xadj, adjncy, adjwgt, vwgt);
    Dev<u32> c(n);
    gk::matching_with_score<<<blocks(n), kThreads>>>(g.vwgt.p, g.adjp.p, g.adjncy.p, g.adjwgt.p, c.p, n);
    sync_check();
    std::vector<u32> h = c.get(n);
    for (int v = 0; v < n; ++v) cand[v] = (int)h[v] - 1;
  });
}

// keys[v] = (1-based label << 32) | iteration of the last raise; *launches =
// kernel launches of the loop (the last one sees no change).
int rk_union_find(int n, const int* cand, unsigned long long* keys, int* launches) {
  if (n < 1) return -3;
  return guarded([&] {
    Dev<u32> c(n), vid(n), chg(1);
    Dev<u64> group(n);
    std::vector<u32> hc(n);
    for (int v = 0; v < n; ++v) hc[v] = (u32)cand[v] + 1;
    c.put(hc);
    gk::init_group_id<<<blocks(n), kThreads>>>(group.p, vid.p, n);
    sync_check();
    const u32 b = exact_block((u32)n);
    u32 it = 1, changed = 1;
    int l = 0;
    while (changed) {
      if (l > n + 2) throw RkError{-2};
      chg.zero(1);
      gk::HEC_union_find<<<(u32)n / b, b>>>(c.p, group.p, chg.p, it, n);
      sync_check();
      chg.get(&changed, 1);
      ++it;
      ++l;
    }
    group.get(keys, n);
    *launches = l;
  });
}

int rk_group_map(int n, const unsigned long long* keys, int group_cap, int* cmap, int* nc) {
  return guarded([&] {
    set_consts(1, 0.f, (u32)group_cap);
    Dev<u32> cm(n);
    std::vector<u64> k(keys, keys + n);
    *nc = group_map_dev(n, k, group_cap, cm);
    std::vector<u32> h = cm.get(n);
    for (int v = 0; v < n; ++v) cmap[v] = (int)h[v] - 1;
  });
}

// Coarse vertex weights, cleared first (the reference leaves them uncleared, Q3).
int rk_coarse_vwgt(int n, const int* vwgt, const int* cmap, int nc, int* cvwgt) {
  return guarded([&] {
    Dev<u32> vw(n), cm(n), cv(nc);
    vw.put(reinterpret_cast<const u32*>(vwgt), n);
    std::vector<u32> h(n);
    for (int v = 0; v < n; ++v) h[v] = (u32)cmap[v] + 1;
    cm.put(h);
    cv.zero(nc);
    gk::cal_coarsen_vwgt<<<blocks(n), kThreads>>>(vw.p, cv.p, cm.p, n);
    sync_check();
    cv.get(reinterpret_cast<u32*>(cvwgt), nc);
  });
}

int rk_contract(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* cmap, int nc, int* cxadj,
                int* cadjncy, int* cadjwgt, long long* mc) {
  return guarded([&] {
    DevCsr g(n, xadj, adjncy, adjwgt, nullptr);
    const u32 m = (u32)xadj[n];
    Dev<u32> cm(n), cp((size_t)nc + 1), ca(m), cw(m);
    std::vector<u32> h(n);
    for (int v = 0; v < n; ++v) h[v] = (u32)cmap[v] + 1;
    cm.put(h);
    const u32 out = contract_dev(g, m, cm, (u32)nc, cp, ca, cw);
    cp.get(reinterpret_cast<u32*>(cxadj), (size_t)nc + 1);
    std::vector<u32> a = ca.get(out);
    for (u32 e = 0; e < out; ++e) cadjncy[e] = (int)a[e] - 1;
    cw.get(reinterpret_cast<u32*>(cadjwgt), out);
    *mc = out;
  });
}

int rk_expand(int n, const int* cmap, const int* part_c, const int* bnd_c, int nc, int* part, int* bnd, int* gain,
              int* target, int* updated) {
  return guarded([&] {
    Dev<u32> cm(n), pc(nc), bc(nc), p(n), b(n), t(n), u(n);
    Dev<int> gn(n);
    std::vector<u32> h(n);
    for (int v = 0; v < n; ++v) h[v] = (u32)cmap[v] + 1;
    cm.put(h);
    pc.put(reinterpret_cast<const u32*>(part_c), nc);
    bc.put(reinterpret_cast<const u32*>(bnd_c), nc);
    gk::expand_partition<<<blocks(n), kThreads>>>(pc.p, p.p, bc.p, b.p, cm.p, u.p, gn.p, t.p, n);
    sync_check();
    p.get(reinterpret_cast<u32*>(part), n);
    b.get(reinterpret_cast<u32*>(bnd), n);
    gn.get(gain, n);
    t.get(reinterpret_cast<u32*>(target), n);
    u.get(reinterpret_cast<u32*>(updated), n);
  });
}

int rk_update_vertex_info(int n, const int* xadj, const int* adjncy, const int* adjwgt, int k, const int* part,
                          const int* updated, int* bnd, int* gain, int* target) {
  if (k < 1 || k * 128 > MAX_SHARE_SIZE) return -3;   // the reference's shared array holds 128 * k words
  return guarded([&] {
    set_consts((u32)k, 0.f, 6);
    DevCsr g(n, xadj, adjncy, adjwgt, nullptr);
    Dev<u32> p(n), u(n), b(n), t(n);
    Dev<int> gn(n);
    p.put(reinterpret_cast<const u32*>(part), n);
    u.put(reinterpret_cast<const u32*>(updated), n);
    b.put(reinterpret_cast<const u32*>(bnd), n);
    gn.put(gain, n);
    t.put(reinterpret_cast<const u32*>(target), n);
    update_dev(g, p, b, gn, t, u);
    b.get(reinterpret_cast<u32*>(bnd), n);
    gn.get(gain, n);
    t.get(reinterpret_cast<u32*>(target), n);
  });
}

// One level, in place, with the calling convention of the oracle's
// orc_refine (pw as unsigned values in int64 slots).
int rk_refine(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt, int k, float maxw,
              int move_cap, int* part, int* boundary, int* gain, int* target, int* updated, long long* pw,
              long long* moves, long long* gain_sum, int do_initial_update, int* rounds) {
  if (k < 1 || k * 128 > MAX_SHARE_SIZE) return -3;
  if (move_cap < 1 || move_cap > MAX_MV_BUFFER_SIZE) return -4;   // d_mv_delta_partition_wgt holds 1024 * k
  return guarded([&] {
    set_consts((u32)k, maxw, 6);
    DevCsr g(n, xadj, adjncy, adjwgt, vwgt);
    Dev<u32> p(n), b(n), t(n), u(n), w(k);
    Dev<int> gn(n);
    p.put(reinterpret_cast<const u32*>(part), n);
    b.put(reinterpret_cast<const u32*>(boundary), n);
    gn.put(gain, n);
    t.put(reinterpret_cast<const u32*>(target), n);
    u.put(reinterpret_cast<const u32*>(updated), n);
    std::vector<u32> hw(k);
    for (int q = 0; q < k; ++q) hw[q] = (u32)pw[q];
    w.put(hw);
    if (do_initial_update) update_dev(g, p, b, gn, t, u);
    *moves = 0;
    *gain_sum = 0;
    *rounds = refine_dev(g, k, maxw, move_cap, p, b, gn, t, u, w, moves, gain_sum);
    p.get(reinterpret_cast<u32*>(part), n);
    b.get(reinterpret_cast<u32*>(boundary), n);
    gn.get(gain, n);
    t.get(reinterpret_cast<u32*>(target), n);
    u.get(reinterpret_cast<u32*>(updated), n);
    hw = w.get(k);
    for (int q = 0; q < k; ++q) pw[q] = hw[q];
  });
}

int rk_cutsize(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* part, long long* cut) {
  return guarded([&] {
    DevCsr g(n, xadj, adjncy, adjwgt, nullptr);
    Dev<u32> p(n), c(1);
    p.put(reinterpret_cast<const u32*>(part), n);
    c.zero(1);
    gk::calculate_cutsize<<<blocks(n), kThreads>>>(p.p, g.adjncy.p, g.adjwgt.p, g.adjp.p, c.p, n);
    sync_check();
    u32 h = 0;
    c.get(&h, 1);
    *cut = h;
  });
}

// The reference's whole partitioner (graph_partitioner.hpp:222-365) with its
// kernels: coarsening while n > 20k (:22, :66) with the level discarded when
// it makes no progress or leaves fewer than k + 1 vertices (:93-96), the
// initial partition from `init` on the coarsest level (METIS in the
// reference, metis_partition.hpp:46-71: part, part weights, boundary flags),
// then per finer level expand_partition + update_vertex_info (uncoarsen.hpp:
// 358-387) and the refinement loop, and the final cut (calculate_cutsize).
// The union-find labels come from `uf` (root: 0-based label, dist: low
// bits).  level_n/level_m receive the sizes of the kept levels (at most 64).
int rk_partition(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt, int k, rk_uf_fn uf,
                 rk_init_fn init, void* init_user, int* part_out, long long* cut_out, int* n_levels,
                 long long* level_n, long long* level_m, int* refine_rounds) {
  if (k < 1 || k * 128 > MAX_SHARE_SIZE) return -3;
  return guarded([&] {
    long long total = 0;
    for (int v = 0; v < n; ++v) total += (u32)vwgt[v];
    const float maxw = (float)((u32)total) / (float)k * (1.0f + IMBALANCE_RATIO) + 1;   // :230
    set_consts((u32)k, maxw, 6);
    struct HostLevel {
      int n;
      std::vector<int> xadj, adjncy, adjwgt, vwgt, cmap;
    };
    std::vector<HostLevel> lv(1);
    lv[0].n = n;
    lv[0].xadj.assign(xadj, xadj + n + 1);
    lv[0].adjncy.assign(adjncy, adjncy + xadj[n]);
    lv[0].adjwgt.assign(adjwgt, adjwgt + xadj[n]);
    lv[0].vwgt.assign(vwgt, vwgt + n);
    while (lv.back().n > 20 * k && lv.size() < 64) {
      HostLevel& f = lv.back();
      const int fn = f.n;
      DevCsr g(fn, f.xadj.data(), f.adjncy.data(), f.adjwgt.data(), f.vwgt.data());
      Dev<u32> cand(fn);
      gk::matching_with_score<<<blocks(fn), kThreads>>>(g.vwgt.p, g.adjp.p, g.adjncy.p, g.adjwgt.p, cand.p, fn);
      sync_check();
      std::vector<u32> hc = cand.get(fn);
      std::vector<int> c0(fn), root(fn), dist(fn);
      for (int v = 0; v < fn; ++v) c0[v] = (int)hc[v] - 1;
      uf(fn, c0.data(), root.data(), dist.data());
      std::vector<u64> keys(fn);
      for (int v = 0; v < fn; ++v) keys[v] = ((u64)((u32)root[v] + 1) << 32) | (u32)dist[v];
      Dev<u32> cm(fn);
      const int nc = group_map_dev(fn, keys, 6, cm);
      if (nc == fn || nc < k + 1) break;   // :93-96
      HostLevel c;
      c.n = nc;
      Dev<u32> cv(nc);
      cv.zero(nc);
      gk::cal_coarsen_vwgt<<<blocks(fn), kThreads>>>(g.vwgt.p, cv.p, cm.p, fn);
      sync_check();
      c.vwgt.resize(nc);
      cv.get(reinterpret_cast<u32*>(c.vwgt.data()), nc);
      const u32 m = (u32)f.xadj[fn];
      Dev<u32> cp((size_t)nc + 1), ca(m), cw(m);
      const u32 mc = contract_dev(g, m, cm, (u32)nc, cp, ca, cw);
      c.xadj.resize((size_t)nc + 1);
      cp.get(reinterpret_cast<u32*>(c.xadj.data()), (size_t)nc + 1);
      std::vector<u32> a = ca.get(mc);
      c.adjncy.resize(mc);
      for (u32 e = 0; e < mc; ++e) c.adjncy[e] = (int)a[e] - 1;
      c.adjwgt.resize(mc);
      cw.get(reinterpret_cast<u32*>(c.adjwgt.data()), mc);
      std::vector<u32> hcm = cm.get(fn);
      f.cmap.resize(fn);
      for (int v = 0; v < fn; ++v) f.cmap[v] = (int)hcm[v] - 1;
      lv.push_back(std::move(c));
    }
    *n_levels = (int)lv.size();
    for (size_t i = 0; i < lv.size(); ++i) {
      level_n[i] = lv[i].n;
      level_m[i] = (long long)lv[i].adjncy.size();
    }
    // initial partition (metis_partition.hpp:52-71)
    HostLevel& cs = lv.back();
    std::vector<int> cpart(cs.n);
    if (init(init_user, cs.n, cs.xadj.data(), cs.adjncy.data(), cs.adjwgt.data(), cs.vwgt.data(), k, cpart.data()))
      throw RkError{-5};
    std::vector<u32> hpw(k, 0), hb(cs.n, 0);
    for (int v = 0; v < cs.n; ++v) {
      if (cpart[v] < 0 || cpart[v] >= k) throw RkError{-6};
      hpw[cpart[v]] += (u32)cs.vwgt[v];
      for (int e = cs.xadj[v]; e < cs.xadj[v + 1]; ++e)
        if (cpart[cs.adjncy[e]] != cpart[v]) {
          hb[v] = 1;
          break;
        }
    }
    Dev<u32> pw(k);
    pw.put(hpw);
    std::vector<u32> cur_part(cpart.begin(), cpart.end()), cur_bnd = hb;
    for (int L = (int)lv.size() - 2; L >= 0; --L) {
      HostLevel& f = lv[L];
      const int fn = f.n, cn = lv[L + 1].n;
      DevCsr g(fn, f.xadj.data(), f.adjncy.data(), f.adjwgt.data(), f.vwgt.data());
      Dev<u32> cm(fn), pc(cn), bc(cn), p(fn), b(fn), t(fn), u(fn);
      Dev<int> gn(fn);
      std::vector<u32> h(fn);
      for (int v = 0; v < fn; ++v) h[v] = (u32)f.cmap[v] + 1;
      cm.put(h);
      pc.put(cur_part);
      bc.put(cur_bnd);
      gk::expand_partition<<<blocks(fn), kThreads>>>(pc.p, p.p, bc.p, b.p, cm.p, u.p, gn.p, t.p, fn);
      sync_check();
      update_dev(g, p, b, gn, t, u);
      long long moves = 0, gsum = 0;
      const int r = refine_dev(g, k, maxw, MAX_MV_BUFFER_SIZE, p, b, gn, t, u, pw, &moves, &gsum);
      if (L < 64) refine_rounds[L] = r;
      cur_part = p.get(fn);
      cur_bnd = b.get(fn);
    }
    for (int v = 0; v < n; ++v) part_out[v] = (int)cur_part[v];
    *cut_out = 0;
    DevCsr g0(n, xadj, adjncy, adjwgt, vwgt);
    Dev<u32> p0(n), c(1);
    p0.put(cur_part);
    c.zero(1);
    gk::calculate_cutsize<<<blocks(n), kThreads>>>(p0.p, g0.adjncy.p, g0.adjwgt.p, g0.adjp.p, c.p, n);
    sync_check();
    u32 hcut = 0;
    c.get(&hcut, 1);
    *cut_out = hcut;
  });
}

}  // extern "C"
