// TEST INFRASTRUCTURE ONLY -- the oracle.  Not part of the product: only the
// tests, the smoke check and the CPU-baseline leg of bench.py load this library,
// and only to check (or time beside) the CUDA path.  Nothing in the product
// links it.
//
// A single-threaded CPU restatement of G-kway's multilevel k-way partitioner
// (wanluanlee/DAC_g-kway), written from the reference's behaviour.  Every
// function cites the reference lines it follows.  Conventions:
//   * ids are 0-based here; the reference keeps 1-based ids on the device
//     (adjncy, cmap, vertex_id).  Every comparison the reference makes on ids
//     (max label, "u < v", sort by id) is invariant under the shift.
//   * all weights and ids are 32-bit unsigned, as in the reference.
//   * "det mode" fixes the one schedule-dependent step of the reference, the
//     low 32 bits of the union-find key (coarsen.hpp:103-111), to the Jacobi
//     schedule of the same kernel: every thread of an iteration reads the
//     previous iteration's keys.  Under that schedule the low bits equal the
//     hop distance from the component's root (the max id), root = 0.
//   * the reference's memory bugs take their intended semantics: coarse vertex
//     weights start at zero (graph_partitioner.hpp:270 / coarsen.hpp:170 never
//     clear them), the per-thread part flags of update_vertex_info have no k cap
//     (uncoarsen.hpp:192-204 overflows for k > 93), and a graph that is not
//     coarsened at all keeps its initial partition (graph_partitioner.hpp:172,
//     194-201 read an uninitialised size in that case).
//
// Parity pins: the initial partition calls the reference's bundled METIS 5.2.1
// (3rd-party/metis/libmetis.so, dlopen'd, link-and-call only), whose known
// answers on simple_test/delaunay_n11.graph are checked by the tests.  The
// reference's own GPU path cannot be built (its ModernGPU submodule is not
// vendored), so the G-kway steps themselves are pinned by this restatement plus
// the tests' hand-checked small cases.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <numeric>
#include <vector>

extern "C" {

typedef int32_t i32;
typedef uint32_t u32;
typedef int64_t i64;
typedef uint64_t u64;

// ---------------------------------------------------------------------------
// Phase A3: heavy-edge candidate with degree tie-break.
// coarsen.hpp:39-78 (matching_with_score).  Serial scan of the row: a strictly
// heavier edge always replaces the candidate; an equal-weight edge replaces it
// only if the neighbour's degree is strictly smaller.  The start state is
// (weight 0, degree 0, self), so zero-weight edges never win and an isolated
// vertex is its own candidate.
// ---------------------------------------------------------------------------
void orc_match(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, i32* cand) {
  for (i32 v = 0; v < n; ++v) {
    u32 best_w = 0, best_d = 0;
    i32 best = v;
    for (i32 e = xadj[v]; e < xadj[v + 1]; ++e) {
      u32 w = (u32)adjwgt[e];
      i32 u = adjncy[e];
      if (best_w < w) {                                   // coarsen.hpp:63-67
        best_w = w;
        best = u;
        best_d = (u32)(xadj[u + 1] - xadj[u]);
      } else if (best_w == w) {                           // coarsen.hpp:68-75
        u32 d = (u32)(xadj[u + 1] - xadj[u]);
        if (d < best_d) { best_d = d; best = u; }
      }
    }
    cand[v] = best;                                       // coarsen.hpp:77
  }
}

// ---------------------------------------------------------------------------
// Phase A4/A5: union-find label propagation over the edges {v, cand(v)}.
// coarsen.hpp:351-359 (init_group_id), 80-118 (HEC_union_find), 461-469 (host
// loop).  Key = (label << 32) | iteration-of-last-raise, raised by atomicMax.
// Jacobi schedule (det mode): iteration `it` reads only iteration it-1's keys.
// Returns the number of kernel launches the loop makes (the last one sees no
// change).  root[v] = final label (the max id of v's component), dist[v] = low
// bits (hop distance from the root under this schedule).
// ---------------------------------------------------------------------------
i32 orc_union_find(i32 n, const i32* cand, i32* root, i32* dist) {
  std::vector<u64> cur(n), nxt(n);
  for (i32 v = 0; v < n; ++v) cur[v] = ((u64)(u32)v << 32);   // coarsen.hpp:357
  i32 launches = 0;
  u64 it = 1;
  for (;;) {
    ++launches;
    bool changed = false;
    nxt = cur;
    for (i32 v = 0; v < n; ++v) {
      i32 c = cand[v];
      u32 a = (u32)(cur[v] >> 32), b = (u32)(cur[c] >> 32);
      if (a > b) {                                              // coarsen.hpp:103-107
        nxt[c] = std::max(nxt[c], ((u64)a << 32) | it);
        changed = true;
      } else if (a < b) {                                       // coarsen.hpp:108-112
        nxt[v] = std::max(nxt[v], ((u64)b << 32) | it);
        changed = true;
      }
    }
    cur.swap(nxt);
    ++it;
    if (!changed) break;                                        // coarsen.hpp:463
  }
  for (i32 v = 0; v < n; ++v) {
    root[v] = (i32)(u32)(cur[v] >> 32);
    dist[v] = (i32)(u32)(cur[v] & 0xffffffffu);
  }
  return launches;
}

// ---------------------------------------------------------------------------
// Phase A6/A7: order groups, cap them, assign coarse ids.
// coarsen.hpp:408-421 (constraint_group_size: count_coarsen_group, scan,
// mergesort, init_group_ptr, breakdown_large_group) and 120-155, 474-481
// (count_num_coarsen_vertex, inclusive scan, construct_cmap).
// Sorted order = (root, dist, id) ascending (the mergesort of (key, vertex_id)
// is taken as stable, so equal keys keep id order).  Each root's run is cut
// into consecutive chunks of `group_cap` (D_MAX_COARSEN_GROUP = 6,
// graph_partitioner.hpp:229); a chunk's coarse id is its rank among chunks in
// sorted order.  Returns n_c.  `order` (optional, n entries) receives the
// sorted vertex order.
// ---------------------------------------------------------------------------
i32 orc_group_map(i32 n, const i32* root, const i32* dist, i32 group_cap, i32* cmap, i32* order) {
  std::vector<i32> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](i32 x, i32 y) {
    if (root[x] != root[y]) return (u32)root[x] < (u32)root[y];
    return (u32)dist[x] < (u32)dist[y];
  });
  i32 nc = 0;
  i32 pos_in_group = 0;
  for (i32 i = 0; i < n; ++i) {
    i32 v = ord[i];
    if (i == 0 || root[ord[i - 1]] != root[v]) pos_in_group = 0;   // new group
    if (pos_in_group % group_cap == 0) ++nc;                        // chunk leader
    cmap[v] = nc - 1;                                               // coarsen.hpp:154
    ++pos_in_group;
    if (order) order[i] = v;
  }
  return nc;
}

// coarsen.hpp:157-171 (cal_coarsen_vwgt), with the coarse weights cleared first.
void orc_coarse_vwgt(i32 n, const i32* vwgt, const i32* cmap, i32 nc, i32* cvwgt) {
  std::fill(cvwgt, cvwgt + nc, 0);
  for (i32 v = 0; v < n; ++v) cvwgt[cmap[v]] = (i32)((u32)cvwgt[cmap[v]] + (u32)vwgt[v]);
}

// ---------------------------------------------------------------------------
// Phase A9: contraction.  coarsen.hpp:302-349 (contraction) with 173-187
// (construct_tmp_adjp), 189-218 (copied_adjncy), the segmented sort (:338),
// 246-300 (HEC_remove_duplicate_edge) and 220-244 (construct_coarsen_graph).
// Coarse row c = the multiset {cmap(u) : u in N(v), cmap(v) = c}, entries equal
// to c dropped, equal ids merged with their weights summed (32-bit), sorted
// ascending.  cxadj has nc+1 entries; cadjncy/cadjwgt need room for m entries.
// Returns m_c.
// ---------------------------------------------------------------------------
i64 orc_contract(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, const i32* cmap,
                 i32 nc, i32* cxadj, i32* cadjncy, i32* cadjwgt) {
  // members of each coarse vertex
  std::vector<i32> cnt(nc + 1, 0);
  for (i32 v = 0; v < n; ++v) cnt[cmap[v] + 1]++;
  for (i32 c = 0; c < nc; ++c) cnt[c + 1] += cnt[c];
  std::vector<i32> mem(n), fill(cnt.begin(), cnt.end() - 1);
  for (i32 v = 0; v < n; ++v) mem[fill[cmap[v]]++] = v;
  std::vector<std::pair<u32, u32>> row;
  i64 out = 0;
  cxadj[0] = 0;
  for (i32 c = 0; c < nc; ++c) {
    row.clear();
    for (i32 j = cnt[c]; j < cnt[c + 1]; ++j) {
      i32 v = mem[j];
      for (i32 e = xadj[v]; e < xadj[v + 1]; ++e)
        row.emplace_back((u32)cmap[adjncy[e]], (u32)adjwgt[e]);
    }
    std::sort(row.begin(), row.end(),
              [](const std::pair<u32, u32>& a, const std::pair<u32, u32>& b) { return a.first < b.first; });
    size_t i = 0;
    while (i < row.size()) {
      u32 l = row[i].first;
      if (l == (u32)c) { ++i; continue; }                    // coarsen.hpp:276-278
      u32 sum = 0;
      size_t j = i;
      while (j < row.size() && row[j].first == l) sum += row[j++].second;   // :280-291
      cadjncy[out] = (i32)l;
      cadjwgt[out] = (i32)sum;
      ++out;
      i = j;
    }
    cxadj[c + 1] = (i32)out;
  }
  return out;
}

// ---------------------------------------------------------------------------
// METIS (the reference's initial partitioner), dlopen'd from a path.
// metis_partition.hpp:4-99: METIS_PartGraphKway(n, ncon=1, xadj, adjncy, vwgt,
// vsize=NULL, adjwgt, k, tpwgts=NULL, ubvec=NULL, options=NULL, &cut, part),
// idx_t 64-bit (metis.h:33).
// ---------------------------------------------------------------------------
typedef int (*metis_kway_fn)(i64*, i64*, i64*, i64*, i64*, i64*, i64*, i64*, double*, double*,
                             i64*, i64*, i64*);
static metis_kway_fn g_metis = nullptr;
// METIS_PartGraphRecursive (metis.h:185), same arguments: the recursive-
// bisection alternative to the k-way initial partition.
static metis_kway_fn g_metis_rb = nullptr;

int orc_set_metis(const char* path) {
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return -1;
  g_metis = (metis_kway_fn)dlsym(h, "METIS_PartGraphKway");
  g_metis_rb = (metis_kway_fn)dlsym(h, "METIS_PartGraphRecursive");
  return g_metis ? 0 : -2;
}

int orc_has_metis() { return g_metis != nullptr; }

// One METIS partitioning call (k-way or recursive bisection) on 64-bit
// copies of the arrays.  Returns METIS's status (1 = METIS_OK).
static int metis_call(metis_kway_fn fn, i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt,
                      const i32* vwgt, i32 k, i32* part, i64* objval);

// Returns METIS's status (1 = METIS_OK) or -1 if METIS is not loaded.
int orc_metis_kway(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, const i32* vwgt,
                   i32 k, i32* part, i64* objval) {
  if (!g_metis) return -1;
  return metis_call(g_metis, n, xadj, adjncy, adjwgt, vwgt, k, part, objval);
}

// The same through METIS_PartGraphRecursive; -1 if it is not loaded.
int orc_metis_recursive(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, const i32* vwgt,
                        i32 k, i32* part, i64* objval) {
  if (!g_metis_rb) return -1;
  return metis_call(g_metis_rb, n, xadj, adjncy, adjwgt, vwgt, k, part, objval);
}

static int metis_call(metis_kway_fn fn, i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt,
                      const i32* vwgt, i32 k, i32* part, i64* objval) {
  i64 nv = n, ncon = 1, nparts = k, cut = 0;
  i64 m = xadj[n];
  std::vector<i64> x(n + 1), a(std::max<i64>(m, 1)), w(std::max<i64>(m, 1)), vw(std::max(n, 1)),
      p(std::max(n, 1));
  for (i32 i = 0; i <= n; ++i) x[i] = xadj[i];
  for (i64 e = 0; e < m; ++e) { a[e] = adjncy[e]; w[e] = adjwgt[e]; }
  for (i32 i = 0; i < n; ++i) vw[i] = vwgt[i];
  int rc = fn(&nv, &ncon, x.data(), a.data(), vw.data(), nullptr, w.data(), &nparts, nullptr,
              nullptr, nullptr, &cut, p.data());
  for (i32 i = 0; i < n; ++i) part[i] = (i32)p[i];
  if (objval) *objval = cut;
  return rc;
}

// ---------------------------------------------------------------------------
// Metrics.  uncoarsen.hpp:398-424 (calculate_cutsize: sum of adjwgt over u<v
// with different parts) and cuda_check.hpp:61-73 (calculate_partition_wgt).
// ---------------------------------------------------------------------------
i64 orc_cut(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, const i32* part) {
  i64 cut = 0;
  for (i32 v = 0; v < n; ++v)
    for (i32 e = xadj[v]; e < xadj[v + 1]; ++e)
      if (v < adjncy[e] && part[v] != part[adjncy[e]]) cut += (u32)adjwgt[e];
  return cut;
}

void orc_part_weights(i32 n, const i32* vwgt, const i32* part, i32 k, i64* pw) {
  std::fill(pw, pw + k, 0);
  for (i32 v = 0; v < n; ++v) pw[part[v]] += (u32)vwgt[v];
}

// graph_partitioner.hpp:230 -- MAX_PARTITION_WGT.  IMBALANCE_RATIO is a double
// literal (declarations.h:17), so (1.0f + 0.03) is evaluated in double, the
// product is double, and the result is stored as float.
float orc_max_part_weight(i64 total_vwgt, i32 k, double eps) {
  float q = (float)(u32)total_vwgt / (float)k;
  return (float)((double)q * (1.0 + eps) + 1);
}

// ---------------------------------------------------------------------------
// Refinement state for one level (uncoarsen.hpp).
// ---------------------------------------------------------------------------
struct RefineState {
  i32 n, k;
  const i32 *xadj, *adjncy, *adjwgt, *vwgt;
  float maxw;
  std::vector<u32> part, boundary, updated, target;
  std::vector<i32> gain;
  std::vector<u32> pw;   // part weights, unsigned as in the reference
};

// uncoarsen.hpp:10-21 (is_valid_move): (float)(dest weight + vwgt) <= MAXW.
static inline bool valid_move(u32 dest_w, u32 vw, float maxw) {
  float b = (float)(u32)(dest_w + vw);
  return !(b > maxw);
}

// uncoarsen.hpp:175-237 (update_vertex_info) with 82-109 (calculate_gain).
// The best part is kept with an UNSIGNED comparison of the int gain against an
// unsigned running max starting at 0 (uncoarsen.hpp:222,229): a negative gain
// compares as a large unsigned value.
static void update_vertex(RefineState& s, i32 v, std::vector<u32>& ed, std::vector<char>& seen,
                          std::vector<i32>& touched) {
  u32 p = s.part[v];
  bool bnd = false;
  touched.clear();
  u32 id = 0;
  for (i32 e = s.xadj[v]; e < s.xadj[v + 1]; ++e) {
    u32 q = s.part[s.adjncy[e]];
    if (q != p) bnd = true;                             // uncoarsen.hpp:209-211
    if (q == p) id += (u32)s.adjwgt[e];                 // uncoarsen.hpp:101-103
    if (!seen[q]) { seen[q] = 1; ed[q] = 0; touched.push_back((i32)q); }   // :208
    ed[q] += (u32)s.adjwgt[e];                          // uncoarsen.hpp:104-106
  }
  s.boundary[v] = bnd;
  if (!bnd) {                                           // uncoarsen.hpp:216-220
    s.gain[v] = 0;
    s.target[v] = p;
  } else {
    std::sort(touched.begin(), touched.end());          // parts scanned in increasing order (:225)
    u32 max_gain = 0, max_part = p;
    for (i32 q : touched) {
      if ((u32)q == p) continue;
      u32 g = ed[q] - id;                               // uncoarsen.hpp:108 (unsigned)
      if (g > max_gain) { max_gain = g; max_part = (u32)q; }   // :229-232
    }
    s.gain[v] = (i32)max_gain;                          // :235-236
    s.target[v] = max_part;
  }
  for (i32 q : touched) seen[q] = 0;
}

static void update_all_flagged(RefineState& s) {
  std::vector<u32> ed(s.k, 0);
  std::vector<char> seen(s.k, 0);
  std::vector<i32> touched;
  for (i32 v = 0; v < s.n; ++v)
    if (s.updated[v]) update_vertex(s, v, ed, seen, touched);
}

struct OrcMove { u32 v, src, des; i32 gain; };

// uncoarsen.hpp:427-506 (refinement).  One round per loop iteration:
// create_independent_move_buffer (:111-173), mergesort by (gain desc, id asc)
// (move_request.hpp:36-41), cap (:475), per-part prefix deltas (:239-257 and the
// scan at :37-80), the largest balanced prefix index (:259-288), apply
// (:290-323), update_vertex_info (:175-237).  Returns the number of rounds that
// applied moves; *moves receives the moved-vertex count, *cut_delta the sum of
// applied gains.
static i32 refine_level(RefineState& s, i32 move_cap, i64* moves, i64* gain_sum) {
  i32 rounds = 0;
  std::vector<OrcMove> buf;
  std::vector<i64> delta;   // delta[p * B + j]
  for (;;) {
    buf.clear();
    std::fill(s.updated.begin(), s.updated.end(), 0u);          // uncoarsen.hpp:133
    for (i32 v = 0; v < s.n; ++v) {
      if (!s.boundary[v]) continue;                              // :134
      i32 g = s.gain[v];
      if (g <= 0) continue;                                      // :140
      u32 t = s.target[v];
      if (!valid_move(s.pw[t], (u32)s.vwgt[v], s.maxw)) continue;   // :143-148
      bool yield = false;
      for (i32 e = s.xadj[v]; e < s.xadj[v + 1]; ++e) {         // :151-162
        i32 u = s.adjncy[e];
        if (s.gain[u] > 0 && valid_move(s.pw[s.target[u]], (u32)s.vwgt[u], s.maxw) && v > u) {
          yield = true;
          break;
        }
      }
      if (yield) continue;
      buf.push_back({(u32)v, s.part[v], t, g});
    }
    if (getenv("ORC_TRACE")) fprintf(stderr, "round n=%d cand=%zu\n", s.n, buf.size());
    if (buf.empty()) break;                                      // :466
    std::sort(buf.begin(), buf.end(), [](const OrcMove& a, const OrcMove& b) {
      if (a.gain != b.gain) return a.gain > b.gain;
      return a.v < b.v;
    });
    i32 B = (i32)std::min<size_t>(buf.size(), (size_t)move_cap);   // :475
    delta.assign((size_t)s.k * B, 0);
    for (i32 j = 0; j < B; ++j) {                                // :239-257
      delta[(size_t)buf[j].src * B + j] = -(i64)(u32)s.vwgt[buf[j].v];
      delta[(size_t)buf[j].des * B + j] = (i64)(u32)s.vwgt[buf[j].v];
    }
    for (i32 p = 0; p < s.k; ++p)                                // scan, :37-80
      for (i32 j = 1; j < B; ++j) delta[(size_t)p * B + j] += delta[(size_t)p * B + j - 1];
    i32 pos = 0;                                                 // op starts at 0 (:481)
    for (i32 j = 0; j < B; ++j) {                                // :268-287
      bool ok = true;
      for (i32 p = 0; p < s.k && ok; ++p) {
        i32 d = (i32)delta[(size_t)p * B + j];
        if (d > 0) {
          u32 w = (u32)d + s.pw[p];
          if ((float)w > s.maxw) ok = false;
        }
      }
      if (ok) pos = j;                                           // atomicMax(op, j)
    }
    for (i32 p = 0; p < s.k; ++p) s.pw[p] += (u32)(i32)delta[(size_t)p * B + pos];   // :305-308
    for (i32 j = 0; j <= pos; ++j) {                             // :309-322
      u32 v = buf[j].v;
      s.part[v] = buf[j].des;
      s.updated[v] = 1;
      for (i32 e = s.xadj[v]; e < s.xadj[v + 1]; ++e) s.updated[s.adjncy[e]] = 1;
      *gain_sum += buf[j].gain;
    }
    *moves += pos + 1;
    ++rounds;
    update_all_flagged(s);                                       // :497-498
  }
  return rounds;
}

// ---------------------------------------------------------------------------
// Balance rounds (default mode only; not in the reference, whose refinement
// never repairs an overweight part, cuda_check.hpp:105-113 only prints it).
// A round: every boundary vertex of an overweight part (float(pw) > cap)
// picks the neighbouring part q != p with room (float(pw[q] + w) <= cap) that
// maximises the signed connection gain ed_q - id (ties: smaller q); if no
// neighbouring part has room, the lightest part (ties: smaller id) if it has
// room, with gain ed - id.  Candidates yield to a smaller-id neighbouring
// candidate; the rest are sorted by (gain desc, id asc), capped, and the
// longest prefix is applied in which every move's source is still overweight
// before the move and every destination stays within cap after it.
// ---------------------------------------------------------------------------
struct BalMove { i64 g; u32 v, src, des; };

static i32 balance_level(RefineState& s, float cap, i32 move_cap, i64* moves_out) {
  i32 rounds = 0;
  std::vector<u32> ed(s.k, 0);
  std::vector<char> seen(s.k, 0);
  std::vector<i32> touched;
  std::vector<char> isc(s.n, 0);
  std::vector<u32> bt(s.n, 0);
  std::vector<i64> bg(s.n, 0);
  std::vector<i32> cand;
  std::vector<BalMove> buf;
  for (;;) {
    // lightest part
    u32 light = 0;
    for (i32 p = 1; p < s.k; ++p)
      if (s.pw[p] < s.pw[light]) light = (u32)p;
    cand.clear();
    for (i32 v = 0; v < s.n; ++v) {
      isc[v] = 0;
      const u32 p = s.part[v];
      if (!s.boundary[v] || !((float)s.pw[p] > cap)) continue;
      const u32 w = (u32)s.vwgt[v];
      touched.clear();
      u32 id = 0;
      for (i32 e = s.xadj[v]; e < s.xadj[v + 1]; ++e) {
        const u32 q = s.part[s.adjncy[e]];
        if (q == p) id += (u32)s.adjwgt[e];
        if (!seen[q]) { seen[q] = 1; ed[q] = 0; touched.push_back((i32)q); }
        ed[q] += (u32)s.adjwgt[e];
      }
      bool found = false;
      i64 bestg = 0;
      u32 bestq = 0;
      for (i32 q : touched) {
        if ((u32)q == p) continue;
        if ((float)(u32)(s.pw[q] + w) > cap) continue;
        const i64 g = (i64)(i32)(ed[q] - id);
        if (!found || g > bestg || (g == bestg && (u32)q < bestq)) { found = true; bestg = g; bestq = (u32)q; }
      }
      if (!found && light != p && !((float)(u32)(s.pw[light] + w) > cap)) {
        found = true;
        bestq = light;
        bestg = (i64)(i32)((seen[light] ? ed[light] : 0u) - id);
      }
      for (i32 q : touched) seen[q] = 0;
      if (!found) continue;
      isc[v] = 1; bt[v] = bestq; bg[v] = bestg;
      cand.push_back(v);
    }
    buf.clear();
    for (i32 v : cand) {
      bool yield = false;
      for (i32 e = s.xadj[v]; e < s.xadj[v + 1]; ++e)
        if (s.adjncy[e] < v && isc[s.adjncy[e]]) { yield = true; break; }
      if (!yield) buf.push_back({bg[v], (u32)v, s.part[v], bt[v]});
    }
    if (buf.empty()) break;
    std::sort(buf.begin(), buf.end(), [](const BalMove& a, const BalMove& b) {
      if (a.g != b.g) return a.g > b.g;
      return a.v < b.v;
    });
    const i32 B = (i32)std::min<size_t>(buf.size(), (size_t)move_cap);
    // greedy pass in sorted order: a move is taken while its source is still
    // overweight and its destination stays within the cap; others are skipped
    std::vector<u32> outw(s.k, 0), inw(s.k, 0);
    std::vector<BalMove> take;
    for (i32 t = 0; t < B; ++t) {
      const u32 w = (u32)s.vwgt[buf[t].v];
      const bool src_over = (float)(u32)(s.pw[buf[t].src] - outw[buf[t].src]) > cap;
      const bool des_ok = !((float)(u32)(s.pw[buf[t].des] + inw[buf[t].des] + w) > cap);
      if (!src_over || !des_ok) continue;
      outw[buf[t].src] += w;
      inw[buf[t].des] += w;
      take.push_back(buf[t]);
    }
    buf.swap(take);
    const i32 pos = (i32)buf.size() - 1;
    for (i32 t = 0; t <= pos; ++t) {
      const u32 v = buf[t].v, w = (u32)s.vwgt[v];
      s.pw[buf[t].src] -= w;
      s.pw[buf[t].des] += w;
      s.part[v] = buf[t].des;
      s.updated[v] = 1;
      for (i32 e = s.xadj[v]; e < s.xadj[v + 1]; ++e) s.updated[s.adjncy[e]] = 1;
    }
    *moves_out += pos + 1;
    ++rounds;
    update_all_flagged(s);
    std::fill(s.updated.begin(), s.updated.end(), 0u);
  }
  return rounds;
}

// Default-mode weight cap: (1 + eps) * W / k without the reference's "+1",
// so that every part weight <= cap means balance <= 1 + eps.
float orc_balance_cap(i64 total_vwgt, i32 k, double eps) {
  return (float)((1.0 + eps) * (double)total_vwgt / (double)k);
}

// ---------------------------------------------------------------------------
// Whole partitioner.  graph_partitioner.hpp:222-365 (graph_partitioner),
// 14-123 (coarsening loop), 125-131 (init_partition), 133-220 (uncoarsening),
// uncoarsen.hpp:325-387 (expand_partition / uncoarsen).
// ---------------------------------------------------------------------------
#define ORC_MAX_LEVELS 64

typedef struct {
  i32 group_cap;         // 6 (graph_partitioner.hpp:229)
  i32 threshold_factor;  // 20 (graph_partitioner.hpp:22)
  i32 move_cap;          // 1024 (uncoarsen.hpp:475)
  double eps;            // 0.03 (declarations.h:17)
  i32 init_method;       // 0 = METIS, 1 = caller-supplied callback
  // callback for init_method 1: fills part[n] for the coarsest graph; 0 = ok
  int (*init_fn)(void* user, i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt,
                 const i32* vwgt, i32 k, i32* part);
  void* init_user;
  i32 enforce_balance;   // 0 = the reference's behaviour; 1 = default mode (balance rounds, cap without +1)
  // default mode only (partitioner.cu partition_impl): balance rounds at every
  // level but the balance_skip_levels coarsest ones (the finest level always),
  // and coarsening stops
  // before a level whose heaviest vertex outweighs coarse_vertex_frac * W/k
  // (<= 0: no such stop)
  i32 balance_skip_levels;
  double coarse_vertex_frac;
} orc_opts;

typedef struct {
  i32 n_levels;                 // levels kept, including the input graph
  i64 level_n[ORC_MAX_LEVELS];
  i64 level_m[ORC_MAX_LEVELS];
  i32 uf_launches[ORC_MAX_LEVELS];
  i32 refine_rounds[ORC_MAX_LEVELS];
  i64 refine_moves[ORC_MAX_LEVELS];
  i32 balance_rounds[ORC_MAX_LEVELS];   // per level; index n_levels-1 = coarsest
  i64 balance_moves[ORC_MAX_LEVELS];
  i64 init_cut;
  i64 cut;
  i64 max_part_weight;
  float maxw;
  i32 status;
} orc_result;

struct Level {
  i32 n;
  std::vector<i32> xadj, adjncy, adjwgt, vwgt, cmap;   // cmap: to the next coarser level
};

int orc_partition(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, const i32* vwgt,
                  i32 k, const orc_opts* opt, i32* part_out, orc_result* res) {
  memset(res, 0, sizeof(*res));
  std::vector<Level> lv(1);
  lv[0].n = n;
  lv[0].xadj.assign(xadj, xadj + n + 1);
  lv[0].adjncy.assign(adjncy, adjncy + xadj[n]);
  lv[0].adjwgt.assign(adjwgt, adjwgt + xadj[n]);
  lv[0].vwgt.assign(vwgt, vwgt + n);
  i64 total = 0;
  for (i32 v = 0; v < n; ++v) total += (u32)vwgt[v];
  float maxw = opt->enforce_balance ? orc_balance_cap(total, k, opt->eps) : orc_max_part_weight(total, k, opt->eps);
  res->maxw = maxw;
  const i64 threshold = (i64)opt->threshold_factor * k;

  // coarsening (graph_partitioner.hpp:66-105)
  std::vector<i32> cand, root, dist;
  while ((i64)lv.back().n > threshold) {
    Level& f = lv.back();
    i32 fn = f.n;
    cand.resize(fn); root.resize(fn); dist.resize(fn);
    orc_match(fn, f.xadj.data(), f.adjncy.data(), f.adjwgt.data(), cand.data());
    i32 launches = orc_union_find(fn, cand.data(), root.data(), dist.data());
    f.cmap.resize(fn);
    i32 nc = orc_group_map(fn, root.data(), dist.data(), opt->group_cap, f.cmap.data(), nullptr);
    if (nc == fn || nc < k + 1) { f.cmap.clear(); break; }       // :93-96
    Level c;
    c.n = nc;
    c.vwgt.resize(nc);
    orc_coarse_vwgt(fn, f.vwgt.data(), f.cmap.data(), nc, c.vwgt.data());
    if (opt->enforce_balance && opt->coarse_vertex_frac > 0) {
      i64 mx = 0;
      for (i32 v = 0; v < nc; ++v) mx = std::max<i64>(mx, (u32)c.vwgt[v]);
      if ((double)mx > opt->coarse_vertex_frac * (double)total / (double)k) { f.cmap.clear(); break; }
    }
    c.xadj.resize(nc + 1);
    std::vector<i32> ta(f.adjncy.size() + 1), tw(f.adjncy.size() + 1);
    i64 mc = orc_contract(fn, f.xadj.data(), f.adjncy.data(), f.adjwgt.data(), f.cmap.data(), nc,
                          c.xadj.data(), ta.data(), tw.data());
    c.adjncy.assign(ta.begin(), ta.begin() + mc);
    c.adjwgt.assign(tw.begin(), tw.begin() + mc);
    if ((i32)lv.size() < ORC_MAX_LEVELS) res->uf_launches[lv.size() - 1] = launches;
    lv.push_back(std::move(c));
    if ((i32)lv.size() >= ORC_MAX_LEVELS) break;
  }
  res->n_levels = (i32)lv.size();
  for (size_t i = 0; i < lv.size(); ++i) {
    res->level_n[i] = lv[i].n;
    res->level_m[i] = (i64)lv[i].adjncy.size();
  }

  // initial partition of the coarsest level (metis_partition.hpp:4-99)
  Level& cs = lv.back();
  std::vector<i32> cpart(cs.n);
  int rc;
  if (opt->init_method == 0) {
    i64 obj = 0;
    rc = orc_metis_kway(cs.n, cs.xadj.data(), cs.adjncy.data(), cs.adjwgt.data(), cs.vwgt.data(), k,
                        cpart.data(), &obj);
    if (rc != 1) { res->status = -10; return -10; }
  } else {
    if (!opt->init_fn) { res->status = -11; return -11; }
    rc = opt->init_fn(opt->init_user, cs.n, cs.xadj.data(), cs.adjncy.data(), cs.adjwgt.data(),
                      cs.vwgt.data(), k, cpart.data());
    if (rc != 0) { res->status = -12; return -12; }
  }
  for (i32 v = 0; v < cs.n; ++v)
    if (cpart[v] < 0 || cpart[v] >= k) { res->status = -13; return -13; }
  res->init_cut = orc_cut(cs.n, cs.xadj.data(), cs.adjncy.data(), cs.adjwgt.data(), cpart.data());

  // state at the coarsest level: part, part weights, boundary (metis_partition.hpp:52-71)
  std::vector<u32> part(cpart.begin(), cpart.end());
  std::vector<u32> boundary(cs.n, 0);
  for (i32 v = 0; v < cs.n; ++v)
    for (i32 e = cs.xadj[v]; e < cs.xadj[v + 1]; ++e)
      if (part[cs.adjncy[e]] != part[v]) { boundary[v] = 1; break; }
  std::vector<u32> pw(k, 0);
  for (i32 v = 0; v < cs.n; ++v) pw[part[v]] += (u32)cs.vwgt[v];
  const i32 nlv = (i32)lv.size();
  auto balances = [&](i32 L) {
    return opt->enforce_balance && (L == 0 || L < nlv - std::max(0, opt->balance_skip_levels));
  };
  if (balances((i32)lv.size() - 1)) {
    RefineState s;
    s.n = cs.n; s.k = k;
    s.xadj = cs.xadj.data(); s.adjncy = cs.adjncy.data(); s.adjwgt = cs.adjwgt.data(); s.vwgt = cs.vwgt.data();
    s.maxw = maxw;
    s.part = part; s.boundary = boundary; s.pw = pw;
    s.updated.assign(cs.n, 0); s.target = part; s.gain.assign(cs.n, 0);
    i64 bm = 0;
    res->balance_rounds[lv.size() - 1] = balance_level(s, maxw, opt->move_cap, &bm);
    res->balance_moves[lv.size() - 1] = bm;
    part.swap(s.part); boundary.swap(s.boundary); pw.swap(s.pw);
  }

  // uncoarsening (graph_partitioner.hpp:174-192); no refinement at the coarsest level
  for (i32 L = (i32)lv.size() - 2; L >= 0; --L) {
    Level& f = lv[L];
    RefineState s;
    s.n = f.n; s.k = k;
    s.xadj = f.xadj.data(); s.adjncy = f.adjncy.data(); s.adjwgt = f.adjwgt.data();
    s.vwgt = f.vwgt.data();
    s.maxw = maxw;
    s.part.resize(f.n); s.boundary.resize(f.n); s.updated.resize(f.n); s.target.resize(f.n);
    s.gain.assign(f.n, 0);
    for (i32 v = 0; v < f.n; ++v) {                      // expand_partition, uncoarsen.hpp:325-356
      u32 c = (u32)f.cmap[v];
      s.part[v] = part[c];
      s.target[v] = part[c];
      s.boundary[v] = boundary[c];
      s.updated[v] = boundary[c] ? 1 : 0;
    }
    s.pw = pw;
    update_all_flagged(s);                               // uncoarsen.hpp:385-386
    if (balances(L)) {
      std::fill(s.updated.begin(), s.updated.end(), 0u);
      i64 bm = 0;
      res->balance_rounds[L] = balance_level(s, maxw, opt->move_cap, &bm);
      res->balance_moves[L] = bm;
    }
    i64 moves = 0, gsum = 0;
    i32 rounds = refine_level(s, opt->move_cap, &moves, &gsum);
    res->refine_rounds[L] = rounds;
    res->refine_moves[L] = moves;
    part.swap(s.part);
    boundary.swap(s.boundary);
    pw.swap(s.pw);
  }
  for (i32 v = 0; v < n; ++v) part_out[v] = (i32)part[v];
  // final metrics (graph_partitioner.hpp:194-202)
  res->cut = orc_cut(n, xadj, adjncy, adjwgt, part_out);
  std::vector<i64> fpw(k);
  orc_part_weights(n, vwgt, part_out, k, fpw.data());
  res->max_part_weight = *std::max_element(fpw.begin(), fpw.end());
  res->status = 0;
  return 0;
}

// Per-level refinement entry for phase tests: runs update_vertex_info on the
// flagged vertices and then the refinement loop on one level, in place.
// part/boundary/gain/target/updated/pw are in-out (pw as u32 in i64 slots).
i32 orc_refine(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, const i32* vwgt, i32 k,
               float maxw, i32 move_cap, i32* part, i32* boundary, i32* gain, i32* target,
               i32* updated, i64* pw, i64* moves, i64* gain_sum, i32 do_initial_update) {
  RefineState s;
  s.n = n; s.k = k; s.xadj = xadj; s.adjncy = adjncy; s.adjwgt = adjwgt; s.vwgt = vwgt; s.maxw = maxw;
  s.part.assign(part, part + n);
  s.boundary.assign(boundary, boundary + n);
  s.gain.assign(gain, gain + n);
  s.target.assign(target, target + n);
  s.updated.assign(updated, updated + n);
  s.pw.resize(k);
  for (i32 p = 0; p < k; ++p) s.pw[p] = (u32)pw[p];
  if (do_initial_update) update_all_flagged(s);
  *moves = 0; *gain_sum = 0;
  i32 rounds = refine_level(s, move_cap, moves, gain_sum);
  for (i32 v = 0; v < n; ++v) {
    part[v] = (i32)s.part[v]; boundary[v] = (i32)s.boundary[v]; gain[v] = s.gain[v];
    target[v] = (i32)s.target[v]; updated[v] = (i32)s.updated[v];
  }
  for (i32 p = 0; p < k; ++p) pw[p] = s.pw[p];
  return rounds;
}

// Phase A13 alone: update_vertex_info for the flagged vertices.
void orc_update_vertex_info(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, i32 k,
                            const i32* part, const i32* updated, i32* boundary, i32* gain,
                            i32* target) {
  RefineState s;
  s.n = n; s.k = k; s.xadj = xadj; s.adjncy = adjncy; s.adjwgt = adjwgt; s.vwgt = nullptr;
  s.part.assign(part, part + n);
  s.boundary.assign(boundary, boundary + n);
  s.gain.assign(gain, gain + n);
  s.target.assign(target, target + n);
  s.updated.assign(updated, updated + n);
  update_all_flagged(s);
  for (i32 v = 0; v < n; ++v) {
    boundary[v] = (i32)s.boundary[v]; gain[v] = s.gain[v]; target[v] = (i32)s.target[v];
  }
}

// ---------------------------------------------------------------------------
// The device initial partitioner's algorithm (recursive bisection by greedy
// graph growing), restated sequentially.  This is NOT a reference function:
// the reference calls host METIS here (metis_partition.hpp:46-47).  It pins
// the CUDA initial partitioner bit for bit; its rules are documented at the
// top of dac_g-kway_b200/csrc/initpart.cu.
// ---------------------------------------------------------------------------
static inline u32 orc_mix32(u64 x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return (u32)x;
}
static inline u64 orc_grow_key(bool frontier, i32 g, i32 idx) {
  return (1ull << 63) | ((u64)(frontier ? 1 : 0) << 62) | ((u64)((u32)g ^ 0x80000000u) << 30) |
         (u64)(0x3fffffffu - (u32)idx);
}
static inline u64 orc_move_key(i32 g, i32 idx) {
  return (1ull << 63) | ((u64)((u32)g ^ 0x80000000u) << 30) | (u64)(0x3fffffffu - (u32)idx);
}
static inline i32 orc_key_idx(u64 key) { return (i32)(0x3fffffffu - (u32)(key & 0x3fffffffu)); }

void orc_init_partition(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, const i32* vwgt,
                        i32 k, double eps, u64 seed, i32 trials, i32* part) {
  std::vector<i32> lo(n, 0), hi(n, k), nlo(n), nhi(n), degS(n), R(n), C(n);
  i32 depth = 0;
  while ((1 << depth) < k) ++depth;
  std::vector<std::vector<i32>> members(k);
  for (i32 d = 0; d < depth; ++d) {
    for (auto& m : members) m.clear();
    for (i32 v = 0; v < n; ++v) members[lo[v]].push_back(v);
    for (i32 p0 = 0; p0 < k; ++p0) {
      const std::vector<i32>& M = members[p0];
      const i32 s = (i32)M.size();
      if (s == 0) continue;
      const i32 p1 = hi[M[0]];
      if (p1 - p0 < 2) {
        for (i32 v : M) { nlo[v] = p0; nhi[v] = p1; }
        continue;
      }
      const i32 pm = p0 + (p1 - p0) / 2;
      i64 WS = 0;
      for (i32 v : M) {
        i32 dd = 0;
        for (i32 e = xadj[v]; e < xadj[v + 1]; ++e)
          if (lo[adjncy[e]] == p0) dd += adjwgt[e];
        degS[v] = dd;
        WS += (u32)vwgt[v];
      }
      const i64 TL = WS * (pm - p0) / (p1 - p0);
      const i64 capL = (i64)((double)TL * (1.0 + eps * 0.5));
      const i64 capR = (i64)((double)(WS - TL) * (1.0 + eps * 0.5));
      i64 best_cut = 0, best_dev = 0;
      i32 best_t = -1;
      std::vector<i32> bestR(s);
      for (i32 t = 0; t < trials; ++t) {
        for (i32 v : M) { R[v] = 0; C[v] = 0; }
        i64 wR = 0;
        i32 pick = (i32)(orc_mix32(seed * 0x9e3779b97f4a7c15ull + (u64)p0 * 1315423911ull + (u64)t) % (u32)s);
        for (i32 step = 0; step < s; ++step) {
          if (step > 0) {
            u64 best = 0;
            for (i32 i = 0; i < s; ++i) {
              const i32 v = M[i];
              if (!R[v]) best = std::max(best, orc_grow_key(C[v] > 0, 2 * C[v] - degS[v], i));
            }
            if (best == 0) break;
            pick = orc_key_idx(best);
            const i64 vw = (u32)vwgt[M[pick]];
            if (wR + vw > TL && (wR + vw - TL) > (TL - wR)) break;
          }
          const i32 v = M[pick];
          R[v] = 1;
          wR += (u32)vwgt[v];
          for (i32 e = xadj[v]; e < xadj[v + 1]; ++e)
            if (lo[adjncy[e]] == p0) C[adjncy[e]] += adjwgt[e];
          if (wR >= TL) break;
        }
        const i32 max_moves = std::min(s / 4 + 32, 256);   // initpart.cu gggp_max_moves
        for (i32 mv = 0; mv < max_moves; ++mv) {
          u64 best = 0;
          for (i32 i = 0; i < s; ++i) {
            const i32 v = M[i];
            const i32 g = R[v] ? (degS[v] - 2 * C[v]) : (2 * C[v] - degS[v]);
            if (g <= 0) continue;
            const i64 vw = (u32)vwgt[v];
            const bool ok = R[v] ? ((WS - wR) + vw <= capR) : (wR + vw <= capL);
            if (!ok) continue;
            best = std::max(best, orc_move_key(g, i));
          }
          if (best == 0) break;
          const i32 v = M[orc_key_idx(best)];
          const i32 r = R[v];
          R[v] = r ^ 1;
          wR += r ? -(i64)(u32)vwgt[v] : (i64)(u32)vwgt[v];
          const i32 sign = r ? -1 : 1;
          for (i32 e = xadj[v]; e < xadj[v + 1]; ++e)
            if (lo[adjncy[e]] == p0) C[adjncy[e]] += sign * adjwgt[e];
        }
        i64 cut = 0;
        for (i32 v : M)
          if (R[v]) cut += degS[v] - C[v];
        const i64 dev = wR > TL ? wR - TL : TL - wR;
        if (best_t < 0 || cut < best_cut || (cut == best_cut && dev < best_dev)) {
          best_t = t; best_cut = cut; best_dev = dev;
          for (i32 i = 0; i < s; ++i) bestR[i] = R[M[i]];
        }
      }
      for (i32 i = 0; i < s; ++i) {
        const i32 v = M[i];
        if (bestR[i]) { nlo[v] = p0; nhi[v] = pm; }
        else { nlo[v] = pm; nhi[v] = p1; }
      }
    }
    lo.swap(nlo);
    hi.swap(nhi);
  }
  for (i32 v = 0; v < n; ++v) part[v] = lo[v];
}


// Balance rounds alone on one level (per-phase check of gkw_balance).
i32 orc_balance(i32 n, const i32* xadj, const i32* adjncy, const i32* adjwgt, const i32* vwgt, i32 k, float cap,
                i32 move_cap, i32* part, i32* boundary, i32* gain, i32* target, i64* pw, i64* moves) {
  RefineState s;
  s.n = n; s.k = k; s.xadj = xadj; s.adjncy = adjncy; s.adjwgt = adjwgt; s.vwgt = vwgt; s.maxw = cap;
  s.part.assign(part, part + n);
  s.boundary.assign(boundary, boundary + n);
  s.gain.assign(gain, gain + n);
  s.target.assign(target, target + n);
  s.updated.assign(n, 0);
  s.pw.resize(k);
  for (i32 p = 0; p < k; ++p) s.pw[p] = (u32)pw[p];
  *moves = 0;
  i32 rounds = balance_level(s, cap, move_cap, moves);
  for (i32 v = 0; v < n; ++v) {
    part[v] = (i32)s.part[v]; boundary[v] = (i32)s.boundary[v]; gain[v] = s.gain[v]; target[v] = (i32)s.target[v];
  }
  for (i32 p = 0; p < k; ++p) pw[p] = s.pw[p];
  return rounds;
}

}  // extern "C"
