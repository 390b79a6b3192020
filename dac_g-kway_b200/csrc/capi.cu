// C ABI entry points (declared in include/gkway.h).  Every entry point
// catches the library's errors and turns them into a status code plus a
// per-thread message; no exception crosses the boundary.
#include <algorithm>
#include <cstring>
#include <exception>
#include <new>

#include "gkw_internal.cuh"

struct gkw_handle {
  gkw::Handle h;
};

using namespace gkw;

namespace gkw {
Handle& handle_of(gkw_handle* h) { return h->h; }
}  // namespace gkw

namespace {

template <class F>
gkw_status guard(F&& f) {
  try {
    f();
    return GKW_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.st;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return GKW_E_NOMEM;
  } catch (const std::exception& e) {
    set_error(e.what());
    return GKW_E_INTERNAL;
  }
}

Handle& H(gkw_handle* h) {
  if (!h) throw Error{GKW_E_INVALID, "handle is NULL"};
  GKW_CUDA(cudaSetDevice(h->h.device));
  return h->h;
}

DevGraph dev_view(const gkw_csr* g) {
  GKW_REQUIRE(g != nullptr, GKW_E_INVALID, "graph is NULL");
  GKW_REQUIRE(g->n >= 0 && g->nnz >= 0, GKW_E_INVALID, "negative size");
  GKW_REQUIRE(g->nnz < ((int64_t)1 << 31), GKW_E_UNSUPPORTED, "nnz must be < 2^31");
  GKW_REQUIRE(g->xadj != nullptr, GKW_E_INVALID, "xadj is NULL");
  GKW_REQUIRE(g->nnz == 0 || g->adjncy != nullptr, GKW_E_INVALID, "adjncy is NULL");
  DevGraph d;
  d.n = g->n;
  d.m = g->nnz;
  d.xadj = g->xadj;
  d.adjncy = g->adjncy;
  d.adjwgt = g->adjwgt;
  d.vwgt = g->vwgt;
  return d;
}

void need_weights(const DevGraph& d) {
  GKW_REQUIRE(d.m == 0 || d.adjwgt != nullptr, GKW_E_INVALID, "adjwgt is NULL");
  GKW_REQUIRE(d.n == 0 || d.vwgt != nullptr, GKW_E_INVALID, "vwgt is NULL");
}

__global__ void k_unpack_keys(i32 n, const u64* __restrict__ keys, i32* __restrict__ root,
                              i32* __restrict__ dist) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) {
    root[v] = (i32)(u32)(keys[v] >> 32);
    dist[v] = (i32)(u32)keys[v];
  }
}

__global__ void k_pack_keys(i32 n, const i32* __restrict__ root, const i32* __restrict__ dist,
                            u64* __restrict__ keys) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) keys[v] = ((u64)(u32)root[v] << 32) | (u32)dist[v];
}

void sync(Handle& h) { GKW_CUDA(cudaStreamSynchronize(h.stream)); }

}  // namespace

extern "C" {

const char* gkw_version(void) { return "gkway-b200 0.1.0"; }

const char* gkw_last_error(void) { return last_error_cstr(); }

uint64_t gkw_kernel_launches(void) { return launch_total(); }

void gkw_default_options(gkw_options* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->eps = 0.03;
  o->group_cap = 6;
  o->threshold_factor = 20;
  o->move_cap = 1024;
  o->init_method = GKW_INIT_DEVICE;
  o->init_fn = nullptr;
  o->init_user = nullptr;
  o->seed = 1;
  o->init_trials = 8;
  o->enforce_balance = 1;
  o->balance_skip_levels = 1;
  o->coarse_vertex_frac = 0.5;
}

float gkw_max_part_weight(int64_t total_vwgt, int32_t k, double eps) {
  return max_part_weight(total_vwgt, k, eps);
}

gkw_status gkw_create(gkw_handle** out, int32_t device) {
  return guard([&] {
    GKW_REQUIRE(out != nullptr, GKW_E_INVALID, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    GKW_CUDA(cudaGetDeviceCount(&ndev));
    GKW_REQUIRE(device >= 0 && device < ndev, GKW_E_INVALID, "no such CUDA device");
    GKW_CUDA(cudaSetDevice(device));
    gkw_handle* h = new gkw_handle();
    h->h.device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&h->h.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete h;
      GKW_CUDA(e);
    }
    h->h.own_stream = true;
    // GKW_GRAPHS=0: launch sequences always run as is (no CUDA-graph replay)
    if (const char* gs = getenv("GKW_GRAPHS")) h->h.graphs_on = *gs != '0';
    e = cudaMallocHost(&h->h.h_pinned, 64 * sizeof(int64_t));
    if (e != cudaSuccess) {
      cudaStreamDestroy(h->h.stream);
      delete h;
      GKW_CUDA(e);
    }
    int sms = 0;
    GKW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    h->h.sm_count = sms;
    int optin = 0;
    GKW_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    h->h.smem_optin = optin;
    // the handle's stream does not wait for the legacy default stream: every
    // initialisation goes on that stream and completes before the handle is used
    e = cudaMalloc(&h->h.coop, sizeof(CoopState));
    if (e == cudaSuccess) e = cudaMemsetAsync(h->h.coop, 0, sizeof(CoopState), h->h.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->h.stream);
    if (e != cudaSuccess) {
      cudaFreeHost(h->h.h_pinned);
      cudaStreamDestroy(h->h.stream);
      delete h;
      GKW_CUDA(e);
    }
    *out = h;
  });
}

gkw_status gkw_destroy(gkw_handle* h) {
  return guard([&] {
    if (!h) return;
    cudaSetDevice(h->h.device);
    cudaStreamSynchronize(h->h.stream);
    if (h->h.own_stream) cudaStreamDestroy(h->h.stream);
    cudaFreeHost(h->h.h_pinned);
    if (h->h.scan) cudaFree(h->h.scan);
    if (h->h.coop) cudaFree(h->h.coop);
    if (h->h.arena) cudaFree(h->h.arena);
    if (h->h.tev_ready)
      for (cudaEvent_t e : h->h.tev) cudaEventDestroy(e);
    graph_cache_clear(h->h);
    forget_coop_event(h->h);
    delete h;
    cudaGetLastError();   // teardown is best effort: leave no error pending for later calls
  });
}

gkw_status gkw_set_stream(gkw_handle* h, void* stream) {
  return guard([&] {
    Handle& hh = H(h);
    sync(hh);
    if (hh.own_stream) cudaStreamDestroy(hh.stream);
    hh.stream = (cudaStream_t)stream;
    hh.own_stream = false;
  });
}

void* gkw_get_stream(gkw_handle* h) { return h ? (void*)h->h.stream : nullptr; }

static void check_tuning(const gkw_tuning& t) {
  for (int b = 0; b < 4; ++b)
    GKW_REQUIRE(t.match_lanes[b] == 2 || t.match_lanes[b] == 4 || t.match_lanes[b] == 8 || t.match_lanes[b] == 16 ||
                    t.match_lanes[b] == 32,
                GKW_E_INVALID, "match_lanes must be 2, 4, 8, 16 or 32");
  GKW_REQUIRE(t.level_verts_per_cta >= 32 && t.level_min_ctas >= 1, GKW_E_INVALID,
              "level_verts_per_cta must be >= 32 and level_min_ctas >= 1");
  GKW_REQUIRE(t.coarsen_fused_max_n >= 0 && t.coarsen_verts_per_cta >= 64, GKW_E_INVALID,
              "coarsen_fused_max_n must be >= 0 and coarsen_verts_per_cta >= 64");
}

gkw_status gkw_get_tuning(gkw_handle* h, gkw_tuning* out) {
  return guard([&] {
    GKW_REQUIRE(out != nullptr, GKW_E_INVALID, "out is NULL");
    *out = H(h).tuning;
  });
}

gkw_status gkw_set_tuning(gkw_handle* h, const gkw_tuning* t) {
  return guard([&] {
    GKW_REQUIRE(t != nullptr, GKW_E_INVALID, "tuning is NULL");
    check_tuning(*t);
    H(h).tuning = *t;
  });
}

gkw_status gkw_autotune(gkw_handle* h, const gkw_csr* d_graph, int32_t k, const gkw_options* opt, gkw_tuning* out) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph g = dev_view(d_graph);
    need_weights(g);
    gkw_options o;
    if (opt) o = *opt; else gkw_default_options(&o);
    GKW_REQUIRE(o.init_method == GKW_INIT_DEVICE, GKW_E_INVALID, "autotune runs the device initial partition");
    autotune(hh, g, k, o);
    if (out) *out = hh.tuning;
  });
}

gkw_status gkw_partition_device(gkw_handle* h, const gkw_csr* d_graph, int32_t k, const gkw_options* opt,
                                int32_t* d_part_out, int64_t* cut_out, gkw_stats* stats) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph g = dev_view(d_graph);
    need_weights(g);
    GKW_REQUIRE(g.n == 0 || d_part_out != nullptr, GKW_E_INVALID, "part_out is NULL");
    gkw_options o;
    if (opt) o = *opt; else gkw_default_options(&o);
    hh.hier.reset();
    hh.scratch.reset();
    partition_impl(hh, g, k, o, d_part_out, cut_out, stats);
  });
}

gkw_status gkw_partition(gkw_handle* h, const gkw_csr* graph, int32_t k, const gkw_options* opt,
                         int32_t* part_out, int64_t* cut_out, gkw_stats* stats) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph hg = dev_view(graph);
    gkw_options o;
    if (opt) o = *opt; else gkw_default_options(&o);
    partition_host(hh, hg, 0, k, o, part_out, cut_out, stats);
  });
}

gkw_status gkw_partition_multi_k(gkw_handle* h, const gkw_csr* graph, int32_t n_k, const int32_t* ks,
                                 const gkw_options* opt, int32_t* parts_out, int64_t* cuts_out) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph hg = dev_view(graph);
    gkw_options o;
    if (opt) o = *opt; else gkw_default_options(&o);
    partition_multi_host(hh, hg, n_k, ks, o, parts_out, cuts_out);
  });
}

gkw_status gkw_match(gkw_handle* h, const gkw_csr* d_graph, int32_t* d_cand) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph g = dev_view(d_graph);
    GKW_REQUIRE(g.m == 0 || g.adjwgt, GKW_E_INVALID, "adjwgt is NULL");
    hh.scratch.reset();
    run_match(hh, g, d_cand);
    sync(hh);
  });
}

gkw_status gkw_union_find(gkw_handle* h, int32_t n, const int32_t* d_cand, int32_t* d_root, int32_t* d_dist,
                          int32_t* rounds_out) {
  return guard([&] {
    Handle& hh = H(h);
    GKW_REQUIRE(n >= 0, GKW_E_INVALID, "negative n");
    hh.scratch.reset();
    u64* keys = hh.scratch.alloc_n<u64>(std::max(n, 1));
    run_union_find(hh, n, d_cand, keys, &hh.coop->uf_rounds);
    if (n) launch(k_unpack_keys, ceil_div(n, 256), 256, 0, hh.stream, n, keys, d_root, d_dist);
    GKW_CHECK_LAUNCH();
    const CoopState c = read_coop(hh);
    if (rounds_out) *rounds_out = c.uf_rounds;
  });
}

gkw_status gkw_group_map(gkw_handle* h, int32_t n, const int32_t* d_root, const int32_t* d_dist,
                         int32_t group_cap, int32_t* d_cmap, int32_t* nc_out) {
  return guard([&] {
    Handle& hh = H(h);
    GKW_REQUIRE(n >= 0, GKW_E_INVALID, "negative n");
    hh.scratch.reset();
    u64* keys = hh.scratch.alloc_n<u64>(std::max(n, 1));
    if (n) launch(k_pack_keys, ceil_div(n, 256), 256, 0, hh.stream, n, d_root, d_dist, keys);
    GKW_CHECK_LAUNCH();
    run_group_map(hh, n, keys, group_cap, d_cmap, &hh.coop->nc);
    const CoopState c = read_coop(hh);
    if (nc_out) *nc_out = c.nc;
  });
}

gkw_status gkw_contract(gkw_handle* h, const gkw_csr* d_graph, const int32_t* d_cmap, int32_t nc, int32_t* d_cxadj,
                        int32_t* d_cadjncy, int32_t* d_cadjwgt, int32_t* d_cvwgt, int64_t* mc_out) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph g = dev_view(d_graph);
    need_weights(g);
    GKW_REQUIRE(nc >= 0 && nc <= std::max(g.n, 0), GKW_E_INVALID, "nc out of range");
    GKW_REQUIRE(d_cadjncy && d_cadjwgt, GKW_E_INVALID, "output arrays are NULL");
    hh.scratch.reset();
    // the member table is sized by the largest member count (any cmap is accepted here)
    i32 cap = 1;
    {
      std::vector<i32> hc(g.n);
      if (g.n) GKW_CUDA(cudaMemcpyAsync(hc.data(), d_cmap, sizeof(i32) * g.n, cudaMemcpyDeviceToHost, hh.stream));
      GKW_CUDA(cudaStreamSynchronize(hh.stream));
      std::vector<i32> cnt(std::max(nc, 1), 0);
      for (i32 v = 0; v < g.n; ++v) {
        GKW_REQUIRE(hc[v] >= 0 && hc[v] < nc, GKW_E_INVALID, "cmap entry out of range");
        cap = std::max(cap, ++cnt[hc[v]]);
      }
    }
    GKW_CUDA(cudaMemcpyAsync(&hh.coop->nc, &nc, sizeof(i32), cudaMemcpyHostToDevice, hh.stream));
    GKW_CUDA(cudaStreamSynchronize(hh.stream));
    run_contract(hh, g, d_cmap, &hh.coop->nc, nc, cap, d_cxadj, d_cadjncy, d_cadjwgt, d_cvwgt, &hh.coop->mc);
    CoopState c = read_coop(hh);
    if (c.arena_overflow) {
      ensure_arena(hh, (u64)((double)(hh.arena_words + (u64)c.arena_need) * 1.25) + 1024);
      run_contract(hh, g, d_cmap, &hh.coop->nc, nc, cap, d_cxadj, d_cadjncy, d_cadjwgt, d_cvwgt, &hh.coop->mc);
      c = read_coop(hh);
      GKW_REQUIRE(!c.arena_overflow, GKW_E_INTERNAL, "long-row arena overflow after growth");
    }
    if (mc_out) *mc_out = c.mc;
  });
}

gkw_status gkw_update_vertex_info(gkw_handle* h, const gkw_csr* d_graph, int32_t k, const int32_t* d_part,
                                  const int32_t* d_updated, int32_t* d_boundary, int32_t* d_gain,
                                  int32_t* d_target) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph g = dev_view(d_graph);
    GKW_REQUIRE(g.m == 0 || g.adjwgt, GKW_E_INVALID, "adjwgt is NULL");
    GKW_REQUIRE(g.n == 0 || d_updated, GKW_E_INVALID, "updated is NULL");
    hh.scratch.reset();
    check_parts(hh, g.n, d_part, k);
    RefineCtx* c = refine_create_ext(hh, g.n, k, 1024, const_cast<i32*>(d_part), d_boundary, d_gain, d_target);
    struct G {
      RefineCtx* c;
      ~G() { refine_destroy(c); }
    } gg{c};
    LevelJob j;
    j.lists = true;
    j.updated = d_updated;
    level_run(hh, c, g, j, 0);
    level_stats(hh, c, 1);
  });
}

gkw_status gkw_refine(gkw_handle* h, const gkw_csr* d_graph, int32_t k, float maxw, int32_t move_cap,
                      int32_t* d_part, int32_t* d_boundary, int32_t* d_gain, int32_t* d_target,
                      const int32_t* d_updated, int32_t* d_pw, int32_t initial_update, int32_t* rounds_out,
                      int64_t* moves_out) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph g = dev_view(d_graph);
    need_weights(g);
    hh.scratch.reset();
    check_parts(hh, g.n, d_part, k);
    check_parts(hh, g.n, d_target, k);
    RefineCtx* c = refine_create_ext(hh, g.n, k, move_cap, d_part, d_boundary, d_gain, d_target);
    struct G {
      RefineCtx* c;
      ~G() { refine_destroy(c); }
    } gg{c};
    GKW_CUDA(cudaMemcpyAsync(refine_pw(c), d_pw, sizeof(i32) * k, cudaMemcpyDeviceToDevice, hh.stream));
    LevelJob j;
    j.lists = true;
    j.updated = initial_update ? d_updated : nullptr;
    j.refine = true;
    j.maxw = maxw;
    j.move_cap = move_cap;
    level_run(hh, c, g, j, 0);
    GKW_CUDA(cudaMemcpyAsync(d_pw, refine_pw(c), sizeof(i32) * k, cudaMemcpyDeviceToDevice, hh.stream));
    RefineLevelStats s = level_stats(hh, c, 1)[0];
    if (rounds_out) *rounds_out = s.rounds;
    if (moves_out) *moves_out = s.moves;
  });
}

gkw_status gkw_balance(gkw_handle* h, const gkw_csr* d_graph, int32_t k, float cap, int32_t move_cap,
                       int32_t* d_part, int32_t* d_boundary, int32_t* d_gain, int32_t* d_target, int32_t* d_pw,
                       int32_t* rounds_out, int64_t* moves_out) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph g = dev_view(d_graph);
    need_weights(g);
    hh.scratch.reset();
    check_parts(hh, g.n, d_part, k);
    RefineCtx* c = refine_create_ext(hh, g.n, k, move_cap, d_part, d_boundary, d_gain, d_target);
    struct G {
      RefineCtx* c;
      ~G() { refine_destroy(c); }
    } gg{c};
    GKW_CUDA(cudaMemcpyAsync(refine_pw(c), d_pw, sizeof(i32) * k, cudaMemcpyDeviceToDevice, hh.stream));
    LevelJob j;
    j.lists = true;   // empty U, P from the caller's gains
    j.balance = true;
    j.bcap = cap;
    j.move_cap = move_cap;
    level_run(hh, c, g, j, 0);
    GKW_CUDA(cudaMemcpyAsync(d_pw, refine_pw(c), sizeof(i32) * k, cudaMemcpyDeviceToDevice, hh.stream));
    RefineLevelStats s = level_stats(hh, c, 1)[0];
    if (rounds_out) *rounds_out = s.brounds;
    if (moves_out) *moves_out = s.bmoves;
  });
}

float gkw_balance_cap(int64_t total_vwgt, int32_t k, double eps) { return balance_cap(total_vwgt, k, eps); }

gkw_status gkw_init_partition(gkw_handle* h, const gkw_csr* d_graph, int32_t k, double eps, uint64_t seed,
                              int32_t trials, int32_t* d_part) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph g = dev_view(d_graph);
    need_weights(g);
    GKW_REQUIRE(k >= 1, GKW_E_INVALID, "k must be >= 1");
    hh.scratch.reset();
    device_init_partition(hh, g, k, eps, seed, trials, d_part);
    sync(hh);
  });
}

gkw_status gkw_cut(gkw_handle* h, const gkw_csr* d_graph, const int32_t* d_part, int32_t k, int64_t* cut_out,
                   int64_t* pw_out) {
  return guard([&] {
    Handle& hh = H(h);
    DevGraph g = dev_view(d_graph);
    need_weights(g);
    GKW_REQUIRE(k >= 1, GKW_E_INVALID, "k must be >= 1");
    hh.scratch.reset();
    i64* d = hh.scratch.alloc_n<i64>(k + 2);
    compute_cut_pw(hh, g, d_part, k, d, d + 2);
    std::vector<i64> hm(k + 2);
    GKW_CUDA(cudaMemcpyAsync(hm.data(), d, sizeof(i64) * (k + 2), cudaMemcpyDeviceToHost, hh.stream));
    sync(hh);
    GKW_REQUIRE(hm[1] == 0, GKW_E_INVALID, "part id out of range [0, k)");
    if (cut_out) *cut_out = hm[0];
    if (pw_out) memcpy(pw_out, hm.data() + 2, sizeof(i64) * k);
  });
}

gkw_status gkw_read_metis_device(gkw_handle* h, const char* path, int32_t reference_quirks, gkw_csr* d_graph) {
  if (!path || !d_graph) {
    set_error("gkw_read_metis_device: NULL argument");
    return GKW_E_INVALID;
  }
  return guard([&] {
    Handle& hh = H(h);
    DeviceCsr g;
    try {
      read_metis_device(hh, path, reference_quirks != 0, g);
    } catch (...) {
      cudaFree(g.xadj);
      cudaFree(g.adjncy);
      cudaFree(g.adjwgt);
      cudaFree(g.vwgt);
      throw;
    }
    d_graph->n = g.n;
    d_graph->nnz = g.nnz;
    d_graph->xadj = g.xadj;
    d_graph->adjncy = g.adjncy;
    d_graph->adjwgt = g.adjwgt;
    d_graph->vwgt = g.vwgt;
  });
}

void gkw_free_device_graph(gkw_csr* d_graph) {
  if (!d_graph) return;
  cudaFree(const_cast<int32_t*>(d_graph->xadj));
  cudaFree(const_cast<int32_t*>(d_graph->adjncy));
  cudaFree(const_cast<int32_t*>(d_graph->adjwgt));
  cudaFree(const_cast<int32_t*>(d_graph->vwgt));
  d_graph->xadj = d_graph->adjncy = d_graph->adjwgt = d_graph->vwgt = nullptr;
}

gkw_status gkw_write_partition_device(gkw_handle* h, const char* path, int32_t n, const int32_t* d_part) {
  if (!path) {
    set_error("gkw_write_partition_device: NULL path");
    return GKW_E_INVALID;
  }
  return guard([&] { write_partition_device(H(h), path, n, d_part); });
}

}  // extern "C"
