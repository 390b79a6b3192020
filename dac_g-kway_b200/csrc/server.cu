// Batched and served partitioning on one GPU.
//
// A server owns a fixed set of partition slots.  Each slot is a library handle
// (its own CUDA stream, its own device pools) driven by one host thread, and
// all slots take jobs from one queue.  A job is one graph: it runs the same
// pipeline as gkw_partition on its slot, so its result does not depend on what
// else is running.  Jobs overlap on the device: while one slot waits on a
// small graph's latency-bound level kernels, the others fill the SMs.
//
// Kernels whose CTAs wait on one another (grid barriers) must never hold part
// of the SMs while waiting for CTAs that other such kernels keep from
// starting.  Jobs of up to narrow_max_n vertices that start beside other jobs
// therefore run in narrow mode: each of those kernels is one thread-block
// cluster, which the hardware starts as a whole.  Larger jobs, and a job that
// starts while no other runs, use wide grids, and wide launches take turns
// (launch_coop chains them per device).
//
// Admission is by predicted device footprint.  Every slot is charged the
// memory it holds (idle) or the larger of that and its job's prediction
// (running); a job starts on a free slot only if the charges stay within the
// server's budget.  The oldest queued job goes first.  When it does not fit,
// a later job that fits may overtake it, at most `max_bypass` times in a row,
// so small requests are co-scheduled beside a large one without starving it.
// A job that does not fit an empty device runs anyway and fails with
// GKW_E_NOMEM if the memory really is not there.
//
// Dynamic batching: a slot that takes a small job (up to batch_graph_max_n
// vertices, device initial partition) also drains the queued small jobs with
// the same options, up to batch_max_n vertices together, and partitions them
// as one disjoint union (batch.cu).  Each graph's result is still exactly its
// lone result; under load the queue is emptied a batch at a time instead of a
// graph at a time.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gkw_internal.cuh"

using namespace gkw;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Job {
  DevGraph host;            // host arrays (the caller's, or own_* below)
  i64 vbase = 0;            // neighbour-id offset of a batch slice
  i32 k = 2;
  gkw_options opt{};
  i32* part_out = nullptr;  // host, n entries
  std::vector<i32> own_x, own_a, own_w, own_v, own_part;   // served: copies
  i64 predicted = 0;
  // results
  i64 cut = 0;
  gkw_status st = GKW_OK;
  std::string err;
  i32 slot = -1;
  i32 n_levels = 0;
  i32 batch_graphs = 1;     // graphs of the union run this job was part of
  bool alone = false;       // no other job was running when this one started
  bool done = false;
  Clock::time_point t_submit, t_start, t_end;
};
using JobPtr = std::shared_ptr<Job>;

struct Slot {
  gkw_handle* h = nullptr;
  bool busy = false;
  i64 held = 0;     // device memory the slot's pools hold
  i64 charge = 0;   // what admission counts for the slot
  // host staging of a union batch (kept between batches)
  std::vector<i32> ux, ua, uw, uv, upart, ugp, uk, ulev;
  std::vector<i64> ucut;
};

// Options under which two jobs partition identically side by side in a union.
bool same_options(const gkw_options& a, const gkw_options& b) {
  return a.eps == b.eps && a.group_cap == b.group_cap && a.threshold_factor == b.threshold_factor &&
         a.move_cap == b.move_cap && a.init_method == b.init_method && a.seed == b.seed &&
         a.init_trials == b.init_trials && a.enforce_balance == b.enforce_balance &&
         a.balance_skip_levels == b.balance_skip_levels && a.coarse_vertex_frac == b.coarse_vertex_frac;
}

constexpr size_t kMaxUnionJobs = 4096;

}  // namespace

struct gkw_server {
  i32 device = 0;
  gkw_server_config cfg{};
  std::vector<Slot> slots;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work;
  std::condition_variable cv_done;
  std::deque<JobPtr> queue;
  std::map<i64, JobPtr> tickets;
  i64 next_ticket = 1;
  bool stop = false;
  i32 head_bypass = 0;
  i32 running = 0;
  // statistics
  i64 submitted = 0, completed = 0, failed = 0;
  std::vector<double> latencies, queue_waits;
  bool have_first = false;
  Clock::time_point first_submit, last_done;
  i64 peak_reserved = 0;
  i32 peak_running = 0;
  // gkw_partition_batch's union path runs on its own handle (one batch at a time)
  std::mutex batch_mu;
  gkw_handle* batch_h = nullptr;

  i64 total_charge() const {
    i64 t = 0;
    for (const Slot& s : slots) t += s.charge;
    return t;
  }
  // Next job for free slot `si` (caller holds mu), or null.
  JobPtr pick(size_t si);
  // Queued jobs that join `first` in one union run (caller holds mu).
  std::vector<JobPtr> drain_batch(size_t si, const Job& first);
  void worker(size_t si);
  void run(Slot& s, Job& j);
  void run_union(Slot& s, std::vector<JobPtr>& jobs);
  bool batchable(const Job& j) const {
    return cfg.batch_union && cfg.batch_max_n > 0 && j.opt.init_method == GKW_INIT_DEVICE &&
           j.host.n <= cfg.batch_graph_max_n;
  }
};

std::vector<JobPtr> gkw_server::drain_batch(size_t si, const Job& first) {
  std::vector<JobPtr> out;
  if (!batchable(first) || queue.empty()) return out;
  const Slot& me = slots[si];
  const i64 others = total_charge() - me.charge;
  i64 tn = first.host.n, tm = first.host.m, tk = first.k;
  for (auto it = queue.begin(); it != queue.end() && out.size() + 1 < kMaxUnionJobs;) {
    const Job& c = **it;
    const i64 n2 = tn + c.host.n, m2 = tm + c.host.m, k2 = tk + c.k;
    const bool ok = batchable(c) && same_options(c.opt, first.opt) && n2 <= cfg.batch_max_n &&
                    m2 < ((i64)1 << 31) && k2 < ((i64)1 << 20) &&
                    (running == 0 || others + std::max(me.held, gkw_predict_footprint((i32)n2, m2, (i32)k2)) <=
                                         cfg.pool_bytes);
    if (ok) {
      tn = n2;
      tm = m2;
      tk = k2;
      out.push_back(*it);
      it = queue.erase(it);
    } else {
      ++it;
    }
  }
  return out;
}

JobPtr gkw_server::pick(size_t si) {
  if (queue.empty()) return nullptr;
  const Slot& me = slots[si];
  const i64 others = total_charge() - me.charge;
  auto fits = [&](const Job& j) {
    return running == 0 || others + std::max(me.held, j.predicted) <= cfg.pool_bytes;
  };
  if (fits(*queue.front())) {
    JobPtr j = queue.front();
    queue.pop_front();
    head_bypass = 0;
    return j;
  }
  if (head_bypass >= cfg.max_bypass) return nullptr;
  for (auto it = queue.begin() + 1; it != queue.end(); ++it) {
    if (fits(**it)) {
      JobPtr j = *it;
      queue.erase(it);
      ++head_bypass;
      return j;
    }
  }
  return nullptr;
}

void gkw_server::run(Slot& s, Job& j) {
  try {
    Handle& hh = handle_of(s.h);
    GKW_CUDA(cudaSetDevice(hh.device));
    // narrow only beside other jobs: a job that starts alone takes the whole
    // device (jobs that start later beside it run narrow, and a wide grid
    // only waits for their clusters to finish, never the reverse)
    hh.narrow = j.host.n <= cfg.narrow_max_n && !j.alone;
    gkw_stats st;
    partition_host(hh, j.host, j.vbase, j.k, j.opt, j.part_out, &j.cut, &st);
    j.n_levels = st.n_levels;
  } catch (const Error& e) {
    j.st = e.st;
    j.err = e.msg + " (job: n=" + std::to_string(j.host.n) + ", nnz=" + std::to_string(j.host.m) +
            ", k=" + std::to_string(j.k) + ")";
  } catch (const std::bad_alloc&) {
    j.st = GKW_E_NOMEM;
    j.err = "host allocation failed";
  } catch (const std::exception& e) {
    j.st = GKW_E_INTERNAL;
    j.err = e.what();
  }
  Handle& hh = handle_of(s.h);
  if (j.st != GKW_OK) {
    cudaStreamSynchronize(hh.stream);
    cudaGetLastError();
  }
  // keep at most slot_keep_bytes between jobs
  hh.hier.reset();
  hh.scratch.reset();
  const i64 held = (i64)(hh.hier.capacity() + hh.scratch.capacity());
  if (held > cfg.slot_keep_bytes) {
    try {
      hh.hier.trim();
      hh.scratch.trim();
    } catch (const Error&) {
    }
  }
}

// Partition jobs[0..] as one disjoint union on slot s.  When the union cannot
// take them (a malformed graph: an edge out of its own range), every job runs
// alone and reports its own error.
void gkw_server::run_union(Slot& s, std::vector<JobPtr>& jobs) {
  Handle& hh = handle_of(s.h);
  const i32 G = (i32)jobs.size();
  bool fallback = false;
  try {
    GKW_CUDA(cudaSetDevice(hh.device));
    i64 tn = 0, tm = 0;
    bool any_w = false, any_v = false;
    for (const JobPtr& j : jobs) {
      tn += j->host.n;
      tm += j->host.m;
      any_w |= j->host.adjwgt != nullptr;
      any_v |= j->host.vwgt != nullptr;
    }
    s.ux.resize(tn + 1);
    s.ua.resize(std::max<i64>(tm, 1));
    if (any_w) s.uw.resize(std::max<i64>(tm, 1));
    if (any_v) s.uv.resize(std::max<i64>(tn, 1));
    s.upart.resize(std::max<i64>(tn, 1));
    s.ugp.resize(G + 1);
    s.uk.resize(G);
    s.ucut.resize(G);
    s.ulev.resize(G);
    i64 vo = 0, eo = 0;
    for (i32 i = 0; i < G; ++i) {
      const DevGraph& g = jobs[i]->host;
      const i32 x0 = g.xadj[0];
      const i64 vb = jobs[i]->vbase;
      s.ugp[i] = (i32)vo;
      s.uk[i] = jobs[i]->k;
      for (i32 v = 0; v < g.n; ++v) s.ux[vo + v] = (i32)(g.xadj[v] - x0 + eo);
      for (i64 e = 0; e < g.m; ++e) s.ua[eo + e] = (i32)(g.adjncy[e] - vb + vo);
      if (any_w) {
        if (g.adjwgt) std::memcpy(s.uw.data() + eo, g.adjwgt, sizeof(i32) * g.m);
        else std::fill(s.uw.begin() + eo, s.uw.begin() + eo + g.m, 1);
      }
      if (any_v) {
        if (g.vwgt) std::memcpy(s.uv.data() + vo, g.vwgt, sizeof(i32) * g.n);
        else std::fill(s.uv.begin() + vo, s.uv.begin() + vo + g.n, 1);
      }
      vo += g.n;
      eo += g.m;
    }
    s.ux[tn] = (i32)tm;
    s.ugp[G] = (i32)tn;
    DevGraph hg;
    hg.n = (i32)tn;
    hg.m = tm;
    hg.xadj = s.ux.data();
    hg.adjncy = s.ua.data();
    hg.adjwgt = any_w ? s.uw.data() : nullptr;
    hg.vwgt = any_v ? s.uv.data() : nullptr;
    hh.narrow = false;   // one wide grid for the whole union (wide launches take turns)
    if (partition_batch_union(hh, hg, G, s.ugp.data(), s.uk.data(), jobs[0]->opt, s.upart.data(),
                              s.ucut.data(), s.ulev.data())) {
      for (i32 i = 0; i < G; ++i) {
        Job& j = *jobs[i];
        if (j.host.n) std::memcpy(j.part_out, s.upart.data() + s.ugp[i], sizeof(i32) * j.host.n);
        j.cut = s.ucut[i];
        j.n_levels = s.ulev[i];
      }
    } else {
      fallback = true;
    }
  } catch (const Error& e) {
    if (e.st == GKW_E_INVALID || e.st == GKW_E_UNSUPPORTED) {   // a bad graph, or too many parts together
      fallback = true;
    } else {
      for (JobPtr& j : jobs) {
        j->st = e.st;
        j->err = e.msg + " (union batch of " + std::to_string(G) + " graphs)";
      }
    }
  } catch (const std::bad_alloc&) {
    for (JobPtr& j : jobs) {
      j->st = GKW_E_NOMEM;
      j->err = "host allocation failed";
    }
  }
  if (fallback || jobs[0]->st != GKW_OK) {
    cudaStreamSynchronize(hh.stream);
    cudaGetLastError();
  }
  if (fallback) {
    for (JobPtr& j : jobs) run(s, *j);
    return;
  }
  hh.hier.reset();
  hh.scratch.reset();
  const i64 held = (i64)(hh.hier.capacity() + hh.scratch.capacity());
  if (held > cfg.slot_keep_bytes) {
    try {
      hh.hier.trim();
      hh.scratch.trim();
    } catch (const Error&) {
    }
  }
}

void gkw_server::worker(size_t si) {
  cudaSetDevice(device);
  std::vector<JobPtr> jobs;
  for (;;) {
    jobs.clear();
    {
      std::unique_lock<std::mutex> lk(mu);
      JobPtr j;
      for (;;) {
        if (stop) return;
        j = pick(si);
        if (j) break;
        cv_work.wait(lk);
      }
      jobs.push_back(j);
      for (JobPtr& c : drain_batch(si, *j)) jobs.push_back(c);
      Slot& s = slots[si];
      s.busy = true;
      i64 pred = j->predicted;
      if (jobs.size() > 1) {
        i64 tn = 0, tm = 0, tk = 0;
        for (const JobPtr& c : jobs) {
          tn += c->host.n;
          tm += c->host.m;
          tk += c->k;
        }
        pred = gkw_predict_footprint((i32)tn, tm, (i32)std::min<i64>(tk, INT32_MAX));
      }
      s.charge = std::max(s.held, pred);
      ++running;
      peak_running = std::max(peak_running, running);
      peak_reserved = std::max(peak_reserved, total_charge());
      const auto now = Clock::now();
      for (JobPtr& c : jobs) {
        c->slot = (i32)si;
        c->t_start = now;
        c->batch_graphs = (i32)jobs.size();
        c->alone = running == 1;
      }
    }
    if (jobs.size() == 1) run(slots[si], *jobs[0]);
    else run_union(slots[si], jobs);
    {
      std::lock_guard<std::mutex> lk(mu);
      Slot& s = slots[si];
      Handle& hh = handle_of(s.h);
      s.held = (i64)(hh.hier.capacity() + hh.scratch.capacity());
      s.charge = s.held;
      s.busy = false;
      --running;
      const auto now = Clock::now();
      for (JobPtr& j : jobs) {
        j->t_end = now;
        j->done = true;
        if (j->st == GKW_OK) {
          ++completed;
          latencies.push_back(ms_between(j->t_submit, j->t_end));
          queue_waits.push_back(ms_between(j->t_submit, j->t_start));
        } else {
          ++failed;
        }
      }
      last_done = now;
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

namespace {

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  // nearest rank
  size_t r = (size_t)std::ceil(q * (double)v.size());
  r = std::min(std::max<size_t>(r, 1), v.size());
  return v[r - 1];
}

template <class F>
gkw_status guard_s(F&& f) {
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

void enqueue(gkw_server* s, const JobPtr& j) {
  std::lock_guard<std::mutex> lk(s->mu);
  GKW_REQUIRE(!s->stop, GKW_E_INVALID, "server is shutting down");
  j->t_submit = Clock::now();
  if (!s->have_first) {
    s->have_first = true;
    s->first_submit = j->t_submit;
  }
  ++s->submitted;
  s->queue.push_back(j);
}

}  // namespace

extern "C" {

void gkw_server_default_config(gkw_server_config* c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->slots = 2;
  c->pool_bytes = (int64_t)64 << 30;
  c->slot_keep_bytes = (int64_t)4 << 30;
  c->max_bypass = 0;   // 0: 4 x slots
  c->narrow_max_n = 262144;
  c->batch_union = 1;
  c->batch_max_n = 1 << 22;
  c->batch_graph_max_n = 262144;
}

int64_t gkw_predict_footprint(int32_t n, int64_t nnz, int32_t k) {
  // bytes per vertex / per CSR entry / per part of one partition, counted
  // from the allocations of the pipeline: the input and output arrays, the
  // coarser levels (each level keeps at most ~0.6 of the vertices and entries
  // of the level below, so they sum to 1.5x the input), the cmaps, the
  // refinement state, and the coarsening scratch of the largest level
  const double nn = std::max<int32_t>(n, 1), mm = (double)std::max<int64_t>(nnz, 1);
  const double input = 4.0 * (nn + 1) + 8.0 * mm + 8.0 * nn;
  const double coarse = 1.5 * (12.0 * nn + 8.0 * mm) + 2.5 * 4.0 * nn;
  const double refine = 96.0 * nn + 32.0 * (double)std::max(k, 1);
  const double scratch = 64.0 * nn + 24.0 * mm;
  const double fixed = 16.0 * (1 << 20);
  return (int64_t)(input + coarse + refine + scratch + fixed);
}

gkw_status gkw_server_create(gkw_server** out, int32_t device, const gkw_server_config* cfg) {
  return guard_s([&] {
    GKW_REQUIRE(out != nullptr, GKW_E_INVALID, "out is NULL");
    *out = nullptr;
    gkw_server_config c;
    if (cfg) c = *cfg; else gkw_server_default_config(&c);
    GKW_REQUIRE(c.slots >= 1 && c.slots <= 256, GKW_E_INVALID, "slots must be in [1, 256]");
    GKW_REQUIRE(c.pool_bytes > 0 && c.slot_keep_bytes >= 0, GKW_E_INVALID, "bad memory budget");
    GKW_REQUIRE(c.narrow_max_n >= 0, GKW_E_INVALID, "narrow_max_n must be >= 0");
    GKW_REQUIRE(c.batch_max_n >= 0, GKW_E_INVALID, "batch_max_n must be >= 0");
    if (c.max_bypass <= 0) c.max_bypass = 4 * c.slots;
    int ndev = 0;
    GKW_CUDA(cudaGetDeviceCount(&ndev));
    GKW_REQUIRE(device >= 0 && device < ndev, GKW_E_INVALID, "no such CUDA device");
    GKW_CUDA(cudaSetDevice(device));
    size_t fr = 0, tot = 0;
    GKW_CUDA(cudaMemGetInfo(&fr, &tot));
    c.pool_bytes = std::min<int64_t>(c.pool_bytes, (int64_t)((double)fr * 0.9));
    std::unique_ptr<gkw_server> s(new gkw_server());
    s->device = device;
    s->cfg = c;
    s->slots.resize((size_t)c.slots);
    for (Slot& sl : s->slots) {
      gkw_status st = gkw_create(&sl.h, device);
      if (st != GKW_OK) {
        for (Slot& t : s->slots)
          if (t.h) gkw_destroy(t.h);
        throw Error{st, std::string("slot handle: ") + gkw_last_error()};
      }
      Handle& hh = handle_of(sl.h);
      hh.hier.set_min_chunk((size_t)16 << 20);
      hh.scratch.set_min_chunk((size_t)16 << 20);
    }
    gkw_server* raw = s.release();
    for (size_t i = 0; i < raw->slots.size(); ++i) raw->threads.emplace_back([raw, i] { raw->worker(i); });
    *out = raw;
  });
}

gkw_status gkw_server_destroy(gkw_server* s) {
  return guard_s([&] {
    if (!s) return;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = true;
      for (JobPtr& j : s->queue) {
        j->st = GKW_E_INVALID;
        j->err = "server destroyed before the job ran";
        j->done = true;
      }
      s->queue.clear();
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    for (std::thread& t : s->threads) t.join();
    for (Slot& sl : s->slots) gkw_destroy(sl.h);
    if (s->batch_h) gkw_destroy(s->batch_h);
    delete s;
  });
}

gkw_status gkw_server_submit(gkw_server* s, const gkw_csr* g, int32_t k, const gkw_options* opt,
                             int64_t* ticket_out) {
  return guard_s([&] {
    GKW_REQUIRE(s != nullptr && g != nullptr && ticket_out != nullptr, GKW_E_INVALID, "NULL argument");
    GKW_REQUIRE(g->n >= 0 && g->nnz >= 0 && g->nnz < ((int64_t)1 << 31), GKW_E_INVALID, "bad graph size");
    GKW_REQUIRE(g->xadj != nullptr && (g->nnz == 0 || g->adjncy != nullptr), GKW_E_INVALID, "NULL array");
    GKW_REQUIRE(k >= 1, GKW_E_INVALID, "k must be >= 1");
    GKW_REQUIRE(g->xadj[0] == 0 && g->xadj[g->n] == g->nnz, GKW_E_INVALID, "xadj does not span nnz");
    JobPtr j = std::make_shared<Job>();
    const size_t n = (size_t)g->n, m = (size_t)g->nnz;
    j->own_x.assign(g->xadj, g->xadj + n + 1);
    if (m) j->own_a.assign(g->adjncy, g->adjncy + m);
    if (g->adjwgt && m) j->own_w.assign(g->adjwgt, g->adjwgt + m);
    if (g->vwgt && n) j->own_v.assign(g->vwgt, g->vwgt + n);
    j->own_part.resize(std::max<size_t>(n, 1));
    j->host.n = g->n;
    j->host.m = g->nnz;
    j->host.xadj = j->own_x.data();
    j->host.adjncy = m ? j->own_a.data() : nullptr;
    j->host.adjwgt = (g->adjwgt && m) ? j->own_w.data() : nullptr;
    j->host.vwgt = (g->vwgt && n) ? j->own_v.data() : nullptr;
    j->k = k;
    if (opt) j->opt = *opt; else gkw_default_options(&j->opt);
    j->part_out = j->own_part.data();
    j->predicted = gkw_predict_footprint(g->n, g->nnz, k);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      GKW_REQUIRE(!s->stop, GKW_E_INVALID, "server is shutting down");
      *ticket_out = s->next_ticket++;
      s->tickets[*ticket_out] = j;
    }
    enqueue(s, j);
    s->cv_work.notify_all();
  });
}

gkw_status gkw_server_poll(gkw_server* s, int64_t ticket, int32_t wait_ms, int32_t* part_out,
                           int64_t* cut_out, gkw_request_info* info) {
  JobPtr j;
  {
    if (!s) {
      set_error("server is NULL");
      return GKW_E_INVALID;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) {
      set_error("unknown ticket " + std::to_string(ticket));
      return GKW_E_INVALID;
    }
    j = it->second;
    auto ready = [&] { return j->done; };
    if (wait_ms < 0) s->cv_done.wait(lk, ready);
    else if (wait_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
    if (!j->done) return GKW_E_PENDING;
    s->tickets.erase(ticket);
  }
  if (info) {
    info->queue_ms = j->slot >= 0 ? ms_between(j->t_submit, j->t_start) : 0.0;
    info->run_ms = j->slot >= 0 ? ms_between(j->t_start, j->t_end) : 0.0;
    info->latency_ms = j->slot >= 0 ? ms_between(j->t_submit, j->t_end) : 0.0;
    info->predicted_bytes = j->predicted;
    info->slot = j->slot;
    info->n_levels = j->n_levels;
    info->batch_graphs = j->batch_graphs;
    info->reserved = 0;
  }
  if (j->st != GKW_OK) {
    set_error(j->err);
    return j->st;
  }
  if (part_out && j->host.n) memcpy(part_out, j->own_part.data(), sizeof(i32) * (size_t)j->host.n);
  if (cut_out) *cut_out = j->cut;
  return GKW_OK;
}

gkw_status gkw_server_stats_get(gkw_server* s, gkw_server_stats* out, int32_t reset) {
  return guard_s([&] {
    GKW_REQUIRE(s != nullptr && out != nullptr, GKW_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->p50_ms = percentile(s->latencies, 0.50);
    out->p99_ms = percentile(s->latencies, 0.99);
    out->max_ms = s->latencies.empty() ? 0.0 : *std::max_element(s->latencies.begin(), s->latencies.end());
    double qs = 0;
    for (double q : s->queue_waits) qs += q;
    out->mean_queue_ms = s->queue_waits.empty() ? 0.0 : qs / (double)s->queue_waits.size();
    const double span = s->have_first ? ms_between(s->first_submit, s->last_done) : 0.0;
    out->graphs_per_s = span > 0 ? (double)s->completed / (span / 1e3) : 0.0;
    out->peak_reserved_bytes = s->peak_reserved;
    out->peak_running = s->peak_running;
    out->slots = (i32)s->slots.size();
    if (reset) {
      s->submitted = s->completed = s->failed = 0;
      s->latencies.clear();
      s->queue_waits.clear();
      s->have_first = false;
      s->peak_reserved = s->total_charge();
      s->peak_running = s->running;
    }
  });
}

gkw_status gkw_partition_batch(gkw_server* s, const gkw_csr_batch* b, const gkw_options* opt, int32_t* part_out,
                               int64_t* cut_out, int32_t* status_out) {
  std::vector<JobPtr> jobs;
  bool union_done = false;
  gkw_status st = guard_s([&] {
    GKW_REQUIRE(s != nullptr && b != nullptr, GKW_E_INVALID, "NULL argument");
    const gkw_csr& g = b->graph;
    GKW_REQUIRE(b->n_graphs >= 0, GKW_E_INVALID, "n_graphs must be >= 0");
    GKW_REQUIRE(g.n >= 0 && g.nnz >= 0 && g.nnz < ((int64_t)1 << 31), GKW_E_INVALID, "bad graph size");
    GKW_REQUIRE(b->graph_ptr != nullptr && (b->k != nullptr || b->n_graphs == 0), GKW_E_INVALID,
                "graph_ptr or k is NULL");
    GKW_REQUIRE(g.xadj != nullptr && (g.nnz == 0 || g.adjncy != nullptr), GKW_E_INVALID, "NULL array");
    GKW_REQUIRE(g.n == 0 || part_out != nullptr, GKW_E_INVALID, "part_out is NULL");
    GKW_REQUIRE(b->graph_ptr[0] == 0 && b->graph_ptr[b->n_graphs] == g.n, GKW_E_INVALID,
                "graph_ptr must run from 0 to n");
    GKW_REQUIRE(g.xadj[0] == 0 && g.xadj[g.n] == g.nnz, GKW_E_INVALID, "xadj does not span nnz");
    gkw_options base;
    if (opt) base = *opt; else gkw_default_options(&base);
    for (i32 i = 0; i < b->n_graphs; ++i) {
      GKW_REQUIRE(b->graph_ptr[i] <= b->graph_ptr[i + 1], GKW_E_INVALID, "graph_ptr must not decrease");
      GKW_REQUIRE(b->k[i] >= 1, GKW_E_INVALID, "k must be >= 1 (graph " + std::to_string(i) + ")");
    }
    // the whole batch as one disjoint union (batch.cu) when every graph uses
    // the same options: one pipeline for all graphs instead of one per graph
    bool same_eps = true;
    for (i32 i = 0; b->eps && i < b->n_graphs; ++i) same_eps &= b->eps[i] == b->eps[0];
    if (s->cfg.batch_union && base.init_method == GKW_INIT_DEVICE && same_eps) {
      gkw_options uo = base;
      if (b->eps && b->n_graphs) uo.eps = b->eps[0];
      std::lock_guard<std::mutex> lk(s->batch_mu);
      if (!s->batch_h) {
        const gkw_status cs = gkw_create(&s->batch_h, s->device);
        if (cs != GKW_OK) throw Error{cs, gkw_last_error()};
      }
      DevGraph hg;
      hg.n = g.n;
      hg.m = g.nnz;
      hg.xadj = g.xadj;
      hg.adjncy = g.adjncy;
      hg.adjwgt = g.adjwgt;
      hg.vwgt = g.vwgt;
      Handle& bh = handle_of(s->batch_h);
      bh.narrow = false;
      std::vector<i64> cuts(std::max(b->n_graphs, 1));
      const auto t0 = Clock::now();
      bool ok = false;
      try {
        ok = partition_batch_union(bh, hg, b->n_graphs, b->graph_ptr, b->k, uo, part_out, cuts.data());
      } catch (const Error& e) {
        // a bad graph, or more parts than one union holds: the per-graph path
        // reports each graph's own status
        if (e.st != GKW_E_INVALID && e.st != GKW_E_UNSUPPORTED) throw;
      }
      if (ok) {
        const auto t1 = Clock::now();
        for (i32 i = 0; i < b->n_graphs; ++i) {
          if (cut_out) cut_out[i] = cuts[i];
          if (status_out) status_out[i] = GKW_OK;
        }
        std::lock_guard<std::mutex> lk2(s->mu);
        if (!s->have_first && b->n_graphs) {
          s->have_first = true;
          s->first_submit = t0;
        }
        s->submitted += b->n_graphs;
        s->completed += b->n_graphs;
        for (i32 i = 0; i < b->n_graphs; ++i) {   // every graph of the batch completes with it
          s->latencies.push_back(ms_between(t0, t1));
          s->queue_waits.push_back(0.0);
        }
        s->last_done = t1;
        union_done = true;
        return;
      }
      // an edge joins two graphs, or a graph is malformed: the per-graph path
      // reports which graph
    }
    for (i32 i = 0; i < b->n_graphs; ++i) {
      const i32 v0 = b->graph_ptr[i], v1 = b->graph_ptr[i + 1];
      GKW_REQUIRE(v0 <= v1, GKW_E_INVALID, "graph_ptr must not decrease");
      GKW_REQUIRE(b->k[i] >= 1, GKW_E_INVALID, "k must be >= 1 (graph " + std::to_string(i) + ")");
      const i64 e0 = g.xadj[v0], e1 = g.xadj[v1];
      GKW_REQUIRE(e0 <= e1, GKW_E_INVALID, "xadj must not decrease");
      JobPtr j = std::make_shared<Job>();
      j->host.n = v1 - v0;
      j->host.m = e1 - e0;
      j->host.xadj = g.xadj + v0;
      j->host.adjncy = g.adjncy ? g.adjncy + e0 : nullptr;
      j->host.adjwgt = g.adjwgt ? g.adjwgt + e0 : nullptr;
      j->host.vwgt = g.vwgt ? g.vwgt + v0 : nullptr;
      j->vbase = v0;
      j->k = b->k[i];
      j->opt = base;
      if (b->eps) j->opt.eps = b->eps[i];
      j->part_out = part_out + v0;
      j->predicted = gkw_predict_footprint(j->host.n, j->host.m, j->k);
      jobs.push_back(j);
    }
    // largest first (longest-processing-time order), ties by graph index
    std::vector<size_t> order(jobs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t x, size_t y) { return jobs[x]->host.m + jobs[x]->host.n >
                                                      jobs[y]->host.m + jobs[y]->host.n; });
    {
      std::lock_guard<std::mutex> lk(s->mu);
      GKW_REQUIRE(!s->stop, GKW_E_INVALID, "server is shutting down");
      const auto now = Clock::now();
      if (!s->have_first && !jobs.empty()) {
        s->have_first = true;
        s->first_submit = now;
      }
      for (size_t i : order) {
        jobs[i]->t_submit = now;
        s->queue.push_back(jobs[i]);
      }
      s->submitted += (i64)jobs.size();
    }
    s->cv_work.notify_all();
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] {
      for (const JobPtr& j : jobs)
        if (!j->done) return false;
      return true;
    });
  });
  if (st != GKW_OK || union_done) return st;
  gkw_status first = GKW_OK;
  for (size_t i = 0; i < jobs.size(); ++i) {
    if (cut_out) cut_out[i] = jobs[i]->cut;
    if (status_out) status_out[i] = jobs[i]->st;
    if (jobs[i]->st != GKW_OK && first == GKW_OK) {
      first = jobs[i]->st;
      set_error("graph " + std::to_string(i) + ": " + jobs[i]->err);
    }
  }
  return first;
}

}  // extern "C"
