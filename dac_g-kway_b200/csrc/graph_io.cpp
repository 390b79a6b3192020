// Host side of the C++ API: the METIS .graph parser, the output writer, the
// GraphPartitioner class and the reference-compatible graph_partitioner().
#include <dlfcn.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <charconv>
#include <fstream>
#include <iostream>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "gkway.hpp"
#include "metis_header.h"

extern "C" void gkw_io_set_error(const std::string& msg);

namespace gk {

namespace {

std::string read_file(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open graph file: " + path);
  std::string buf;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (sz > 0) {
    buf.resize((size_t)sz);
    size_t got = fread(&buf[0], 1, (size_t)sz, f);
    buf.resize(got);
  }
  fclose(f);
  return buf;
}

struct Cursor {
  const char* p;
  const char* end;
  // next line (without the newline); returns false at end of input
  bool line(const char*& b, const char*& e) {
    if (p >= end) return false;
    b = p;
    const char* q = (const char*)memchr(p, '\n', (size_t)(end - p));
    e = q ? q : end;
    p = q ? q + 1 : end;
    if (e > b && e[-1] == '\r') --e;
    return true;
  }
};

// parse unsigned/negative decimal integers from [b, e)
inline bool next_int(const char*& b, const char* e, long long& out) {
  while (b < e && (*b == ' ' || *b == '\t')) ++b;
  if (b >= e) return false;
  bool neg = false;
  if (*b == '-') { neg = true; ++b; }
  if (b >= e || *b < '0' || *b > '9') throw std::runtime_error("graph file: bad token");
  long long v = 0;
  while (b < e && *b >= '0' && *b <= '9') v = v * 10 + (*b++ - '0');
  out = neg ? -v : v;
  return true;
}

// Layout of a vertex line: [size] [weight] (neighbour [edge weight])*.
struct LineFormat {
  bool vsize, vw, ew;
  long long n;
};

inline bool comment_line(const char* b, const char* e) {
  while (b < e && (*b == ' ' || *b == '\t')) ++b;
  return b < e && *b == '%';
}

// One vertex line: its weight into vw, its neighbours (0-based) and edge
// weights appended to adj / w.
void parse_vertex_line(const char* b, const char* e, const LineFormat& lf, int32_t& vw, std::vector<int32_t>& adj,
                       std::vector<int32_t>& w) {
  long long x;
  if (lf.vsize && !next_int(b, e, x)) throw std::runtime_error("graph file: missing vertex size");
  if (lf.vw) {
    if (!next_int(b, e, x)) throw std::runtime_error("graph file: missing vertex weight");
    vw = (int32_t)x;
  }
  while (next_int(b, e, x)) {
    if (x < 1 || x > lf.n) throw std::runtime_error("graph file: neighbour id out of range");
    adj.push_back((int32_t)(x - 1));
    long long ew = 1;
    if (lf.ew && !next_int(b, e, ew)) throw std::runtime_error("graph file: missing edge weight");
    w.push_back((int32_t)ew);
  }
}

// Files above this size are parsed by several threads.
constexpr size_t kParallelParseBytes = (size_t)8 << 20;

// The body [p, end) split at line starts into T chunks.  Pass 1 counts each
// chunk's vertex lines, so every chunk knows the global index of its first
// vertex; pass 2 parses the lines of vertices 0..n-1 (lines beyond them are
// never read, as in the sequential reading); the chunks are then placed
// one after the other.  An error is reported for the first failing vertex in
// file order, the one the sequential reading would stop at.  Returns the
// number of vertex lines read (<= n).
long long parse_parallel(const char* p, const char* end, int T, const LineFormat& lf, std::vector<int32_t>& xadj,
                         std::vector<int32_t>& vwgt, std::vector<int32_t>& adjncy, std::vector<int32_t>& adjwgt) {
  std::vector<const char*> cut(T + 1);
  cut[0] = p;
  cut[T] = end;
  for (int t = 1; t < T; ++t) {
    const char* q = p + (size_t)(end - p) * t / T;
    if (q < cut[t - 1]) q = cut[t - 1];
    if (q > p && q < end && q[-1] != '\n') {
      const char* nl = (const char*)memchr(q, '\n', (size_t)(end - q));
      q = nl ? nl + 1 : end;
    }
    cut[t] = q;
  }
  std::vector<long long> lines(T, 0);
  auto run = [&](auto&& body) {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(body, t);
    for (auto& x : th) x.join();
  };
  run([&](int t) {
    Cursor cc{cut[t], cut[t + 1]};
    const char *b, *e;
    long long k = 0;
    while (cc.line(b, e))
      if (!comment_line(b, e)) ++k;
    lines[t] = k;
  });
  std::vector<long long> first(T + 1, 0);
  for (int t = 0; t < T; ++t) first[t + 1] = first[t] + lines[t];
  struct Part {
    std::vector<int32_t> deg, adj, w;
    long long err_v = -1;
    std::string err;
  };
  std::vector<Part> part(T);
  run([&](int t) {
    Part& P = part[t];
    Cursor cc{cut[t], cut[t + 1]};
    const char *b, *e;
    long long v = first[t];
    while (v < lf.n && cc.line(b, e)) {
      if (comment_line(b, e)) continue;
      const size_t before = P.adj.size();
      try {
        parse_vertex_line(b, e, lf, vwgt[(size_t)v], P.adj, P.w);
      } catch (const std::exception& ex) {
        P.err_v = v;
        P.err = ex.what();
        return;
      }
      P.deg.push_back((int32_t)(P.adj.size() - before));
      ++v;
    }
  });
  for (int t = 0; t < T; ++t)
    if (part[t].err_v >= 0) throw std::runtime_error(part[t].err);   // chunks are in file order
  size_t total = 0;
  for (const Part& P : part) total += P.adj.size();
  if (total >= ((size_t)1 << 31)) throw std::runtime_error("graph file: too many adjacency entries");
  adjncy.resize(total);
  adjwgt.resize(total);
  long long v = 0;
  size_t at = 0;
  for (const Part& P : part) {
    for (int32_t d : P.deg) {
      at += (size_t)d;
      xadj[(size_t)++v] = (int32_t)at;
    }
  }
  std::vector<size_t> eoff(T + 1, 0);
  for (int t = 0; t < T; ++t) eoff[t + 1] = eoff[t] + part[t].adj.size();
  run([&](int t) {
    std::copy(part[t].adj.begin(), part[t].adj.end(), adjncy.begin() + eoff[t]);
    std::copy(part[t].w.begin(), part[t].w.end(), adjwgt.begin() + eoff[t]);
  });
  return v;
}

}  // namespace

}  // namespace gk

// The header line of a METIS .graph text: "n m [fmt [ncon]]", after any
// comment and blank lines; the same rules as gk::Graph's reading.
bool gkw::parse_metis_header(const char* buf, size_t size, bool reference_quirks, gkw::MetisHeader* out,
                             std::string* err) {
  try {
    gk::Cursor c{buf, buf + size};
    const char *b, *e;
    for (;;) {
      if (!c.line(b, e)) throw std::runtime_error("graph file: missing header");
      const char* t = b;
      while (t < e && (*t == ' ' || *t == '\t')) ++t;
      if (t < e && *t == '%') continue;
      if (t == e) continue;
      break;
    }
    long long n = 0, m = 0, fmt = 0, ncon = 1;
    if (!gk::next_int(b, e, n) || !gk::next_int(b, e, m)) throw std::runtime_error("graph file: bad header");
    std::string fmt_s;
    {
      const char* t = b;
      while (t < e && (*t == ' ' || *t == '\t')) ++t;
      const char* s0 = t;
      while (t < e && *t >= '0' && *t <= '9') ++t;
      fmt_s.assign(s0, t);
      b = t;
      if (!fmt_s.empty()) fmt = std::atoll(fmt_s.c_str());
      long long nc;
      if (gk::next_int(b, e, nc)) ncon = nc;
    }
    if (n < 0 || m < 0 || n >= (1LL << 31) || 2 * m >= (1LL << 31))
      throw std::runtime_error("graph file: sizes out of range");
    if (ncon != 1) throw std::runtime_error("graph file: only ncon = 1 is supported");
    out->n = n;
    out->m = m;
    out->vsize = (fmt / 100) % 10 == 1;
    out->vw = (fmt / 10) % 10 == 1;
    out->ew = fmt % 10 == 1;
    if (reference_quirks) {   // graph.hpp:93-97,125-137
      out->vsize = out->vw = false;
      out->ew = fmt_s == "11";
    }
    out->body = (size_t)(c.p - buf);
    return true;
  } catch (const std::exception& ex) {
    *err = ex.what();
    return false;
  }
}

namespace gk {

Graph::Graph(const std::string& input_path, bool reference_quirks) {
  const std::string buf = read_file(input_path);
  Cursor c{buf.data(), buf.data() + buf.size()};
  const char *b, *e;
  // header (skip comment lines)
  for (;;) {
    if (!c.line(b, e)) throw std::runtime_error("graph file: missing header");
    const char* t = b;
    while (t < e && (*t == ' ' || *t == '\t')) ++t;
    if (t < e && *t == '%') continue;
    if (t == e) continue;
    break;
  }
  long long n = 0, m = 0, fmt = 0, ncon = 1;
  if (!next_int(b, e, n) || !next_int(b, e, m)) throw std::runtime_error("graph file: bad header");
  std::string fmt_s;
  {
    const char* t = b;
    while (t < e && (*t == ' ' || *t == '\t')) ++t;
    const char* s = t;
    while (t < e && *t >= '0' && *t <= '9') ++t;
    fmt_s.assign(s, t);
    b = t;
    if (!fmt_s.empty()) fmt = std::atoll(fmt_s.c_str());
    long long nc;
    if (next_int(b, e, nc)) ncon = nc;
  }
  if (n < 0 || m < 0 || n >= (1LL << 31) || 2 * m >= (1LL << 31))
    throw std::runtime_error("graph file: sizes out of range");
  if (ncon != 1) throw std::runtime_error("graph file: only ncon = 1 is supported");
  bool has_vsize = (fmt / 100) % 10 == 1;
  bool has_vw = (fmt / 10) % 10 == 1;
  bool has_ew = fmt % 10 == 1;
  bool pairs_only = false;
  if (reference_quirks) {
    // graph.hpp:93-97,125-137: "11" means neighbour/weight pairs, nothing else is read
    pairs_only = (fmt_s == "11");
    has_vsize = has_vw = false;
    has_ew = pairs_only;
  }
  const LineFormat lf{has_vsize, has_vw, has_ew, n};
  xadj_.assign((size_t)n + 1, 0);
  vwgt_.assign((size_t)n, 1);
  adjncy_.clear();
  adjwgt_.clear();
  const size_t body = (size_t)(c.end - c.p);
  const unsigned hw = std::thread::hardware_concurrency();
  const int T = body < kParallelParseBytes ? 1 : (int)std::min<unsigned>(std::max(hw, 1u), 32u);
  long long v = 0;
  if (T == 1) {
    adjncy_.reserve((size_t)(2 * m));
    adjwgt_.reserve((size_t)(2 * m));
    while (v < n) {
      if (!c.line(b, e)) break;
      if (comment_line(b, e)) continue;
      parse_vertex_line(b, e, lf, vwgt_[(size_t)v], adjncy_, adjwgt_);
      ++v;
      xadj_[(size_t)v] = (int32_t)adjncy_.size();
    }
  } else {
    v = parse_parallel(c.p, c.end, T, lf, xadj_, vwgt_, adjncy_, adjwgt_);
  }
  for (; v < n; ++v) xadj_[(size_t)v + 1] = (int32_t)adjncy_.size();   // missing trailing lines: isolated
  if (!reference_quirks && (long long)adjncy_.size() != 2 * m)
    throw std::runtime_error("graph file: header says " + std::to_string(m) + " edges, found " +
                             std::to_string(adjncy_.size()) + " adjacency entries (expected 2m)");
}

Graph::Graph(std::vector<int32_t> xadj, std::vector<int32_t> adjncy0, std::vector<int32_t> adjwgt,
             std::vector<int32_t> vwgt)
    : xadj_(std::move(xadj)), adjncy_(std::move(adjncy0)), adjwgt_(std::move(adjwgt)), vwgt_(std::move(vwgt)) {
  if (adjwgt_.empty()) adjwgt_.assign(adjncy_.size(), 1);
  if (vwgt_.empty() && !xadj_.empty()) vwgt_.assign(xadj_.size() - 1, 1);
}

Graph::~Graph() = default;

const int* Graph::get_adjncy() {
  if (adjncy1_.size() != adjncy_.size()) {
    adjncy1_.resize(adjncy_.size());
    for (size_t i = 0; i < adjncy_.size(); ++i) adjncy1_[i] = adjncy_[i] + 1;
  }
  return adjncy1_.data();
}
const int* Graph::get_adjp() { return xadj_.data(); }
const int* Graph::get_adjwgt() { return adjwgt_.data(); }
const int* Graph::get_vwgt() { return vwgt_.data(); }
size_t Graph::get_num_vertex() { return xadj_.empty() ? 0 : xadj_.size() - 1; }
size_t Graph::get_num_edge() { return adjncy_.size(); }
int Graph::get_total_vertex_weight() { return std::accumulate(vwgt_.begin(), vwgt_.end(), 0); }

// One part id per line (graph.hpp:227-240), formatted into one buffer.
static std::string format_parts(const int32_t* part, size_t n) {
  std::string buf(n * 12 + 1, '\0');
  char* p = &buf[0];
  char* const end = p + buf.size();
  for (size_t i = 0; i < n; ++i) {
    p = std::to_chars(p, end, part[i]).ptr;
    *p++ = '\n';
  }
  buf.resize((size_t)(p - buf.data()));
  return buf;
}

void Graph::dump_result(const std::vector<int>& vertex_partition, const std::string& file_name) {
  char cwd[4096];
  std::string dir = getcwd(cwd, sizeof(cwd)) ? std::string(cwd) : std::string(".");
  const std::string out_path = dir + "/" + file_name + ".out";
  std::cout << "out_path:" << out_path << "\n";
  FILE* f = fopen(out_path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot open output file " + out_path);
  static_assert(sizeof(int) == sizeof(int32_t), "part ids are 32-bit");
  const std::string buf = format_parts(reinterpret_cast<const int32_t*>(vertex_partition.data()),
                                       vertex_partition.size());
  fwrite(buf.data(), 1, buf.size(), f);
  fclose(f);
}

gkw_csr Graph::csr() const {
  gkw_csr c;
  c.n = (int32_t)(xadj_.empty() ? 0 : xadj_.size() - 1);
  c.nnz = (int64_t)adjncy_.size();
  c.xadj = xadj_.data();
  c.adjncy = adjncy_.data();
  c.adjwgt = adjwgt_.data();
  c.vwgt = vwgt_.data();
  return c;
}

// ---------------------------------------------------------------------------
GraphPartitioner::GraphPartitioner(const gkw_options* opt, int device) {
  if (opt) opt_ = *opt;
  else gkw_default_options(&opt_);
  if (gkw_create(&h_, device) != GKW_OK) throw std::runtime_error(std::string("gkw_create: ") + gkw_last_error());
}

GraphPartitioner::~GraphPartitioner() { gkw_destroy(h_); }

PartitionResult GraphPartitioner::partition_with_stats(const Graph& g, int k) {
  PartitionResult r;
  gkw_csr c = g.csr();
  r.part.assign((size_t)c.n, 0);
  gkw_status st = gkw_partition(h_, &c, k, &opt_, r.part.data(), &r.cut, &r.stats);
  if (st != GKW_OK) throw std::runtime_error(std::string("gkw_partition: ") + gkw_last_error());
  return r;
}

std::vector<int> GraphPartitioner::partition(const Graph& g, int k) { return partition_with_stats(g, k).part; }

std::vector<PartitionResult> GraphPartitioner::partition_multi_k(const Graph& g, const std::vector<int>& ks) {
  gkw_csr c = g.csr();
  const size_t n = (size_t)c.n, nk = ks.size();
  std::vector<int32_t> kk(ks.begin(), ks.end()), parts(std::max<size_t>(n * nk, 1));
  std::vector<int64_t> cuts(std::max<size_t>(nk, 1));
  gkw_status st = gkw_partition_multi_k(h_, &c, (int32_t)nk, kk.data(), &opt_, parts.data(), cuts.data());
  if (st != GKW_OK) throw std::runtime_error(std::string("gkw_partition_multi_k: ") + gkw_last_error());
  std::vector<PartitionResult> out(nk);
  for (size_t q = 0; q < nk; ++q) {
    out[q].part.assign(parts.begin() + q * n, parts.begin() + (q + 1) * n);
    out[q].cut = cuts[q];
    std::memset(&out[q].stats, 0, sizeof(out[q].stats));
  }
  return out;
}

// ---------------------------------------------------------------------------
// METIS as the initial partitioner (the reference's behaviour), loaded at run
// time.  idx_t is 64-bit in the reference's bundled METIS (metis.h:33).
namespace {
typedef int (*metis_kway_fn)(int64_t*, int64_t*, int64_t*, int64_t*, int64_t*, int64_t*, int64_t*, int64_t*,
                             double*, double*, int64_t*, int64_t*, int64_t*);

int32_t metis_init_cb(void* user, int32_t n, const int32_t* xadj, const int32_t* adjncy, const int32_t* adjwgt,
                      const int32_t* vwgt, int32_t k, int32_t* part_out) {
  metis_kway_fn fn = (metis_kway_fn)user;
  const int64_t m = xadj[n];
  std::vector<int64_t> x(n + 1), a(std::max<int64_t>(m, 1)), w(std::max<int64_t>(m, 1)),
      vw(std::max<int32_t>(n, 1)), p(std::max<int32_t>(n, 1));
  for (int32_t i = 0; i <= n; ++i) x[i] = xadj[i];
  for (int64_t e = 0; e < m; ++e) { a[e] = adjncy[e]; w[e] = adjwgt[e]; }
  for (int32_t i = 0; i < n; ++i) vw[i] = vwgt[i];
  int64_t nv = n, ncon = 1, np = k, cut = 0;
  int rc = fn(&nv, &ncon, x.data(), a.data(), vw.data(), nullptr, w.data(), &np, nullptr, nullptr, nullptr, &cut,
              p.data());
  if (rc != 1) return -1;
  for (int32_t i = 0; i < n; ++i) part_out[i] = (int32_t)p[i];
  return 0;
}
}  // namespace

bool use_metis_init(gkw_options* opt, const std::string& path, bool recursive) {
  void* h = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
  if (!h) return false;
  // METIS_PartGraphRecursive takes the same arguments (metis.h:185)
  void* fn = dlsym(h, recursive ? "METIS_PartGraphRecursive" : "METIS_PartGraphKway");
  if (!fn) return false;
  opt->init_method = GKW_INIT_CALLBACK;
  opt->init_fn = metis_init_cb;
  opt->init_user = fn;
  return true;
}

}  // namespace gk

// ---------------------------------------------------------------------------
// C ABI helpers for files.
extern "C" {

gkw_status gkw_read_metis(const char* path, int32_t reference_quirks, int32_t* n_out, int64_t* nnz_out,
                          int32_t** xadj, int32_t** adjncy, int32_t** adjwgt, int32_t** vwgt) {
  if (!path || !n_out || !nnz_out || !xadj || !adjncy || !adjwgt || !vwgt) return GKW_E_INVALID;
  try {
    gk::Graph g(path, reference_quirks != 0);
    const size_t n = g.get_num_vertex(), m = g.get_num_edge();
    auto dup = [](const std::vector<int32_t>& v) {
      int32_t* p = (int32_t*)std::malloc(std::max<size_t>(v.size(), 1) * sizeof(int32_t));
      if (!p) throw std::bad_alloc();
      if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(int32_t));
      return p;
    };
    *xadj = dup(g.xadj());
    *adjncy = dup(g.adjncy0());
    *adjwgt = dup(g.adjwgt());
    *vwgt = dup(g.vwgt());
    *n_out = (int32_t)n;
    *nnz_out = (int64_t)m;
    return GKW_OK;
  } catch (const std::bad_alloc&) {
    return GKW_E_NOMEM;
  } catch (const std::exception& e) {
    gkw_io_set_error(e.what());
    return GKW_E_INVALID;
  }
}

gkw_status gkw_write_partition(const char* path, int32_t n, const int32_t* part) {
  if (!path || n < 0 || (n > 0 && !part)) return GKW_E_INVALID;
  FILE* f = fopen(path, "wb");
  if (!f) {
    gkw_io_set_error(std::string("cannot open ") + path);
    return GKW_E_INVALID;
  }
  const std::string buf = gk::format_parts(part, (size_t)n);
  size_t wr = fwrite(buf.data(), 1, buf.size(), f);
  fclose(f);
  return wr == buf.size() ? GKW_OK : GKW_E_INVALID;
}

void gkw_free(void* p) { std::free(p); }

}  // extern "C"

// ---------------------------------------------------------------------------
// graph_partitioner.hpp:222-365: parse, partition, print the four phase
// timers and the cut, write <cwd>/<out>.out.  Environment:
//   GKW_METIS_LIB=<path to libmetis.so>  initial partition by METIS, as the
//                                        reference does (default: on device)
//   GKW_METIS_RECURSIVE=1                with GKW_METIS_LIB: METIS's recursive
//                                        bisection instead of its k-way call
//   GKW_SEED=<n>                         seed of the device initial partition
void graph_partitioner(const std::string& GRAPH_FILE, const std::string& OUT_FILE, const int NUM_PARTITIONS) {
  // the file is parsed on the device, partitioned there, and the part ids are
  // formatted there; only the text crosses to and from the host
  gkw_options opt;
  gkw_default_options(&opt);
  if (const char* s = std::getenv("GKW_SEED")) opt.seed = std::strtoull(s, nullptr, 10);
  if (const char* lib = std::getenv("GKW_METIS_LIB")) {
    const char* rb = std::getenv("GKW_METIS_RECURSIVE");
    if (!gk::use_metis_init(&opt, lib, rb && *rb == '1'))
      throw std::runtime_error(std::string("cannot load METIS from ") + lib);
  }
  if (FILE* f = fopen(GRAPH_FILE.c_str(), "rb")) fclose(f);   // a missing file is reported before any device work
  else throw std::runtime_error("cannot open graph file: " + GRAPH_FILE);
  gkw_handle* h = nullptr;
  if (gkw_create(&h, 0) != GKW_OK) throw std::runtime_error(std::string("gkw_create: ") + gkw_last_error());
  struct Cleanup {
    gkw_handle* h;
    gkw_csr g{};
    int32_t* part = nullptr;
    ~Cleanup() {
      if (part) cudaFree(part);
      gkw_free_device_graph(&g);
      gkw_destroy(h);
    }
  } c{h};
  const auto t0 = std::chrono::steady_clock::now();
  if (gkw_read_metis_device(h, GRAPH_FILE.c_str(), 0, &c.g) != GKW_OK)
    throw std::runtime_error(gkw_last_error());
  const auto t1 = std::chrono::steady_clock::now();
  if (cudaMalloc((void**)&c.part, sizeof(int32_t) * std::max<size_t>((size_t)c.g.n, 1)) != cudaSuccess)
    throw std::runtime_error("cudaMalloc failed for the part ids");
  int64_t cut = 0;
  gkw_stats s{};
  if (gkw_partition_device(h, &c.g, NUM_PARTITIONS, &opt, c.part, &cut, &s) != GKW_OK)
    throw std::runtime_error(gkw_last_error());
  std::cout << "#################### Execution Time ################# \n";
  std::cout << "Total time: " << s.ms_total / 1000.0 << "s\n";
  std::cout << "Coarsen time: " << s.ms_coarsen / 1000.0 << "s\n";
  std::cout << "Init partition time: " << s.ms_init / 1000.0 << "s\n";
  std::cout << "Refinement time: " << s.ms_refine / 1000.0 << "s\n";
  std::cout << "#################### Partition Summary ################# \n";
  std::cout << "***** h_cutsize " << cut << '\n';
  if ((double)s.max_part_weight > (double)s.maxw)
    std::cout << "!!!@@@ ERROR, max part weight " << s.max_part_weight << " is above " << s.maxw << '\n';
  char cwd[4096];
  const std::string dir = getcwd(cwd, sizeof(cwd)) ? std::string(cwd) : std::string(".");
  const std::string out_path = dir + "/" + OUT_FILE + ".out";
  std::cout << "out_path:" << out_path << "\n";
  if (gkw_write_partition_device(h, out_path.c_str(), c.g.n, c.part) != GKW_OK)
    throw std::runtime_error(gkw_last_error());
  const auto t2 = std::chrono::steady_clock::now();
  if (std::getenv("GKW_TIMES"))
    std::cout << "read " << std::chrono::duration<double>(t1 - t0).count() << "s, end to end "
              << std::chrono::duration<double>(t2 - t0).count() << "s\n";
}
