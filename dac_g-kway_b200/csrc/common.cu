// Errors, the device pool, handles and the device-wide exclusive scan.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include "gkw_internal.cuh"

namespace gkw {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void uncount_launches(uint64_t n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
uint64_t launch_total() { return g_launches.load(std::memory_order_relaxed); }

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error_cstr() { return g_last_error.c_str(); }

}  // namespace gkw

// error hook for the host-only file helpers (graph_io.cpp)
extern "C" void gkw_io_set_error(const std::string& msg) { gkw::set_error(msg); }

namespace gkw {

// ---------------------------------------------------------------------------
// Pool
// ---------------------------------------------------------------------------
Pool::~Pool() {
  for (auto& c : chunks_) cudaFree(c.base);
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

void* Pool::alloc(size_t bytes) {
  bytes = align_up(bytes == 0 ? 1 : bytes, 256);
  while (cur_ < chunks_.size()) {
    Chunk& c = chunks_[cur_];
    if (c.top + bytes <= c.cap) {
      void* p = c.base + c.top;
      c.top += bytes;
      note_use();
      return p;
    }
    if (cur_ + 1 < chunks_.size()) {
      ++cur_;
      chunks_[cur_].top = 0;
      continue;
    }
    break;
  }
  // need a new chunk (appended after the current one)
  size_t cap = std::max(bytes, min_chunk_);
  if (!chunks_.empty()) cap = std::max(cap, chunks_.back().cap);   // geometric-ish growth
  char* base = nullptr;
  cudaError_t e = cudaMalloc(&base, cap);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error{GKW_E_NOMEM, "device allocation of " + std::to_string(cap) + " bytes failed: " +
                                 cudaGetErrorString(e)};
  }
  chunks_.push_back({base, cap, bytes});
  cur_ = chunks_.size() - 1;
  note_use();
  return base;
}

void Pool::note_use() {
  size_t used = chunks_[cur_].top;
  for (size_t i = 0; i < cur_; ++i) used += chunks_[i].cap;
  peak_ = std::max(peak_, used);
}

void Pool::trim() {
  for (auto& c : chunks_) GKW_REQUIRE(c.top == 0, GKW_E_INTERNAL, "trim of a pool in use");
  for (auto& c : chunks_) cudaFree(c.base);
  chunks_.clear();
  cur_ = 0;
}

void Pool::release(Mark m) {
  if (chunks_.empty()) return;
  cur_ = m.chunk;
  chunks_[cur_].top = m.top;
  for (size_t i = cur_ + 1; i < chunks_.size(); ++i) chunks_[i].top = 0;
}

size_t Pool::capacity() const {
  size_t s = 0;
  for (auto& c : chunks_) s += c.cap;
  return s;
}

void Pool::reserve(size_t bytes) {
  if (!chunks_.empty() && chunks_[0].cap >= bytes) return;
  bool all_free = true;
  for (auto& c : chunks_) all_free &= (c.top == 0);
  if (!all_free) return;
  for (auto& c : chunks_) cudaFree(c.base);
  chunks_.clear();
  cur_ = 0;
  char* base = nullptr;
  cudaError_t e = cudaMalloc(&base, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error{GKW_E_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed: " +
                                 cudaGetErrorString(e)};
  }
  chunks_.push_back({base, bytes, 0});
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan (reduce, scan the tile sums, scan down).
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Exclusive block scan of one value per thread; returns the block total.
__device__ __forceinline__ i32 block_exclusive_scan(i32 x, i32* s_warp, i32& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  i32 inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    i32 y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    i32 w = lane < nw ? s_warp[lane] : 0;
    i32 wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      i32 y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) s_warp[lane] = wi - w;   // exclusive warp offsets
    if (lane == nw - 1) s_warp[32] = wi;     // block total
  }
  __syncthreads();
  i32 r = inc - x + s_warp[wid];
  total = s_warp[32];
  __syncthreads();   // s_warp reusable by the caller afterwards
  return r;
}

// Single-pass scan with decoupled look-back.  Tile t publishes its aggregate
// (status 1) and then its inclusive prefix (status 2) in a status word
// (epoch << 34 | status << 32 | value); a word of an older epoch reads as
// "not published".  Tiles take tickets in launch order, so a tile only waits
// on tiles that already hold an SM.  The ticket counter, the epoch and a
// finished-tile counter live on the device: the last tile to finish resets
// the counters and advances the epoch for the next scan, so a scan needs no
// per-call argument from the host (it can be replayed from a CUDA graph).  A
// wait longer than kScanSpinCycles sets the error word and the tile
// continues (the result is then reported as an error, never a hang).
constexpr long long kScanSpinCycles = 2000000000ll;
constexpr u32 kScanEpochMask = (1u << 29) - 1;

__device__ __forceinline__ u64 ld_relaxed_gpu_u64(const unsigned long long* p) {
  u64 v;
  asm volatile("ld.relaxed.gpu.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_1pass(const i32* in, i32* out, i64 n, i32* total,
                                                             ScanState* ss, i32 ntiles) {
  __shared__ i32 s_warp[33];
  __shared__ i32 s_tile;
  __shared__ i32 s_excl;
  __shared__ u32 s_epoch;
  if (threadIdx.x == 0) {
    s_tile = (i32)atomicAdd(&ss->ticket, 1u);
    s_epoch = *(volatile u32*)&ss->epoch;   // set by the previous scan, stream-ordered before this one
  }
  __syncthreads();
  const i32 tile = s_tile;
  const u64 epoch = s_epoch;
  const i64 b0 = (i64)tile * kScanTile + (i64)threadIdx.x * kScanItems;
  i32 v[kScanItems];
  i32 sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (b0 + i < n) ? in[b0 + i] : 0;
    sum += v[i];
  }
  i32 agg;
  const i32 off = block_exclusive_scan(sum, s_warp, agg);
  if (threadIdx.x < 32) {
    // warp 0 looks back 32 predecessors per step: every lane waits for its
    // predecessor's word, the nearest inclusive prefix ends the walk
    const int lane = threadIdx.x;
    unsigned long long* st = (unsigned long long*)ss->tiles;
    const u64 tag = epoch << 34;
    i32 excl = 0;
    if (tile == 0) {
      if (lane == 0) atomicExch(&st[0], (unsigned long long)(tag | (2ull << 32) | (u32)agg));
    } else {
      if (lane == 0) atomicExch(&st[tile], (unsigned long long)(tag | (1ull << 32) | (u32)agg));
      i64 hi = (i64)tile - 1;
      const long long t0 = clock64();
      for (;;) {
        const i64 j = hi - lane;
        u32 status = 2, val = 0;   // before tile 0: an empty prefix
        if (j >= 0) {
          for (;;) {
            const u64 w = ld_relaxed_gpu_u64(&st[j]);
            status = (w >> 34) == epoch ? (u32)((w >> 32) & 3u) : 0u;
            val = (u32)w;
            if (status != 0) break;
            if (clock64() - t0 > kScanSpinCycles) {
              atomicExch(&ss->err, 1);
              status = 2;
              val = 0;
              break;
            }
          }
        }
        const u32 m2 = __ballot_sync(0xffffffffu, status == 2);
        const int first2 = m2 ? __ffs(m2) - 1 : 32;   // nearest published prefix
        i32 add = lane <= first2 ? (i32)val : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) add += __shfl_xor_sync(0xffffffffu, add, o);
        excl += add;
        if (m2) break;
        hi -= 32;
      }
      if (lane == 0) atomicExch(&st[tile], (unsigned long long)(tag | (2ull << 32) | (u32)(excl + agg)));
    }
    if (lane == 0) {
      s_excl = excl;
      if (tile == ntiles - 1 && total) *total = excl + agg;
    }
  }
  __syncthreads();
  i32 run = off + s_excl;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (b0 + i < n) out[b0 + i] = run;
    run += v[i];
  }
  if (threadIdx.x == 0) {
    // the last tile to finish: every other tile has taken its ticket, read
    // the epoch and published; reset for the next scan
    __threadfence();
    if (atomicAdd(&ss->done, 1u) == (u32)ntiles - 1) {
      ss->ticket = 0;
      ss->done = 0;
      ss->epoch = (ss->epoch + 1) & kScanEpochMask;
      __threadfence();
    }
  }
}

__global__ void k_set_i32(i32* p, i32 v) { *p = v; }

// A scan that fits one tile: one CTA, no tickets, status words or look-back
// (the single-pass scan's bookkeeping is several dependent round trips to L2,
// most of a small scan's time).
__global__ void __launch_bounds__(kScanThreads) k_scan_small(const i32* in, i32* out, i32 n, i32* total) {
  __shared__ i32 s_warp[33];
  const i32 b0 = threadIdx.x * kScanItems;
  i32 v[kScanItems];
  i32 sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (b0 + i < n) ? in[b0 + i] : 0;
    sum += v[i];
  }
  i32 agg;
  i32 run = block_exclusive_scan(sum, s_warp, agg);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (b0 + i < n) out[b0 + i] = run;
    run += v[i];
  }
  if (threadIdx.x == 0 && total) *total = agg;
}

void exclusive_scan_i32(Handle& h, const i32* in, i32* out, i64 n, i32* total) {
  if (n <= 0) {
    if (total) launch(k_set_i32, 1, 1, 0, h.stream, total, 0);
    GKW_CHECK_LAUNCH();
    return;
  }
  if (n <= kScanTile) {
    launch(k_scan_small, 1, kScanThreads, 0, h.stream, in, out, (i32)n, total);
    GKW_CHECK_LAUNCH();
    return;
  }
  const i64 nt64 = (n + kScanTile - 1) / kScanTile;
  GKW_REQUIRE(nt64 < (i64)1 << 30, GKW_E_UNSUPPORTED, "scan too large");
  const i32 nt = (i32)nt64;
  // the device epoch wraps after 2^29 scans: before it could meet a status
  // word of the same epoch, start again from cleared state (never inside a
  // graph capture: a captured scan's epoch is read on the device)
  const bool fresh = h.scan_tiles_cap < nt || (h.scan_epoch >= kScanEpochMask - 4096 && !h.capturing);
  if (fresh) {
    GKW_REQUIRE(!h.capturing, GKW_E_INTERNAL, "scan state grown during a graph capture");
    // queued scans may still use the old state; the new state is cleared on
    // the handle's stream (which does not wait for the legacy stream), so the
    // scan below sees it cleared
    GKW_CUDA(cudaStreamSynchronize(h.stream));
    const i32 cap = std::max(nt, h.scan_tiles_cap < nt ? std::max(nt, 1024) : h.scan_tiles_cap);
    if (h.scan_tiles_cap < nt) {
      if (h.scan) GKW_CUDA(cudaFree(h.scan));
      h.scan = nullptr;
      GKW_CUDA(cudaMalloc(&h.scan, sizeof(ScanState) + sizeof(u64) * (size_t)cap));
      h.scan_tiles_cap = cap;
      graph_cache_clear(h);   // graphs hold the old state's address
    }
    GKW_CUDA(cudaMemsetAsync(h.scan, 0, sizeof(ScanState) + sizeof(u64) * (size_t)h.scan_tiles_cap, h.stream));
    h.scan_epoch = 0;
  }
  h.scan_epoch += 1;   // host mirror of the device epoch (wrap guard only)
  ++h.scans_enqueued;
  launch(k_scan_1pass, nt, kScanThreads, 0, h.stream, in, out, n, total, h.scan, nt);
  GKW_CHECK_LAUNCH();
}

namespace {
struct ClusterKey {
  const void* kern;
  i32 block;
  size_t smem;
  int device;
  bool operator<(const ClusterKey& o) const {
    if (kern != o.kern) return kern < o.kern;
    if (block != o.block) return block < o.block;
    if (smem != o.smem) return smem < o.smem;
    return device < o.device;
  }
};
std::mutex g_cluster_mu;
std::map<ClusterKey, i32> g_cluster_limit;
constexpr int kMaxDevices = 64;
std::mutex g_chain_mu[kMaxDevices];
cudaEvent_t g_chain_last[kMaxDevices] = {};
}  // namespace

i32 coop_cluster_limit(Handle& h, const void* kern, i32 block, size_t smem) {
  const ClusterKey key{kern, block, smem, h.device};
  {
    std::lock_guard<std::mutex> lk(g_cluster_mu);
    auto it = g_cluster_limit.find(key);
    if (it != g_cluster_limit.end()) return it->second;
  }
  i32 best = 1;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    cudaGetLastError();
  for (i32 c = 16; c >= 2; c >>= 1) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = c;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) == cudaSuccess && nclusters >= 1) {
      best = c;
      break;
    }
    cudaGetLastError();
  }
  std::lock_guard<std::mutex> lk(g_cluster_mu);
  g_cluster_limit[key] = best;
  return best;
}

i32 coop_grid(Handle& h, const void* kern, i32 want, i32 block, size_t smem) {
  want = std::max(want, 1);
  if (!h.narrow) return want;
  return std::min(want, coop_cluster_limit(h, kern, block, smem));
}

void launch_coop(Handle& h, const void* kern, i32 grid, i32 block, size_t smem, void** args) {
  GKW_REQUIRE(grid >= 1, GKW_E_INTERNAL, "empty grid");
  if (grid > 1 && grid <= coop_cluster_limit(h, kern, block, smem)) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h.stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = grid;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    GKW_CUDA(cudaLaunchKernelExC(&cfg, kern, args));
    count_launch();
    return;
  }
  if (grid == 1) {   // one CTA waits on no other
    GKW_CUDA(cudaLaunchKernel(kern, dim3(1), dim3(block), args, smem, h.stream));
    count_launch();
    return;
  }
  GKW_REQUIRE(h.device >= 0 && h.device < kMaxDevices, GKW_E_UNSUPPORTED, "device index too large");
  if (h.capturing) {   // in a graph: graph_run chains the whole graph instead
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h.stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    GKW_CUDA(cudaLaunchKernelExC(&cfg, kern, args));
    count_launch();
    h.capture_wide = true;
    return;
  }
  if (!h.coop_ev) GKW_CUDA(cudaEventCreateWithFlags(&h.coop_ev, cudaEventDisableTiming));
  std::lock_guard<std::mutex> lk(g_chain_mu[h.device]);
  if (g_chain_last[h.device] && g_chain_last[h.device] != h.coop_ev)
    GKW_CUDA(cudaStreamWaitEvent(h.stream, g_chain_last[h.device], 0));
  GKW_CUDA(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(block), args, smem, h.stream));
  count_launch();
  GKW_CUDA(cudaEventRecord(h.coop_ev, h.stream));
  g_chain_last[h.device] = h.coop_ev;
}

void graph_cache_clear(Handle& h) {
  for (Handle::GraphEntry& e : h.graphs)
    if (e.exec) cudaGraphExecDestroy(e.exec);
  h.graphs.clear();
}

bool graph_run(Handle& h, const std::string& key, const std::function<void()>& body) {
  if (!h.graphs_on || h.capturing) {
    body();
    return false;
  }
  Handle::GraphEntry* e = nullptr;
  for (Handle::GraphEntry& x : h.graphs)
    if (x.key == key) e = &x;
  if (!e) {   // first sight: run as is (pools grow, shapes settle)
    if (h.graphs.size() >= 64) graph_cache_clear(h);
    h.graphs.push_back(Handle::GraphEntry{key, 1});
    body();
    return false;
  }
  if (!e->exec) {   // second sight: capture, then run the graph
    const u64 l0 = launch_total(), s0 = h.scans_enqueued, ep0 = h.scan_epoch;
    cudaGraph_t g = nullptr;
    h.capture_wide = false;
    cudaError_t err = cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      h.capturing = true;
      try {
        body();
      } catch (...) {
        h.capturing = false;
        cudaStreamEndCapture(h.stream, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        uncount_launches(launch_total() - l0);
        h.scans_enqueued = s0;
        h.scan_epoch = ep0;
        h.graphs_on = false;   // the body needs something a capture cannot hold: run it plainly from now on
        body();
        return false;
      }
      h.capturing = false;
      err = cudaStreamEndCapture(h.stream, &g);
    }
    const u64 nl = launch_total() - l0, ns = h.scans_enqueued - s0;
    uncount_launches(nl);   // nothing ran yet
    h.scans_enqueued = s0;
    h.scan_epoch = ep0;
    if (err == cudaSuccess) err = cudaGraphInstantiate(&e->exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (err != cudaSuccess) {
      cudaGetLastError();
      e->exec = nullptr;
      h.graphs_on = false;
      body();
      return false;
    }
    e->launches = nl;
    e->scans = ns;
    e->wide = h.capture_wide;
  }
  if (e->wide) {   // wide launches of all handles take turns (launch_coop)
    GKW_REQUIRE(h.device >= 0 && h.device < kMaxDevices, GKW_E_UNSUPPORTED, "device index too large");
    if (!h.coop_ev) GKW_CUDA(cudaEventCreateWithFlags(&h.coop_ev, cudaEventDisableTiming));
    std::lock_guard<std::mutex> lk(g_chain_mu[h.device]);
    if (g_chain_last[h.device] && g_chain_last[h.device] != h.coop_ev)
      GKW_CUDA(cudaStreamWaitEvent(h.stream, g_chain_last[h.device], 0));
    GKW_CUDA(cudaGraphLaunch(e->exec, h.stream));
    GKW_CUDA(cudaEventRecord(h.coop_ev, h.stream));
    g_chain_last[h.device] = h.coop_ev;
  } else {
    GKW_CUDA(cudaGraphLaunch(e->exec, h.stream));
  }
  count_launches(e->launches);
  h.scans_enqueued += e->scans;
  h.scan_epoch += e->scans;
  return true;
}

// Drop a handle's chain event (the handle is going away).
void forget_coop_event(Handle& h) {
  if (!h.coop_ev) return;
  if (h.device >= 0 && h.device < kMaxDevices) {
    std::lock_guard<std::mutex> lk(g_chain_mu[h.device]);
    if (g_chain_last[h.device] == h.coop_ev) g_chain_last[h.device] = nullptr;
  }
  cudaEventDestroy(h.coop_ev);
  h.coop_ev = nullptr;
}

float balance_cap(i64 total_vwgt, i32 k, double eps) {
  return (float)((1.0 + eps) * (double)total_vwgt / (double)k);
}

float max_part_weight(i64 total_vwgt, i32 k, double eps) {
  // graph_partitioner.hpp:230: (float)W/(float)k * (1.0f + IMBALANCE_RATIO) + 1,
  // IMBALANCE_RATIO a double literal, result stored as float.
  float q = (float)(u32)total_vwgt / (float)k;
  return (float)((double)q * (1.0 + eps) + 1);
}

}  // namespace gkw
