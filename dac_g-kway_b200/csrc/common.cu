// Errors, the device pool, handles and the device-wide exclusive scan.
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>

#include "gkw_internal.cuh"

namespace gkw {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
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
  return base;
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
// "not published".  Tiles take tickets from a persistent 64-bit counter in
// launch order (tile = ticket - base, base = tickets handed out by earlier
// calls), so a tile only waits on tiles that already hold an SM.  A wait
// longer than kScanSpinCycles sets the error word and the tile continues
// (the result is then reported as an error, never a hang).
constexpr long long kScanSpinCycles = 2000000000ll;

__global__ void __launch_bounds__(kScanThreads) k_scan_1pass(const i32* in, i32* out, i64 n, i32* total,
                                                             ScanState* ss, u64 base, u64 epoch, i32 ntiles) {
  __shared__ i32 s_warp[33];
  __shared__ i32 s_tile;
  __shared__ i32 s_excl;
  if (threadIdx.x == 0) s_tile = (i32)(atomicAdd((unsigned long long*)&ss->ticket, 1ull) - base);
  __syncthreads();
  const i32 tile = s_tile;
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
  if (threadIdx.x == 0) {
    unsigned long long* st = (unsigned long long*)ss->tiles;
    const u64 tag = epoch << 34;
    i32 excl = 0;
    if (tile == 0) {
      atomicExch(&st[0], (unsigned long long)(tag | (2ull << 32) | (u32)agg));
    } else {
      atomicExch(&st[tile], (unsigned long long)(tag | (1ull << 32) | (u32)agg));
      i32 j = tile - 1;
      const long long t0 = clock64();
      while (j >= 0) {
        const u64 w = (u64)atomicAdd(&st[j], 0ull);
        const u32 status = (w >> 34) == epoch ? (u32)((w >> 32) & 3u) : 0u;
        if (status == 0) {
          if (clock64() - t0 > kScanSpinCycles) {
            atomicExch(&ss->err, 1);
            break;
          }
          continue;
        }
        excl += (i32)(u32)w;
        if (status == 2) break;
        --j;
      }
      atomicExch(&st[tile], (unsigned long long)(tag | (2ull << 32) | (u32)(excl + agg)));
    }
    s_excl = excl;
    if (tile == ntiles - 1 && total) *total = excl + agg;
  }
  __syncthreads();
  i32 run = off + s_excl;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (b0 + i < n) out[b0 + i] = run;
    run += v[i];
  }
}

__global__ void k_set_i32(i32* p, i32 v) { *p = v; }

void exclusive_scan_i32(Handle& h, const i32* in, i32* out, i64 n, i32* total) {
  if (n <= 0) {
    if (total) launch(k_set_i32, 1, 1, 0, h.stream, total, 0);
    GKW_CHECK_LAUNCH();
    return;
  }
  const i64 nt64 = (n + kScanTile - 1) / kScanTile;
  GKW_REQUIRE(nt64 < (i64)1 << 30, GKW_E_UNSUPPORTED, "scan too large");
  const i32 nt = (i32)nt64;
  if (h.scan_tiles_cap < nt) {
    if (h.scan) GKW_CUDA(cudaFree(h.scan));
    h.scan = nullptr;
    const i32 cap = std::max(nt, 1024);
    GKW_CUDA(cudaMalloc(&h.scan, sizeof(ScanState) + sizeof(u64) * (size_t)cap));
    GKW_CUDA(cudaMemset(h.scan, 0, sizeof(ScanState) + sizeof(u64) * (size_t)cap));
    h.scan_tiles_cap = cap;
    h.scan_tickets = 0;
    h.scan_epoch = 0;
  }
  h.scan_epoch += 1;
  GKW_REQUIRE(h.scan_epoch < ((u64)1 << 29), GKW_E_INTERNAL, "scan epoch overflow");
  launch(k_scan_1pass, nt, kScanThreads, 0, h.stream, in, out, n, total, h.scan, h.scan_tickets, h.scan_epoch,
         nt);
  GKW_CHECK_LAUNCH();
  h.scan_tickets += (u64)nt;
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
