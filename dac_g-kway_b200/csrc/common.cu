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

__global__ void k_scan_reduce(const i32* __restrict__ in, i64 n, i32* __restrict__ partial) {
  __shared__ i32 s_warp[33];
  const i64 base = (i64)blockIdx.x * kScanTile + (i64)threadIdx.x * kScanItems;
  i32 s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) s += in[base + i];
  i32 total;
  block_exclusive_scan(s, s_warp, total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// single block: exclusive scan of the nb tile sums in place, grand total out
__global__ void k_scan_partials(i32* __restrict__ partial, i32 nb, i32* __restrict__ total_out) {
  __shared__ i32 s_warp[33];
  i32 carry = 0;
  for (i32 base = 0; base < nb; base += kScanTile) {
    i32 v[kScanItems];
    i32 s = 0;
    const i32 b0 = base + threadIdx.x * kScanItems;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      v[i] = (b0 + i < nb) ? partial[b0 + i] : 0;
      s += v[i];
    }
    i32 tot;
    i32 off = block_exclusive_scan(s, s_warp, tot) + carry;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      if (b0 + i < nb) partial[b0 + i] = off;
      off += v[i];
    }
    carry += tot;
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void k_scan_down(const i32* in, i32* out, i64 n, const i32* __restrict__ partial) {
  __shared__ i32 s_warp[33];
  const i64 base = (i64)blockIdx.x * kScanTile + (i64)threadIdx.x * kScanItems;
  i32 v[kScanItems];
  i32 s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (base + i < n) ? in[base + i] : 0;
    s += v[i];
  }
  i32 tot;
  i32 off = block_exclusive_scan(s, s_warp, tot) + partial[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = off;
    off += v[i];
  }
}

__global__ void k_set_i32(i32* p, i32 v) { *p = v; }

void exclusive_scan_i32(Handle& h, const i32* in, i32* out, i64 n, i32* total) {
  if (n <= 0) {
    if (total) {
      launch(k_set_i32, 1, 1, 0, h.stream, total, 0);
      GKW_CHECK_LAUNCH();
    }
    return;
  }
  const i64 nb64 = (n + kScanTile - 1) / kScanTile;
  GKW_REQUIRE(nb64 < (i64)1 << 30, GKW_E_UNSUPPORTED, "scan too large");
  const i32 nb = (i32)nb64;
  Pool::Mark mk = h.scratch.mark();
  i32* partial = h.scratch.alloc_n<i32>(nb);
  launch(k_scan_reduce, nb, kScanThreads, 0, h.stream, in, n, partial);
  GKW_CHECK_LAUNCH();
  launch(k_scan_partials, 1, kScanThreads, 0, h.stream, partial, nb, total);
  GKW_CHECK_LAUNCH();
  launch(k_scan_down, nb, kScanThreads, 0, h.stream, in, out, n, partial);
  GKW_CHECK_LAUNCH();
  h.scratch.release(mk);   // stream-ordered reuse is safe: later kernels run after these
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
