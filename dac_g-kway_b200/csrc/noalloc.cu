// gkw_cut_noalloc: the exact edge cut and part weights of a partition without
// any device allocation and without a library handle.
//
// Who needs it: code that must not allocate device memory while it runs --
// a caller inside a region where allocation is forbidden or would break its
// own memory accounting (a serving loop that budgets every byte up front, a
// host thread that runs under a device-memory cap, a plugin that receives
// only pre-allocated buffers from its host application).  gkw_cut needs a
// handle, and gkw_create allocates a stream, pinned staging and device state.
//
// How: the kernel's accumulators (the cut, a bad-part flag and k part
// weights) live in the file-scope array g_cut_scratch below instead of pool
// memory.  That array is part of the library image: every GPU that loads the
// library holds kMaxParts + 2 int64 words (about 64 KB) until the process
// exits.  Host code cannot pass the array's name to a kernel (in host code it
// names a host-side stand-in, not device memory), so the first call on each
// device looks up its device address with cudaGetSymbolAddress, with that
// device current, and caches it; later calls reuse the cached address.  Make
// that first call outside any stream capture.
//
// Every call shares the one array: calls on the same device whose work
// overlaps on the GPU (different streams, no ordering) race on it.  Each call
// clears the words it uses before its kernel runs.
#include <cuda_runtime.h>

#include <mutex>

#include "gkw_internal.cuh"

namespace gkw {
namespace {

constexpr i32 kMaxParts = 8190;   // accumulators: cut, bad flag, kMaxParts part weights
constexpr i32 kMaxDevices = 64;

static __device__ __align__(256) long long g_cut_scratch[kMaxParts + 2];

std::mutex g_mu;
i64* g_addr[kMaxDevices] = {};
i32 g_sms[kMaxDevices] = {};

}  // namespace
}  // namespace gkw

using namespace gkw;

extern "C" gkw_status gkw_cut_noalloc(const gkw_csr* d_graph, const int32_t* d_part, int32_t k, void* stream,
                                      int64_t* cut_out, int64_t* pw_out) {
  if (!d_graph || d_graph->n < 0 || d_graph->nnz < 0 || d_graph->nnz >= ((int64_t)1 << 31)) {
    set_error("gkw_cut_noalloc: bad graph");
    return GKW_E_INVALID;
  }
  if (d_graph->n > 0 && (!d_graph->xadj || !d_graph->vwgt || !d_part)) {
    set_error("gkw_cut_noalloc: NULL array");
    return GKW_E_INVALID;
  }
  if (d_graph->nnz > 0 && (!d_graph->adjncy || !d_graph->adjwgt)) {
    set_error("gkw_cut_noalloc: NULL adjacency");
    return GKW_E_INVALID;
  }
  if (k < 1 || k > kMaxParts) {
    set_error("gkw_cut_noalloc: k must be in [1, 8190]");
    return GKW_E_UNSUPPORTED;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error(std::string("gkw_cut_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return GKW_E_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("gkw_cut_noalloc: device index too large (the address table has " + std::to_string(kMaxDevices) +
              " entries)");
    return GKW_E_UNSUPPORTED;
  }
  i64* acc = nullptr;
  i32 sms = 0;
  {
    // set-up once per device, with that device current
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_cut_scratch);
      if (e != cudaSuccess || !p) {
        set_error(std::string("gkw_cut_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return GKW_E_CUDA;
      }
      int n_sm = 0;
      e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) {
        set_error(std::string("gkw_cut_noalloc: cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
        return GKW_E_CUDA;
      }
      g_sms[dev] = n_sm;
      g_addr[dev] = static_cast<i64*>(p);
    }
    acc = g_addr[dev];
    sms = g_sms[dev];
  }
  try {
    DevGraph g;
    g.n = d_graph->n;
    g.m = d_graph->nnz;
    g.xadj = d_graph->xadj;
    g.adjncy = d_graph->adjncy;
    g.adjwgt = d_graph->adjwgt;
    g.vwgt = d_graph->vwgt;
    GKW_CUDA(cudaMemsetAsync(acc, 0, sizeof(i64) * ((size_t)k + 2), st));
    launch_cut_pw(st, sms, g, d_part, k, acc);
    i64 head[2] = {0, 0};
    GKW_CUDA(cudaMemcpyAsync(head, acc, sizeof(i64) * 2, cudaMemcpyDeviceToHost, st));
    if (pw_out) GKW_CUDA(cudaMemcpyAsync(pw_out, acc + 2, sizeof(i64) * (size_t)k, cudaMemcpyDeviceToHost, st));
    GKW_CUDA(cudaStreamSynchronize(st));
    if (head[1] != 0) {
      set_error("gkw_cut_noalloc: part id out of range [0, k)");
      return GKW_E_INVALID;
    }
    if (cut_out) *cut_out = head[0];
  } catch (const Error& err) {
    set_error(err.msg);
    return err.st;
  }
  return GKW_OK;
}
