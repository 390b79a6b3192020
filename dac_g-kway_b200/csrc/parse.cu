// METIS .graph reading and part-id writing on the device (the reference does
// both on the host: gkway/graph.hpp:70-152 and :227-240).
//
// The header line is read on the host (parse_metis_header, graph_io.cpp);
// the body's bytes are copied to the device once and parsed there by passes
// over 4096-byte tiles, each thread taking 16 bytes with one 128-bit load:
//   1. newlines per tile, scanned over the tiles;
//   2. every line's start and end ('\r' before the newline dropped);
//   3. each line's kind: a '%' comment, or the next vertex line (lines after
//      the n-th vertex line are never read, as on the host);
//   4. tokens per tile over the vertex lines (a digit run, or '-' and digits;
//      any other character but blank, tab and the line's newline is a bad
//      token), scanned over the tiles; then every token's value, line and
//      offset, and each vertex line's first token;
//   5. each vertex's degree from its token count and the line layout
//      ([size] [weight] (neighbour [edge weight])*), scanned into xadj;
//   6. every token scattered to its slot; neighbour ids checked against n.
// Errors carry their byte position, so the one reported is the first in file
// order, the one the sequential host reading stops at, with the host's
// message.  Results equal gkw_read_metis's (standard format and the
// reference's "11" reading).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "device_util.cuh"

namespace gkw {

constexpr int kParseThreads = 256;
constexpr int kParseVec = 16;                               // bytes per thread (one 128-bit load)
constexpr i64 kParseTile = (i64)kParseThreads * kParseVec;   // bytes per CTA

enum : u32 { PE_BAD_TOKEN = 1, PE_MISSING_VSIZE = 2, PE_MISSING_VW = 3, PE_MISSING_EW = 4, PE_RANGE = 5 };

__device__ __forceinline__ bool pdigit(unsigned char c) { return c >= '0' && c <= '9'; }

// The thread's 16 bytes (zero past the body; the buffer is padded to whole tiles).
__device__ __forceinline__ void load16(const unsigned char* buf, i64 at, unsigned char (&c)[kParseVec]) {
  const uint4 q = *reinterpret_cast<const uint4*>(buf + at);
  const u32 w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int j = 0; j < kParseVec; ++j) c[j] = (unsigned char)(w[j >> 2] >> (8 * (j & 3)));
}

// Block-wide exclusive scan of one i32 per thread (kParseThreads threads).
__device__ __forceinline__ i32 parse_exscan(i32 x, i32* s_warp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  i32 inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const i32 y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const int nw = kParseThreads / 32;
    const i32 w = lane < nw ? s_warp[lane] : 0;
    i32 wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const i32 y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) s_warp[lane] = wi - w;
  }
  __syncthreads();
  const i32 r = inc - x + s_warp[wid];
  __syncthreads();
  return r;
}

// pass 1: newlines per tile
__global__ void __launch_bounds__(kParseThreads) k_tile_newlines(const unsigned char* __restrict__ buf, i64 B,
                                                                 i32* __restrict__ tile_nl) {
  __shared__ i32 s_red[kParseThreads / 32];
  const i64 at = (i64)blockIdx.x * kParseTile + (i64)threadIdx.x * kParseVec;
  unsigned char c[kParseVec];
  load16(buf, at, c);
  i32 k = 0;
#pragma unroll
  for (int j = 0; j < kParseVec; ++j) k += (at + j < B && c[j] == '\n') ? 1 : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x == 0) {
    i32 t = 0;
    for (int w = 0; w < kParseThreads / 32; ++w) t += s_red[w];
    tile_nl[blockIdx.x] = t;
  }
}

// pass 2: line l = [ls[l], le[l]); the l-th newline ends line l
__global__ void __launch_bounds__(kParseThreads) k_line_bounds(const unsigned char* __restrict__ buf, i64 B,
                                                               const i32* __restrict__ tile_nl0,
                                                               const i32* __restrict__ n_nl, i64* __restrict__ ls,
                                                               i64* __restrict__ le) {
  __shared__ i32 s_warp[33];
  const i64 at = (i64)blockIdx.x * kParseTile + (i64)threadIdx.x * kParseVec;
  unsigned char c[kParseVec];
  load16(buf, at, c);
  i32 k = 0;
#pragma unroll
  for (int j = 0; j < kParseVec; ++j) k += (at + j < B && c[j] == '\n') ? 1 : 0;
  i32 line = tile_nl0[blockIdx.x] + parse_exscan(k, s_warp);
#pragma unroll
  for (int j = 0; j < kParseVec; ++j) {
    const i64 i = at + j;
    if (i < B && c[j] == '\n') {
      const bool cr = i > 0 && buf[i - 1] == '\r';
      le[line] = cr ? i - 1 : i;   // clipped at the line start below when the line is only "\r"
      ls[line + 1] = i + 1;
      ++line;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ls[0] = 0;
    const i32 nl = *n_nl;
    if (B > 0 && buf[B - 1] != '\n') le[nl] = (buf[B - 1] == '\r') ? B - 1 : B;   // last line, no newline
  }
}

// pass 3: 1 for a vertex line, 0 for a comment line (blank then '%')
__global__ void k_line_kind(const unsigned char* __restrict__ buf, const i64* __restrict__ ls,
                            i64* __restrict__ le, i32 L, i32* __restrict__ vl) {
  const i64 l = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L) return;
  const i64 b = ls[l];
  i64 e = le[l];
  if (e < b) {   // a line of "\r" alone ends at its start
    e = b;
    le[l] = b;
  }
  i64 i = b;
  while (i < e && (buf[i] == ' ' || buf[i] == '\t')) ++i;
  vl[l] = (i < e && buf[i] == '%') ? 0 : 1;
}

// vertex index of every line (-1: comment, or after the n-th vertex line);
// the line of every read vertex
__global__ void k_line_vertex(i32 L, i32 n, const i32* __restrict__ vl, const i32* __restrict__ vfirst,
                              i32* __restrict__ lv, i32* __restrict__ vline) {
  const i64 l = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L) return;
  const i32 v = vl[l] ? vfirst[l] : -1;
  const i32 r = v >= 0 && v < n ? v : -1;
  lv[l] = r;
  if (r >= 0) vline[r] = (i32)l;
}

// The line of byte i: the newline count before it (walked per thread).
// Classifies the thread's bytes of read vertex lines: token starts, bad
// characters.  With `count` only token starts are counted (pass 4a); else
// each token's value, line and offset are written and every vertex line's
// first token is recorded (pass 4b).
template <bool kCount>
__global__ void __launch_bounds__(kParseThreads) k_tokens(const unsigned char* __restrict__ buf, i64 B,
                                                          const i32* __restrict__ tile_nl0, const i64* __restrict__ ls,
                                                          const i64* __restrict__ le, const i32* __restrict__ lv,
                                                          i32* __restrict__ tile_tok, const i32* __restrict__ tile_tok0,
                                                          i64* __restrict__ tokval, i32* __restrict__ tokline,
                                                          u32* __restrict__ tokoff, i32* __restrict__ line_tok0,
                                                          unsigned long long* __restrict__ errkey) {
  __shared__ i32 s_warp[33];
  __shared__ i32 s_red[kParseThreads / 32];
  const i64 at = (i64)blockIdx.x * kParseTile + (i64)threadIdx.x * kParseVec;
  unsigned char c[kParseVec];
  load16(buf, at, c);
  i32 k = 0;
#pragma unroll
  for (int j = 0; j < kParseVec; ++j) k += (at + j < B && c[j] == '\n') ? 1 : 0;
  i32 line = tile_nl0[blockIdx.x] + parse_exscan(k, s_warp);
  unsigned char prev = at > 0 && at - 1 < B ? buf[at - 1] : '\n';
  // token starts of this thread (pass 4a: counted; 4b: their global indices)
  i32 ntok = 0;
  i32 cur_line = -1, cur_v = -1;
  i64 cur_ls = 0, cur_le = 0;
  i32 g = 0;
  if (!kCount) {
    // the thread's first token index: the tile's plus the tokens of earlier threads
    i32 mine = 0;
    i32 ln = line;
    unsigned char pv = prev;
    for (int j = 0; j < kParseVec; ++j) {
      const i64 i = at + j;
      if (i >= B) break;
      if (ln != cur_line) {
        cur_line = ln;
        cur_v = lv[ln];
        cur_le = le[ln];
      }
      const unsigned char ch = c[j];
      if (cur_v >= 0 && i < cur_le && (ch == '-' || (pdigit(ch) && !pdigit(pv) && pv != '-'))) ++mine;
      if (ch == '\n') ++ln;
      pv = ch;
    }
    g = tile_tok0[blockIdx.x] + parse_exscan(mine, s_warp);
    cur_line = -1;
  }
  for (int j = 0; j < kParseVec; ++j) {
    const i64 i = at + j;
    if (i >= B) break;
    if (line != cur_line) {
      cur_line = line;
      cur_v = lv[line];
      cur_ls = ls[line];
      cur_le = le[line];
    }
    const unsigned char ch = c[j];
    if (!kCount && cur_v >= 0 && i == cur_ls) line_tok0[line] = g;   // the line's first token
    if (cur_v >= 0 && i < cur_le) {
      bool start = false;
      if (ch == '-') {
        start = true;
        if (!(i + 1 < cur_le && pdigit(buf[i + 1]))) atomicMin(errkey, (unsigned long long)(i * 16 + PE_BAD_TOKEN));
      } else if (pdigit(ch)) {
        start = !pdigit(prev) && prev != '-';
      } else if (ch != ' ' && ch != '\t') {
        atomicMin(errkey, (unsigned long long)(i * 16 + PE_BAD_TOKEN));
      }
      if (start) {
        if (kCount) {
          ++ntok;
        } else {
          i64 q = i;
          const bool neg = buf[q] == '-';
          if (neg) ++q;
          i64 val = 0;
          for (int d = 0; q < cur_le && pdigit(buf[q]) && d < 18; ++q, ++d) val = val * 10 + (buf[q] - '0');
          if (q < cur_le && pdigit(buf[q])) val = (i64)1 << 60;   // too long for any id or weight
          tokval[g] = neg ? -val : val;
          tokline[g] = line;
          tokoff[g] = (u32)(i - cur_ls);
          ++g;
        }
      }
    }
    if (ch == '\n') ++line;
    prev = ch;
  }
  if (kCount) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ntok += __shfl_xor_sync(0xffffffffu, ntok, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = ntok;
    __syncthreads();
    if (threadIdx.x == 0) {
      i32 t = 0;
      for (int w = 0; w < kParseThreads / 32; ++w) t += s_red[w];
      tile_tok[blockIdx.x] = t;
    }
  }
}

// pass 5: degree and vertex weight of every vertex from its line's tokens
__global__ void k_vertex_degrees(i32 n, i32 nread, const i32* __restrict__ vline, const i32* __restrict__ line_tok0,
                                 const i32* __restrict__ ntok_total, const i64* __restrict__ le,
                                 const i64* __restrict__ tokval, i32 vsize, i32 vwf, i32 ewf, i32* __restrict__ deg,
                                 i32* __restrict__ vwgt, unsigned long long* __restrict__ errkey) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  if (v >= nread) {   // missing trailing lines: isolated vertices
    deg[v] = 0;
    vwgt[v] = 1;
    return;
  }
  const i32 l = vline[v];
  const i32 t0 = line_tok0[l];
  const i32 t1 = v + 1 < nread ? line_tok0[vline[v + 1]] : *ntok_total;
  const i32 T = t1 - t0;
  const u64 endpos = (u64)le[l];
  i32 d = 0;
  if (vsize && T < 1) {
    atomicMin(errkey, endpos * 16 + PE_MISSING_VSIZE);
  } else if (vwf && T < vsize + 1) {
    atomicMin(errkey, endpos * 16 + PE_MISSING_VW);
  } else {
    const i32 rem = T - vsize - vwf;
    if (ewf && (rem & 1)) atomicMin(errkey, endpos * 16 + PE_MISSING_EW);
    d = ewf ? rem >> 1 : rem;
  }
  deg[v] = d;
  vwgt[v] = vwf && T >= vsize + 1 ? (i32)tokval[t0 + vsize] : 1;
}

// pass 6: every token of a vertex's neighbour list to its CSR slot
__global__ void k_scatter_tokens(i32 ntok, i32 n, const i32* __restrict__ tokline, const u32* __restrict__ tokoff,
                                 const i64* __restrict__ tokval, const i32* __restrict__ lv,
                                 const i32* __restrict__ line_tok0, const i64* __restrict__ ls,
                                 const i32* __restrict__ xadj, i32 hdr, i32 ewf, i32* __restrict__ adjncy,
                                 i32* __restrict__ adjwgt, unsigned long long* __restrict__ errkey) {
  for (i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x; g < ntok; g += (i64)gridDim.x * blockDim.x) {
    const i32 l = tokline[g];
    const i32 v = lv[l];
    const i32 j = (i32)g - line_tok0[l] - hdr;
    if (j < 0) continue;   // the vertex size / weight
    const i64 x = tokval[g];
    const i32 e = ewf ? (j >> 1) : j;
    if (e >= xadj[v + 1] - xadj[v]) continue;   // an unpaired id (its line reports the missing weight)
    const i64 slot = (i64)xadj[v] + e;
    if (ewf && (j & 1)) {
      adjwgt[slot] = (i32)x;
    } else {
      if (x < 1 || x > n) atomicMin(errkey, (u64)(ls[l] + tokoff[g]) * 16 + PE_RANGE);
      adjncy[slot] = (i32)(x - 1);
      if (!ewf) adjwgt[slot] = 1;
    }
  }
}

// ---------------------------------------------------------------------------
// part ids to text: digit counts, a scan, the digits
// ---------------------------------------------------------------------------
__device__ __forceinline__ i32 ndigits(u32 x) {
  i32 d = 1;
  while (x >= 10) {
    x /= 10;
    ++d;
  }
  return d;
}

__global__ void k_id_len(i32 n, const i32* __restrict__ part, i32* __restrict__ len, i32* __restrict__ bad) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const i32 p = part[v];
  if (p < 0) atomicOr(bad, 1);
  len[v] = ndigits((u32)(p < 0 ? 0 : p)) + 1;
}

__global__ void k_id_text(i32 n, const i32* __restrict__ part, const i32* __restrict__ off, char* __restrict__ out) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  u32 x = (u32)part[v];
  const i32 d = ndigits(x);
  char* p = out + off[v];
  p[d] = '\n';
  for (i32 q = d - 1; q >= 0; --q) {
    p[q] = (char)('0' + x % 10);
    x /= 10;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

struct PinnedBuf {
  char* p = nullptr;
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

const char* parse_error_text(u32 code) {
  switch (code) {
    case PE_BAD_TOKEN: return "graph file: bad token";
    case PE_MISSING_VSIZE: return "graph file: missing vertex size";
    case PE_MISSING_VW: return "graph file: missing vertex weight";
    case PE_MISSING_EW: return "graph file: missing edge weight";
    case PE_RANGE: return "graph file: neighbour id out of range";
    default: return "graph file: parse error";
  }
}

}  // namespace

void read_metis_device(Handle& h, const char* path, bool quirks, DeviceCsr& out) {
  FILE* f = fopen(path, "rb");
  if (!f) throw Error{GKW_E_INVALID, std::string("cannot open graph file: ") + path};
  fseek(f, 0, SEEK_END);
  const long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  PinnedBuf hb;
  const size_t size = sz > 0 ? (size_t)sz : 0;
  if (cudaHostAlloc((void**)&hb.p, std::max<size_t>(size, 1), cudaHostAllocDefault) != cudaSuccess) {
    fclose(f);
    cudaGetLastError();
    throw Error{GKW_E_NOMEM, "cannot allocate pinned memory for the graph file"};
  }
  const size_t got = size ? fread(hb.p, 1, size, f) : 0;
  fclose(f);
  MetisHeader hd;
  std::string err;
  if (!parse_metis_header(hb.p, got, quirks, &hd, &err)) throw Error{GKW_E_INVALID, err};
  const i64 B = (i64)got - (i64)hd.body;
  GKW_REQUIRE(B < ((i64)1 << 31) - kParseTile, GKW_E_UNSUPPORTED, "graph file body above 2 GB: read it on the host");
  const i32 n = (i32)hd.n;
  const i32 ntiles = (i32)std::max<i64>(1, (B + kParseTile - 1) / kParseTile);
  Pool::Mark mk = h.scratch.mark();
  unsigned char* buf = h.scratch.alloc_n<unsigned char>((size_t)ntiles * kParseTile + kParseTile);
  GKW_CUDA(cudaMemsetAsync(buf + std::max<i64>(B, 0), 0, (size_t)ntiles * kParseTile + kParseTile - B, h.stream));
  if (B > 0) GKW_CUDA(cudaMemcpyAsync(buf, hb.p + hd.body, (size_t)B, cudaMemcpyHostToDevice, h.stream));
  i32* tile_a = h.scratch.alloc_n<i32>(ntiles);
  i32* tile_b = h.scratch.alloc_n<i32>(ntiles);
  i32* scal = h.scratch.alloc_n<i32>(8);   // [0] newlines, [1] vertex lines, [2] tokens, [3] adjacency entries
  unsigned long long* errkey = h.scratch.alloc_n<unsigned long long>(1);
  GKW_CUDA(cudaMemsetAsync(errkey, 0xff, sizeof(unsigned long long), h.stream));
  launch(k_tile_newlines, ntiles, kParseThreads, 0, h.stream, (const unsigned char*)buf, B, tile_a);
  GKW_CHECK_LAUNCH();
  exclusive_scan_i32(h, tile_a, tile_b, ntiles, scal);
  GKW_CUDA(cudaMemcpyAsync(h.h_pinned, scal, sizeof(i32), cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  const i32 nl = (i32)(*reinterpret_cast<i32*>(h.h_pinned));
  const i32 L = nl + ((B > 0 && hb.p[got - 1] != '\n') ? 1 : 0);
  i64* ls = h.scratch.alloc_n<i64>((size_t)L + 2);
  i64* le = h.scratch.alloc_n<i64>((size_t)L + 1);
  i32* vl = h.scratch.alloc_n<i32>((size_t)L + 1);
  i32* vfirst = h.scratch.alloc_n<i32>((size_t)L + 1);
  i32* lv = h.scratch.alloc_n<i32>((size_t)L + 1);
  i32* vline = h.scratch.alloc_n<i32>((size_t)std::max(n, 1));
  i32* line_tok0 = h.scratch.alloc_n<i32>((size_t)L + 1);
  launch(k_line_bounds, ntiles, kParseThreads, 0, h.stream, (const unsigned char*)buf, B, (const i32*)tile_b,
         (const i32*)scal, ls, le);
  if (L > 0) {
    launch(k_line_kind, ceil_div(L, 256), 256, 0, h.stream, (const unsigned char*)buf, (const i64*)ls, le, L, vl);
    exclusive_scan_i32(h, vl, vfirst, L, scal + 1);
    launch(k_line_vertex, ceil_div(L, 256), 256, 0, h.stream, L, n, (const i32*)vl, (const i32*)vfirst, lv, vline);
  }
  GKW_CHECK_LAUNCH();
  // tokens
  launch(k_tokens<true>, ntiles, kParseThreads, 0, h.stream, (const unsigned char*)buf, B, (const i32*)tile_b,
         (const i64*)ls, (const i64*)le, (const i32*)lv, tile_a, (const i32*)nullptr, (i64*)nullptr, (i32*)nullptr,
         (u32*)nullptr, (i32*)nullptr, errkey);
  GKW_CHECK_LAUNCH();
  i32* tile_t0 = h.scratch.alloc_n<i32>(ntiles);
  exclusive_scan_i32(h, tile_a, tile_t0, ntiles, scal + 2);
  GKW_CUDA(cudaMemcpyAsync(h.h_pinned, scal, sizeof(i32) * 4, cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  const i32* hs = reinterpret_cast<const i32*>(h.h_pinned);
  const i32 nvl = L > 0 ? hs[1] : 0;
  const i32 ntok = hs[2];
  const i32 nread = std::min(nvl, n);
  i64* tokval = h.scratch.alloc_n<i64>((size_t)std::max(ntok, 1));
  i32* tokline = h.scratch.alloc_n<i32>((size_t)std::max(ntok, 1));
  u32* tokoff = h.scratch.alloc_n<u32>((size_t)std::max(ntok, 1));
  launch(k_tokens<false>, ntiles, kParseThreads, 0, h.stream, (const unsigned char*)buf, B, (const i32*)tile_b,
         (const i64*)ls, (const i64*)le, (const i32*)lv, (i32*)nullptr, (const i32*)tile_t0, tokval, tokline, tokoff,
         line_tok0, errkey);
  GKW_CHECK_LAUNCH();
  // degrees, xadj
  const i32 vsize = hd.vsize ? 1 : 0, vwf = hd.vw ? 1 : 0, ewf = hd.ew ? 1 : 0;
  i32* deg = h.scratch.alloc_n<i32>((size_t)n + 1);
  GKW_CUDA(cudaMemsetAsync(deg + n, 0, sizeof(i32), h.stream));   // xadj[n] = the total
  out.n = n;
  GKW_CUDA(cudaMalloc((void**)&out.xadj, sizeof(i32) * ((size_t)n + 1)));
  GKW_CUDA(cudaMalloc((void**)&out.vwgt, sizeof(i32) * std::max<size_t>(n, 1)));
  if (n > 0)
    launch(k_vertex_degrees, ceil_div(n, 256), 256, 0, h.stream, n, nread, (const i32*)vline, (const i32*)line_tok0,
           (const i32*)(scal + 2), (const i64*)le, (const i64*)tokval, vsize, vwf, ewf, deg, out.vwgt, errkey);
  GKW_CHECK_LAUNCH();
  exclusive_scan_i32(h, deg, out.xadj, (i64)n + 1, scal + 3);
  GKW_CUDA(cudaMemcpyAsync(h.h_pinned, scal + 3, sizeof(i32), cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaMemcpyAsync(h.h_pinned + 1, errkey, sizeof(u64), cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  const i32 nnz = *reinterpret_cast<const i32*>(h.h_pinned);
  u64 ek = (u64)h.h_pinned[1];
  // the scatter also runs after an error: an out-of-range id earlier in the
  // file than that error is the one to report (it stays inside each row)
  {
    out.nnz = nnz;
    GKW_CUDA(cudaMalloc((void**)&out.adjncy, sizeof(i32) * std::max<size_t>(nnz, 1)));
    GKW_CUDA(cudaMalloc((void**)&out.adjwgt, sizeof(i32) * std::max<size_t>(nnz, 1)));
    if (ntok > 0)
      launch(k_scatter_tokens, std::max<u32>(1, std::min<u32>(ceil_div(ntok, 256), (u32)h.sm_count * 16)), 256, 0,
             h.stream, ntok, n, (const i32*)tokline, (const u32*)tokoff, (const i64*)tokval, (const i32*)lv,
             (const i32*)line_tok0, (const i64*)ls, (const i32*)out.xadj, vsize + vwf, ewf, out.adjncy, out.adjwgt,
             errkey);
    GKW_CHECK_LAUNCH();
    GKW_CUDA(cudaMemcpyAsync(h.h_pinned + 1, errkey, sizeof(u64), cudaMemcpyDeviceToHost, h.stream));
    GKW_CUDA(cudaStreamSynchronize(h.stream));
    ek = (u64)h.h_pinned[1];
  }
  h.scratch.release(mk);
  if (ek != ~0ull) throw Error{GKW_E_INVALID, parse_error_text((u32)(ek & 15))};
  if (!quirks && (i64)nnz != 2 * hd.m)
    throw Error{GKW_E_INVALID, "graph file: header says " + std::to_string(hd.m) + " edges, found " +
                                   std::to_string(nnz) + " adjacency entries (expected 2m)"};
}

void write_partition_device(Handle& h, const char* path, i32 n, const i32* d_part) {
  GKW_REQUIRE(n >= 0 && (n == 0 || d_part), GKW_E_INVALID, "part is NULL");
  Pool::Mark mk = h.scratch.mark();
  i32* len = h.scratch.alloc_n<i32>((size_t)n + 1);
  i32* off = h.scratch.alloc_n<i32>((size_t)n + 1);
  i32* misc = h.scratch.alloc_n<i32>(2);   // [0] bad id, [1] bytes
  GKW_CUDA(cudaMemsetAsync(misc, 0, sizeof(i32) * 2, h.stream));
  if (n > 0) launch(k_id_len, ceil_div(n, 256), 256, 0, h.stream, n, d_part, len, misc);
  GKW_CHECK_LAUNCH();
  exclusive_scan_i32(h, len, off, n, misc + 1);
  GKW_CUDA(cudaMemcpyAsync(h.h_pinned, misc, sizeof(i32) * 2, cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  const i32 bad = reinterpret_cast<const i32*>(h.h_pinned)[0];
  const i32 bytes = reinterpret_cast<const i32*>(h.h_pinned)[1];
  GKW_REQUIRE(!bad, GKW_E_INVALID, "negative part id");
  char* text = h.scratch.alloc_n<char>((size_t)std::max(bytes, 1));
  if (n > 0) launch(k_id_text, ceil_div(n, 256), 256, 0, h.stream, n, d_part, (const i32*)off, text);
  GKW_CHECK_LAUNCH();
  PinnedBuf hb;
  GKW_CUDA(cudaHostAlloc((void**)&hb.p, std::max<size_t>(bytes, 1), cudaHostAllocDefault));
  if (bytes) GKW_CUDA(cudaMemcpyAsync(hb.p, text, (size_t)bytes, cudaMemcpyDeviceToHost, h.stream));
  GKW_CUDA(cudaStreamSynchronize(h.stream));
  h.scratch.release(mk);
  FILE* f = fopen(path, "wb");
  GKW_REQUIRE(f != nullptr, GKW_E_INVALID, std::string("cannot open ") + path);
  const size_t wr = fwrite(hb.p, 1, (size_t)bytes, f);
  fclose(f);
  GKW_REQUIRE(wr == (size_t)bytes, GKW_E_INVALID, std::string("cannot write ") + path);
}

}  // namespace gkw
