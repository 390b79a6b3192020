// Internal declarations shared by the partitioner's CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gkway.h"
#include "metis_header.h"

namespace gkw {

typedef int32_t i32;
typedef uint32_t u32;
typedef int64_t i64;
typedef uint64_t u64;

constexpr int kMaxLevels = GKW_MAX_LEVELS;
constexpr int kMatchLaneChoices = 5;   // heavy-edge match lanes per vertex: 2, 4, 8, 16, 32

// ---------------------------------------------------------------------------
// Errors: C-ABI calls return a status; the message is kept per host thread.
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
struct Error {
  gkw_status st;
  std::string msg;
};

#define GKW_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      throw ::gkw::Error{GKW_E_CUDA, std::string(#call " failed: ") + cudaGetErrorString(e_) + \
                                         " (" __FILE__ ":" + std::to_string(__LINE__) + ")"}; \
  } while (0)

#define GKW_CHECK_LAUNCH() GKW_CUDA(cudaGetLastError())

#define GKW_REQUIRE(cond, code, msg)                   \
  do {                                                 \
    if (!(cond)) throw ::gkw::Error{(code), (msg)};    \
  } while (0)

// ---------------------------------------------------------------------------
// Device memory: a chunked bump allocator.  Chunks are kept across calls; a
// mark/release pair frees everything allocated after the mark.
// ---------------------------------------------------------------------------
class Pool {
 public:
  explicit Pool(size_t min_chunk = size_t(64) << 20) : min_chunk_(min_chunk) {}
  ~Pool();
  void* alloc(size_t bytes);
  template <class T>
  T* alloc_n(size_t n) { return static_cast<T*>(alloc(n * sizeof(T))); }
  struct Mark { size_t chunk; size_t top; };
  Mark mark() const { return {cur_, chunks_.empty() ? 0 : chunks_[cur_].top}; }
  // Where the next allocations will land (current chunk's base and top): two
  // equal fingerprints hand out the same addresses for the same requests.
  std::pair<const void*, size_t> fingerprint() const {
    return chunks_.empty() ? std::pair<const void*, size_t>{nullptr, 0}
                           : std::pair<const void*, size_t>{chunks_[cur_].base, chunks_[cur_].top};
  }
  void release(Mark m);
  void reset() { release({0, 0}); }
  size_t capacity() const;
  void reserve(size_t bytes);   // make sure one chunk of at least `bytes` exists at the front
  // Free every chunk.  Only when nothing is allocated (after reset()) and no
  // queued work uses the memory; cudaFree waits for the whole device.
  void trim();
  void set_min_chunk(size_t bytes) { min_chunk_ = bytes; }
  // Largest amount handed out since the last reset_peak() (chunk tails that
  // could not be used count as handed out).
  size_t peak() const { return peak_; }
  void reset_peak() { peak_ = 0; }

 private:
  struct Chunk { char* base; size_t cap; size_t top; };
  void note_use();
  std::vector<Chunk> chunks_;
  size_t cur_ = 0;
  size_t min_chunk_;
  size_t peak_ = 0;
};

// ---------------------------------------------------------------------------
// Device-side CSR view of one level (0-based ids).
// ---------------------------------------------------------------------------
struct DevGraph {
  i32 n = 0;
  i64 m = 0;
  const i32* xadj = nullptr;
  const i32* adjncy = nullptr;
  const i32* adjwgt = nullptr;
  const i32* vwgt = nullptr;
  i64 maxdeg = -1;   // longest row, when known (-1: unknown)
};

struct Level {
  DevGraph g;
  i32* cmap = nullptr;   // to the next coarser level (n entries), null at the coarsest
};

// Per-level result of one coarsening step.
struct CoarsenOut {
  i32 nc = 0;
  i64 mc = 0;
  i32* cmap = nullptr;
  i32* cxadj = nullptr;
  i32* cadjncy = nullptr;
  i32* cadjwgt = nullptr;
  i32* cvwgt = nullptr;
  i32 uf_rounds = 0;
  i32 max_cvw = 0;   // heaviest coarse vertex
  i32 maxdeg = 0;    // longest coarse row
};

// Grid barrier word of a cooperative launch (see device_util.cuh); zero
// before the launch.
struct GridBarrier {
  u32 count;
  u32 pad;
};

// Three rotating 64-bit barrier words that also sum a count per CTA
// (grid_barrier_count, device_util.cuh); zero before a launch.
struct CountBarrier {
  unsigned long long w[3];
};

// Device-side state of one handle shared by the cooperative kernels and the
// per-level scalars read back once per level.
struct CoopState {
  GridBarrier bar;
  i32 err;        // nonzero: a cooperative kernel timed out or ran away
  i32 nc;         // coarse vertex count of the last coarsening step
  i32 mc;         // coarse CSR entries of the last coarsening step
  i32 uf_rounds;  // union-find round launches of the last coarsening step
  i32 scan_err;
  i32 arena_overflow;
  i64 arena_need;
  i32 max_cvw;    // heaviest coarse vertex of the last coarsening step
  i32 maxdeg;     // longest coarse row of the last coarsening step
};

// Bump arena for the hash tables of very long coarse rows (handle-owned,
// grown when a level reports overflow).
struct ArenaHdr {
  u64 used;
  u64 need;
  i32 overflow;
  i32 pad;
};

// Single-pass scan state (one per handle): the current scan's ticket and
// finished-tile counters and its epoch (all kept on the device, so a scan
// replayed from a CUDA graph needs no host-side argument), the error word;
// tile status words follow the header.
struct ScanState {
  u32 ticket;
  u32 done;
  u32 epoch;
  i32 err;
  u64 tiles[1];
};

// The library handle: one stream, two pools (level hierarchy and scratch),
// small pinned host staging, the device id.
struct Handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  Pool hier;
  Pool scratch;
  i64* h_pinned = nullptr;      // 64 pinned i64 slots for scalar readbacks
  i32 sm_count = 148;
  i32 smem_optin = 232448;      // opt-in shared memory per block of the device
  ScanState* scan = nullptr;    // single-pass scan state
  CoopState* coop = nullptr;    // cooperative-kernel state and per-level scalars
  ArenaHdr* arena = nullptr;    // long-row hash tables: header + words
  u64 arena_words = 0;
  i32 scan_tiles_cap = 0;
  u64 scan_epoch = 0;           // host mirror of the device scan epoch (wrap guard)
  u64 scans_enqueued = 0;
  // CUDA-graph replay of launch sequences (graph_run): captured sequences by
  // key, whether capture is on for this handle, and whether one is running
  struct GraphEntry {
    std::string key;
    int seen = 0;
    cudaGraphExec_t exec = nullptr;
    u64 launches = 0, scans = 0;
    bool wide = false;   // holds a cooperative (non-cluster) launch
  };
  std::vector<GraphEntry> graphs;
  bool graphs_on = true;
  bool capturing = false;
  bool capture_wide = false;
  // timing events of the partition driver: 5 phase marks, then a start/end
  // pair per level-kernel launch; created on first use, destroyed with the handle
  static constexpr int kTimerEvents = 5 + 2 * kMaxLevels;
  cudaEvent_t tev[kTimerEvents] = {};
  bool tev_ready = false;
  // Grid-barrier kernels: with narrow set, their grids are capped at one
  // thread-block cluster (a server's small jobs; see launch_coop)
  bool narrow = false;
  cudaEvent_t coop_ev = nullptr;   // this handle's last wide cooperative launch
  gkw_tuning tuning{{4, 8, 16, 32}, 512, 32, 0, 256};   // launch shapes (gkw_autotune)
  // while the autotuner collects: per average-degree bucket, the summed time
  // of each match lane count (4, 8, 16, 32) over the levels met
  bool tune_collect = false;
  double tune_match_ms[4][kMatchLaneChoices] = {};
  Handle() : hier(size_t(256) << 20), scratch(size_t(256) << 20) {}
};
void ensure_timer_events(Handle& h);

// ---- kernels with grid barriers (common.cu) ----
// Largest thread-block cluster the kernel can be launched as with this block
// size and dynamic shared memory (1 if none).
i32 coop_cluster_limit(Handle& h, const void* kern, i32 block, size_t smem);
// Grid size for a barrier kernel: `want`, capped at the cluster limit in
// narrow mode.
i32 coop_grid(Handle& h, const void* kern, i32 want, i32 block, size_t smem);
// Launch a kernel whose CTAs wait on one another (grid_barrier).  A grid that
// fits in one cluster is launched as that cluster: the hardware schedules all
// of its CTAs together, so it cannot wait on CTAs that never start, whatever
// else runs.  A wider grid is a cooperative launch, and the wide launches of
// all handles of the process on one device are chained (each waits for the
// previous one to finish): two wide grids running at once could each hold
// part of the SMs and wait for the rest.
void launch_coop(Handle& h, const void* kern, i32 grid, i32 block, size_t smem, void** args);
// Runs `body` (a sequence of launches, memsets and copies on h.stream, no
// host synchronisation) through the handle's graph cache: the first time a
// key is seen the body runs as is; the second time it is captured into a CUDA
// graph, which then runs in its place, that time and every later time.  The
// key must name everything the body's launches depend on (sizes, pointers,
// the scratch pool's position, launch shapes).  Returns true if a graph ran.
// Results never differ from running the body.
bool graph_run(Handle& h, const std::string& key, const std::function<void()>& body);
void graph_cache_clear(Handle& h);
// Removes launches counted during a capture (they run only with the graph).
void uncount_launches(uint64_t n);
void count_launches(uint64_t n);
void forget_coop_event(Handle& h);   // before the handle is destroyed

// ---- kernel launches ----
// Every kernel of the library is launched through launch(), which counts the
// launches (gkw_kernel_launches() reports the total).
void count_launch();
uint64_t launch_total();
template <typename... KArgs, typename... Args>
inline void launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                   Args&&... args) {
  kern<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
  count_launch();
}

// ---- device primitives (scan.cu) ----
// Exclusive scan of `in` (n entries) into `out` (n entries); if `total` is not
// null, the grand total is stored there (device pointer).  `in` may equal `out`.
void exclusive_scan_i32(Handle& h, const i32* in, i32* out, i64 n, i32* total);

// ---- coarsening (coarsen.cu) ----
// maxdeg: the longest row if known (< 0: unknown); rows above the sub-warp
// limit go to one CTA each.
void run_match(Handle& h, const DevGraph& g, i32* cand, i64 maxdeg = -1);
// Average-degree bucket of a level for gkw_tuning::match_lanes.
i32 match_bucket(const DevGraph& g);
// The autotuner's measurement of every match lane count on one level.
void time_match_variants(Handle& h, const DevGraph& g, i32* cand);
// returns the number of round launches the reference's loop would make
// These run without host synchronisation; results that the host needs are
// left in device memory (see CoopState) and read once per level.
void run_union_find(Handle& h, i32 n, const i32* cand, u64* keys_out, i32* d_rounds);
void run_group_map(Handle& h, i32 n, const u64* keys, i32 group_cap, i32* cmap, i32* d_nc);
// Contraction with the coarse vertex count on the device (d_nc) and an upper
// bound nc_ub on the host; cxadj needs nc_ub+1 entries, cadjncy/cadjwgt room
// for g.m, cvwgt nc_ub.  *d_mc receives m_c.  Returns false if the long-row
// arena overflowed (the caller grows it and runs the step again).
void run_contract(Handle& h, const DevGraph& g, const i32* cmap, const i32* d_nc, i32 nc_ub, i32 group_cap,
                  i32* cxadj, i32* cadjncy, i32* cadjwgt, i32* cvwgt, i32* d_mc);
void ensure_arena(Handle& h, u64 words);
// Reads the CoopState (one host sync) and throws on a recorded error.
CoopState read_coop(Handle& h);
void coarsen_level(Handle& h, const DevGraph& g, i32 group_cap, CoarsenOut& out);

// ---- refinement (refine.cu) ----
struct RefineCtx;   // opaque
struct RefineLevelStats {
  i32 rounds = 0;
  i64 moves = 0;
  i64 gain_sum = 0;
  i32 brounds = 0;
  i64 bmoves = 0;
  i64 rows = 0;   // adjacency entries read by the gain updates of the rounds
};
// One persistent launch over one level.  With cmap: project the state held in
// the context (the coarser level) onto this level and update the gains of its
// boundary vertices.  With lists: take the caller's state, U from `updated`,
// P from the current gains, update U.  Then balance rounds (balance) and/or
// refinement rounds (refine).
struct LevelJob {
  const i32* cmap = nullptr;
  const i32* updated = nullptr;
  bool lists = false;
  bool balance = false;
  float bcap = 0.f;
  bool refine = false;
  float maxw = 0.f;
  i32 move_cap = 1024;
  cudaEvent_t ev_start = nullptr;   // optional: recorded right before / after the launch
  cudaEvent_t ev_end = nullptr;
  const struct BatchLevel* batch = nullptr;   // a batched level (batch.cu), or null
};
// Per-level tables of a batched level: the disjoint union of G graphs with
// global part ids (graph g owns parts [gpbase[g], gpbase[g] + gk[g])).
struct BatchLevel {
  i32 G = 0;
  const i32* gid = nullptr;      // [n] graph of each vertex
  const i32* gvbase = nullptr;   // [G + 1] vertex offsets at this level
  const i32* gpbase = nullptr;   // [G]
  const i32* gk = nullptr;       // [G]
  const i32* gflags = nullptr;   // [G] bit 0 refine, bit 1 balance rounds, bit 2 coarsest level here
  const float* pmaxw = nullptr;  // [parts]
  const float* pbcap = nullptr;  // [parts]
  i32* gcc = nullptr;            // [G] zeroed
  i32* glight = nullptr;         // [G]
  i32* mcount = nullptr;         // [1] zeroed
  i32* anyf = nullptr;           // [3] zeroed
  // graphs entering at this level (gflags bit 2): cmap[v] = -(1 + i) names
  // entry i of their initial parts and boundary flags
  const i32* part_init = nullptr;
  const i32* bnd_init = nullptr;
};
// kacc: part-row length of the gain updates (largest k of a batch; 0 = k)
RefineCtx* refine_create(Handle& h, i32 n_max, i32 k, i32 move_cap, i32 kacc = 0);
RefineCtx* refine_create_ext(Handle& h, i32 n, i32 k, i32 move_cap, i32* part, i32* bnd, i32* gain,
                             i32* target);
void refine_destroy(RefineCtx* c);
i32* refine_part(RefineCtx* c);
i32* refine_boundary(RefineCtx* c);
i32* refine_gain(RefineCtx* c);
i32* refine_target(RefineCtx* c);
u32* refine_pw(RefineCtx* c);
// Coarsest level: part given; computes boundary flags and part weights.
void refine_init_coarsest(Handle& h, RefineCtx* c, const DevGraph& g, const i32* d_part_in);
// Batched levels: part weights (global part ids) and boundary flags of the
// initial parts of the coarsest union.
void refine_init_union(Handle& h, RefineCtx* c, const DevGraph& cu, const i32* part, i32* bnd_out);
void level_run(Handle& h, RefineCtx* c, const DevGraph& g, const LevelJob& j, i32 stats_slot);
// Reads the per-level statistics of slots [0, nslots) (one host sync); throws
// if a level kernel reported an error.
std::vector<RefineLevelStats> level_stats(Handle& h, RefineCtx* c, i32 nslots);
// (1 + eps) * W / k, the default-mode weight cap (no "+1").
float balance_cap(i64 total_vwgt, i32 k, double eps);

// ---- metrics (refine.cu) ----
// d_cut needs 2 slots ([0] cut, [1] nonzero if a part id was out of range);
// d_pw needs k.
void compute_cut_pw(Handle& h, const DevGraph& g, const i32* part, i32 k, i64* d_cut, i64* d_pw);
// The cut / part-weight kernel alone: d_acc[0] cut, [1] bad-part flag,
// [2..k+2) part weights; the caller zeroes d_acc first.
void launch_cut_pw(cudaStream_t stream, i32 sm_count, const DevGraph& g, const i32* part, i32 k, i64* d_acc);
void check_parts(Handle& h, i32 n, const i32* part, i32 k);

// ---- initial partition (initpart.cu) ----
// Batched initial partition: the disjoint union of graphs, global part ids;
// every vertex starts in [gpbase[g], gpbase[g] + gk[g]) of its graph, and the
// seeds name parts by part - part_base[part] as a lone run would.
struct GggpBatch {
  const i32* gid = nullptr;
  const i32* gpbase = nullptr;
  const i32* gk = nullptr;
  const i32* part_base = nullptr;   // [parts] first part of the part's graph
  const i32* part_v0 = nullptr;     // [parts] vertex range of the part's graph
  const i32* part_v1 = nullptr;
  i32 depth = 0;                    // recursion depth of the largest k
};
void device_init_partition(Handle& h, const DevGraph& g, i32 k, double eps, u64 seed, i32 trials,
                           i32* d_part, const GggpBatch* batch = nullptr);

// ---- driver (partitioner.cu) ----
// total vertex weight (and the longest row in *maxdeg); throws on malformed input
i64 validate(Handle& h, const DevGraph& g, i64* maxdeg = nullptr);
void partition_impl(Handle& h, const DevGraph& g0, i32 k, const gkw_options& opt, i32* d_part_out,
                    i64* cut_out, gkw_stats* stats);
// The same from host arrays (a slice of a concatenated CSR: xadj values offset
// by xadj[0], neighbour ids by vbase); part_out is host memory.
void partition_host(Handle& h, const DevGraph& host_graph, i64 vbase, i32 k, const gkw_options& opt,
                    i32* part_out, i64* cut_out, gkw_stats* stats);
// One graph for several k over one hierarchy (each k's result as alone).
void partition_multi_impl(Handle& h, const DevGraph& g0, i32 nk, const i32* ks, const gkw_options& opt,
                          i32* d_parts, i64* cuts_out);
void partition_multi_host(Handle& h, const DevGraph& host_graph, i32 nk, const i32* ks, const gkw_options& opt,
                          i32* parts_out, i64* cuts_out);
Handle& handle_of(gkw_handle* h);   // the handle behind a C-ABI handle (capi.cu)
// gkw_autotune: the fastest launch shapes for this graph into h.tuning.
void autotune(Handle& h, const DevGraph& g, i32 k, const gkw_options& opt);
// Many independent graphs partitioned as one disjoint union (batch.cu): host
// arrays with global ids, graph g = vertices [graph_ptr[g], graph_ptr[g+1]).
// part_out gets each graph's own part ids.  Returns false, having computed
// nothing, if an edge joins two graphs.
// levels_out (optional): levels each graph kept, its input included.
bool partition_batch_union(Handle& h, const DevGraph& host_union, i32 G, const i32* graph_ptr, const i32* ks,
                           const gkw_options& opt, i32* part_out, i64* cuts_out, i32* levels_out = nullptr);
const char* last_error_cstr();

// ---- METIS .graph files on the device (parse.cu; header: metis_header.h) ----
// A graph in device memory allocated with cudaMalloc (gkw_free_device_graph).
struct DeviceCsr {
  i32 n = 0;
  i64 nnz = 0;
  i32* xadj = nullptr;
  i32* adjncy = nullptr;
  i32* adjwgt = nullptr;
  i32* vwgt = nullptr;
};
// Parse a METIS .graph file on the device (the same result and errors as the
// host reader); on error nothing stays allocated in `out` beyond what the
// caller frees with its arrays.
void read_metis_device(Handle& h, const char* path, bool reference_quirks, DeviceCsr& out);
// One part id per line, formatted on the device.
void write_partition_device(Handle& h, const char* path, i32 n, const i32* d_part);

// ---- host helpers ----
float max_part_weight(i64 total_vwgt, i32 k, double eps);
inline u32 ceil_div(u64 a, u64 b) { return (u32)((a + b - 1) / b); }

}  // namespace gkw
