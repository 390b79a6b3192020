/*
 * gkway.h -- C ABI of the B200 multilevel k-way graph partitioner.
 *
 * Drop-in for the G-kway (wanluanlee/DAC_g-kway) partitioning path.  The
 * reference has no library target: its stages are C++ functions over raw
 * device pointers, included as headers.  Each entry point below names the
 * reference function it replaces (file:line in the reference tree).
 *
 * Conventions
 *   - Graphs are CSR with int32 arrays and 0-based neighbour ids (the
 *     reference keeps 1-based ids on the device; gk::Graph converts).
 *     xadj[n+1], adjncy[nnz], adjwgt[nnz], vwgt[n]; nnz = xadj[n] = 2|E|.
 *     The graph must be symmetric, without self loops; weights >= 0.
 *   - "host" entry points take host pointers and copy; "_device" and the
 *     per-phase entry points take device pointers on the handle's device and
 *     run on the handle's stream; they return after that stream is idle.
 *   - Every call returns a gkw_status; gkw_last_error() gives the message of
 *     the last failure on the calling thread.  No C++ exception crosses the ABI.
 *   - A handle is not re-entrant: one host thread per handle at a time.
 */
#ifndef GKWAY_H_
#define GKWAY_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GKW_MAX_LEVELS 64

typedef enum gkw_status {
  GKW_OK = 0,
  GKW_E_INVALID = 1,      /* bad argument or malformed graph */
  GKW_E_CUDA = 2,         /* CUDA runtime error */
  GKW_E_NOMEM = 3,        /* device allocation failed */
  GKW_E_UNSUPPORTED = 4,  /* input outside the supported range (e.g. k too large) */
  GKW_E_INIT = 5,         /* the initial-partition callback failed */
  GKW_E_INTERNAL = 6,
  GKW_E_PENDING = 7       /* served request not finished yet (gkw_server_poll) */
} gkw_status;

typedef struct gkw_handle gkw_handle;

typedef struct gkw_csr {
  int32_t n;
  int64_t nnz;
  const int32_t* xadj;
  const int32_t* adjncy;
  const int32_t* adjwgt; /* may be NULL: unit edge weights (host calls only) */
  const int32_t* vwgt;   /* may be NULL: unit vertex weights (host calls only) */
} gkw_csr;

/* Initial partition of the coarsest graph.  Host arrays, 0-based; fill
 * part_out[n] with values in [0,k) and return 0.  The reference calls host
 * METIS here (gkway/metis_partition.hpp:4-99); a caller that wants the
 * reference's exact behaviour passes a callback that calls METIS. */
typedef int32_t (*gkw_init_fn)(void* user, int32_t n, const int32_t* xadj, const int32_t* adjncy,
                               const int32_t* adjwgt, const int32_t* vwgt, int32_t k,
                               int32_t* part_out);

enum { GKW_INIT_DEVICE = 0, GKW_INIT_CALLBACK = 1 };

typedef struct gkw_options {
  double eps;               /* imbalance, 0.03 (declarations.h:17) */
  int32_t group_cap;        /* max fine vertices per coarse vertex, 6 (graph_partitioner.hpp:229) */
  int32_t threshold_factor; /* coarsen while n > threshold_factor*k, 20 (graph_partitioner.hpp:22) */
  int32_t move_cap;         /* moves applied per refinement round, 1024 (uncoarsen.hpp:475) */
  int32_t init_method;      /* GKW_INIT_DEVICE (default) or GKW_INIT_CALLBACK */
  gkw_init_fn init_fn;
  void* init_user;
  uint64_t seed;            /* seed of the device initial partitioner */
  int32_t init_trials;      /* independent device initial-partition trials (best cut kept) */
  int32_t enforce_balance;  /* 1 (default): every part <= (1+eps)W/k, balance rounds at each
                               level; 0: the reference's behaviour (MAX_PARTITION_WGT =
                               (1+eps)W/k + 1 checked on move destinations only) */
  int32_t balance_skip_levels; /* default mode: the coarsest levels refined without balance rounds
                                 (1; 0: every level balanced); the finest level always is */
  int32_t reserved1;
  double coarse_vertex_frac; /* default mode: coarsening stops before a level whose heaviest vertex
                               outweighs this fraction of W/k (0.5; <= 0: no such stop) */
  int32_t reserved[2];
} gkw_options;

typedef struct gkw_stats {
  int32_t n_levels;                     /* levels kept, the input graph included */
  int64_t level_n[GKW_MAX_LEVELS];
  int64_t level_m[GKW_MAX_LEVELS];      /* directed CSR entries */
  int32_t uf_rounds[GKW_MAX_LEVELS];    /* union-find round launches, per coarsening step */
  int32_t refine_rounds[GKW_MAX_LEVELS];
  int64_t refine_moves[GKW_MAX_LEVELS];
  int32_t balance_rounds[GKW_MAX_LEVELS];   /* per level, the coarsest included */
  int64_t balance_moves[GKW_MAX_LEVELS];
  int64_t init_cut;
  int64_t cut;                          /* exact weighted edge cut of the output */
  int64_t max_part_weight;
  float maxw;                           /* MAX_PARTITION_WGT (graph_partitioner.hpp:230) */
  double ms_coarsen, ms_init, ms_refine, ms_total;   /* device time per phase */
  /* Per level: device time of its level-kernel launch (projection, balance
   * and refinement rounds; the coarsest level's is its balance pass, -1 when
   * it has none), and the adjacency entries read by the gain updates of its
   * rounds (the first full gain pass of the level not included). */
  double ms_level[GKW_MAX_LEVELS];
  int64_t round_entries[GKW_MAX_LEVELS];
} gkw_stats;

/* ---- handle ---------------------------------------------------------- */
gkw_status gkw_create(gkw_handle** out, int32_t device);
gkw_status gkw_destroy(gkw_handle* h);
/* Use the caller's CUDA stream (a cudaStream_t) instead of the handle's own. */
gkw_status gkw_set_stream(gkw_handle* h, void* stream);

/* Launch shapes of a handle's kernels (results never depend on them).  No
 * counterpart in the reference, whose shapes are fixed constants
 * (declarations.h:12-18).
 *   match_lanes[b]       lanes per vertex of the heavy-edge match on levels
 *                        whose average degree is <= 6.5, <= 14, <= 28, above
 *                        (b = 0..3; 2, 4, 8, 16 or 32; rows above 512 entries
 *                        always go to one CTA each)
 *   level_verts_per_cta  level-kernel CTAs: one per this many vertices ...
 *   level_min_ctas       ... and at least this many (capped at 2 per SM)
 *   coarsen_fused_max_n  coarsening levels of at most this many vertices run
 *                        as one fused launch with grid barriers between the
 *                        phases (default 0: every level as per-phase kernels)
 *   coarsen_verts_per_cta  fused coarsening CTAs: one per this many vertices
 *                        (capped at the co-resident CTAs; default 256) */
typedef struct gkw_tuning {
  int32_t match_lanes[4];
  int32_t level_verts_per_cta;
  int32_t level_min_ctas;
  int32_t coarsen_fused_max_n;
  int32_t coarsen_verts_per_cta;
} gkw_tuning;
gkw_status gkw_get_tuning(gkw_handle* h, gkw_tuning* out);
gkw_status gkw_set_tuning(gkw_handle* h, const gkw_tuning* t);
/* Autotuner: partitions the device-resident graph with candidate shapes --
 * every match lane count on every level of its hierarchy, a grid of level-
 * kernel densities -- timing each with CUDA events, and keeps the fastest in
 * the handle (also returned in *out, may be NULL).  Takes a few dozen
 * partitions of the graph; later partitions on the handle use the result. */
gkw_status gkw_autotune(gkw_handle* h, const gkw_csr* d_graph, int32_t k, const gkw_options* opt, gkw_tuning* out);
void* gkw_get_stream(gkw_handle* h);
const char* gkw_last_error(void);
void gkw_default_options(gkw_options* opt);
const char* gkw_version(void);
/* Kernels this library has launched in the process so far (all handles).
 * Diagnostic, no counterpart in the reference. */
uint64_t gkw_kernel_launches(void);

/* ---- whole partitioner ------------------------------------------------
 * Replaces graph_partitioner() (gkway/graph_partitioner.hpp:222-365):
 * coarsening (:14-123), init_partition (:125-131), uncoarsening (:133-220).
 * part_out receives n part ids in [0,k). cut_out and stats may be NULL. */
gkw_status gkw_partition(gkw_handle* h, const gkw_csr* graph, int32_t k, const gkw_options* opt,
                         int32_t* part_out, int64_t* cut_out, gkw_stats* stats);
/* Same with device-resident input and output (d_part_out on the device). */
gkw_status gkw_partition_device(gkw_handle* h, const gkw_csr* d_graph, int32_t k,
                                const gkw_options* opt, int32_t* d_part_out, int64_t* cut_out,
                                gkw_stats* stats);
/* One host graph partitioned for n_k values of k, coarsened once.  The levels
 * do not depend on k except where the coarsening stops (threshold 20k,
 * gkway/graph_partitioner.hpp:22; the discard rule, :93-96), so every k runs
 * on a prefix of one hierarchy.  No counterpart in the reference, where each
 * run coarsens again.  parts_out holds n_k rows of n part ids; row q and
 * cuts_out[q] equal gkw_partition's result for ks[q]. */
gkw_status gkw_partition_multi_k(gkw_handle* h, const gkw_csr* graph, int32_t n_k, const int32_t* ks,
                                 const gkw_options* opt, int32_t* parts_out, int64_t* cuts_out);

/* ---- per-phase entry points (device pointers) --------------------------
 * Heavy-edge candidate per vertex.  Replaces gk::matching_with_score
 * (gkway/coarsen.hpp:39-78).  d_cand[n] (0-based; a vertex with no positive
 * edge weight is its own candidate). */
gkw_status gkw_match(gkw_handle* h, const gkw_csr* d_graph, int32_t* d_cand);

/* Union-find over the edges {v, cand(v)} in the deterministic (Jacobi)
 * schedule.  Replaces the HEC_union_find loop (gkway/coarsen.hpp:80-118,
 * 461-469).  d_root[v] = max id of v's component, d_dist[v] = hop distance
 * from that root.  rounds_out: round launches of the loop (may be NULL). */
gkw_status gkw_union_find(gkw_handle* h, int32_t n, const int32_t* d_cand, int32_t* d_root,
                          int32_t* d_dist, int32_t* rounds_out);

/* Coarse ids: order (root, dist, id), groups cut into chunks of group_cap.
 * Replaces constraint_group_size + count_num_coarsen_vertex + construct_cmap
 * (gkway/coarsen.hpp:408-421, 120-155, 474-481). */
gkw_status gkw_group_map(gkw_handle* h, int32_t n, const int32_t* d_root, const int32_t* d_dist,
                         int32_t group_cap, int32_t* d_cmap, int32_t* nc_out);

/* Contraction: coarse CSR with sorted rows, self loops removed, parallel
 * edges merged with summed weights; coarse vertex weights.  Replaces
 * gk::contraction + cal_coarsen_vwgt (gkway/coarsen.hpp:302-349, 157-171).
 * d_cxadj[nc+1]; d_cadjncy/d_cadjwgt need room for d_graph->nnz entries;
 * d_cvwgt[nc]. */
gkw_status gkw_contract(gkw_handle* h, const gkw_csr* d_graph, const int32_t* d_cmap, int32_t nc,
                        int32_t* d_cxadj, int32_t* d_cadjncy, int32_t* d_cadjwgt, int32_t* d_cvwgt,
                        int64_t* mc_out);

/* Gains and targets of the flagged vertices (d_updated[v] != 0).  Replaces
 * gk::update_vertex_info (gkway/uncoarsen.hpp:175-237), including its unsigned
 * comparison of gains.  d_boundary, d_gain, d_target are in-out. */
gkw_status gkw_update_vertex_info(gkw_handle* h, const gkw_csr* d_graph, int32_t k,
                                  const int32_t* d_part, const int32_t* d_updated,
                                  int32_t* d_boundary, int32_t* d_gain, int32_t* d_target);

/* One level of independent-set refinement, in place, until no move is left.
 * Replaces gk::refinement (gkway/uncoarsen.hpp:427-506).  If initial_update,
 * the flagged vertices are first passed through update_vertex_info (as
 * gk::uncoarsen does, gkway/uncoarsen.hpp:385-386).  d_pw[k] holds the part
 * weights (in-out).  rounds_out/moves_out may be NULL. */
gkw_status gkw_refine(gkw_handle* h, const gkw_csr* d_graph, int32_t k, float maxw,
                      int32_t move_cap, int32_t* d_part, int32_t* d_boundary, int32_t* d_gain,
                      int32_t* d_target, const int32_t* d_updated, int32_t* d_pw,
                      int32_t initial_update, int32_t* rounds_out, int64_t* moves_out);

/* Balance rounds on one level, in place: moves boundary vertices out of parts
 * heavier than cap (float compare) until none is, or no move is possible.  No
 * counterpart in the reference, which only reports an overweight part
 * (gkway/cuda_check.hpp:105-113); gkw_partition runs it at every level when
 * enforce_balance is set.  d_boundary must be exact for d_part; d_gain and
 * d_target are refreshed for the vertices it touches.  d_pw[k] in-out. */
gkw_status gkw_balance(gkw_handle* h, const gkw_csr* d_graph, int32_t k, float cap, int32_t move_cap,
                       int32_t* d_part, int32_t* d_boundary, int32_t* d_gain, int32_t* d_target,
                       int32_t* d_pw, int32_t* rounds_out, int64_t* moves_out);
/* The default-mode cap (1+eps)W/k. */
float gkw_balance_cap(int64_t total_vwgt, int32_t k, double eps);

/* Device initial partition of a (coarsest) graph: recursive bisection by greedy
 * graph growing.  Replaces the host METIS call of metis_init_partition
 * (gkway/metis_partition.hpp:46-47). */
gkw_status gkw_init_partition(gkw_handle* h, const gkw_csr* d_graph, int32_t k, double eps,
                              uint64_t seed, int32_t trials, int32_t* d_part);

/* Exact weighted edge cut and part weights.  Replaces gk::calculate_cutsize
 * and calculate_partition_wgt (gkway/uncoarsen.hpp:398-424,
 * gkway/cuda_check.hpp:61-73).  pw_out: host array of k entries (may be NULL). */
gkw_status gkw_cut(gkw_handle* h, const gkw_csr* d_graph, const int32_t* d_part, int32_t k,
                   int64_t* cut_out, int64_t* pw_out);

/* Read a METIS .graph file (standard format: "n m [fmt [ncon]]", '%'
 * comments, ncon 1).  reference_quirks != 0 reads a format field of "11" as
 * neighbour/weight pairs without vertex weights, as the reference parser does
 * (gkway/graph.hpp:70-152).  The four arrays are allocated with malloc and
 * released with gkw_free; ids are 0-based.  No device is touched. */
gkw_status gkw_read_metis(const char* path, int32_t reference_quirks, int32_t* n_out, int64_t* nnz_out,
                          int32_t** xadj, int32_t** adjncy, int32_t** adjwgt, int32_t** vwgt);
/* Write one part id per line to `path` (gkway/graph.hpp:227-240 writes
 * <cwd>/<name>.out this way). */
gkw_status gkw_write_partition(const char* path, int32_t n, const int32_t* part);
void gkw_free(void* p);

/* Read a METIS .graph file into device memory, parsing it on the device: the
 * file's bytes are copied to the GPU once and split into lines, tokens and
 * CSR rows there (the header line is read on the host).  Same format, result
 * and error messages as gkw_read_metis.  On success the four arrays of
 * *d_graph (0-based ids, n and nnz set) are device memory on the handle's
 * device allocated with cudaMalloc; release them with gkw_free_device_graph.
 * Replaces the reference's host parser (gkway/graph.hpp:70-152) for callers
 * that partition on the device. */
gkw_status gkw_read_metis_device(gkw_handle* h, const char* path, int32_t reference_quirks, gkw_csr* d_graph);
void gkw_free_device_graph(gkw_csr* d_graph);
/* Write one part id per line to `path`, the text formatted on the device from
 * the device array d_part (n ids); the reference writes <cwd>/<name>.out this
 * way on the host (gkway/graph.hpp:227-240). */
gkw_status gkw_write_partition_device(gkw_handle* h, const char* path, int32_t n, const int32_t* d_part);

/* Exact cut and part weights like gkw_cut, but with no device allocation and
 * no handle.  No counterpart in the reference.  For callers that may not
 * allocate device memory while they run (a serving loop with a fixed memory
 * budget, a plugin that only receives pre-allocated buffers): the kernel's
 * accumulators live in a fixed array inside the library (8192 int64 words,
 * 64 KB, held on every device that loads the library until exit), so k is
 * limited to 8190.  Runs on `stream` (a cudaStream_t, NULL = the default
 * stream) of the current device and returns when that stream is idle; cut_out
 * and pw_out (k entries, may be NULL) are host memory.  The first call on a
 * device looks up the array's device address; make it outside stream capture.
 * That address is kept for the life of the process: it does not survive a
 * cudaDeviceReset of the device.  All calls share the array: calls whose work
 * overlaps on the GPU race. */
gkw_status gkw_cut_noalloc(const gkw_csr* d_graph, const int32_t* d_part, int32_t k, void* stream,
                           int64_t* cut_out, int64_t* pw_out);

/* MAX_PARTITION_WGT as the reference computes it (graph_partitioner.hpp:230). */
float gkw_max_part_weight(int64_t total_vwgt, int32_t k, double eps);

/* ---- batched and served forms -----------------------------------------
 * No counterpart in the reference, whose driver partitions one graph per
 * process run (main/main.cu:5-20).  A server owns `slots` partition slots on
 * one device (each a handle with its own stream and device memory) and a
 * queue of jobs; slots take jobs as they and the device-memory budget free
 * up, so jobs of different sizes overlap on the GPU.  Every job runs the same
 * pipeline as gkw_partition: a graph's result is the same alone, in a batch
 * and among served requests.  Input graphs are host memory. */
typedef struct gkw_server gkw_server;

typedef struct gkw_server_config {
  int32_t slots;             /* concurrent partitions (default 2) */
  int32_t narrow_max_n;      /* jobs up to this many vertices run their barrier kernels as
                                one thread-block cluster each, so any number of them can
                                share the device; larger jobs take turns for their wide
                                grids (default 262144) */
  int64_t pool_bytes;        /* device-memory budget of all slots together (default 64 GiB,
                                capped at 90% of the free memory at creation) */
  int64_t slot_keep_bytes;   /* memory a slot keeps between jobs (default 4 GiB) */
  int32_t max_bypass;        /* times the oldest waiting job may be overtaken by smaller
                                jobs that fit when it does not (default 4 x slots) */
  int32_t batch_union;       /* 1 (default): graphs that share the options run as one disjoint
                                union -- a whole gkw_partition_batch call, and queued served
                                requests of up to batch_graph_max_n vertices drained together;
                                0: one job per graph on the slots */
  int32_t batch_max_n;       /* served requests drained into one union: at most this many
                                vertices together (default 4194304) */
  int32_t batch_graph_max_n; /* served requests of up to this many vertices join unions
                                (default 262144) */
  int32_t reserved[4];
} gkw_server_config;

void gkw_server_default_config(gkw_server_config* cfg);
gkw_status gkw_server_create(gkw_server** out, int32_t device, const gkw_server_config* cfg);
/* Waits for the running jobs, drops the queued ones, frees everything. */
gkw_status gkw_server_destroy(gkw_server* s);

/* Device memory one partition of a graph of n vertices and nnz CSR entries
 * is predicted to need (input, level hierarchy, refinement state, scratch):
 * the admission measure of the server. */
int64_t gkw_predict_footprint(int32_t n, int64_t nnz, int32_t k);

/* Served form.  submit copies the graph (the caller may free it on return) and
 * queues it; `ticket_out` names the request.  poll waits up to wait_ms
 * (0: no wait, <0: until done) and returns GKW_E_PENDING if the request is
 * still queued or running, else its status; on GKW_OK it copies the n part
 * ids to part_out (may be NULL) and the cut to cut_out (may be NULL).  A
 * finished request is forgotten after the poll that reports it. */
typedef struct gkw_request_info {
  double queue_ms;           /* submit -> start on a slot */
  double run_ms;             /* start -> result on the host */
  double latency_ms;         /* submit -> result on the host */
  int64_t predicted_bytes;
  int32_t slot;
  int32_t n_levels;
  int32_t batch_graphs;      /* graphs partitioned together with this one as one union (1: alone) */
  int32_t reserved;
} gkw_request_info;

gkw_status gkw_server_submit(gkw_server* s, const gkw_csr* graph, int32_t k, const gkw_options* opt,
                             int64_t* ticket_out);
gkw_status gkw_server_poll(gkw_server* s, int64_t ticket, int32_t wait_ms, int32_t* part_out,
                           int64_t* cut_out, gkw_request_info* info);

typedef struct gkw_server_stats {
  int64_t submitted, completed, failed;
  double p50_ms, p99_ms, max_ms;   /* latency (submit -> result) of the completed requests */
  double mean_queue_ms;
  double graphs_per_s;             /* completed / (last completion - first submit) */
  int64_t peak_reserved_bytes;     /* largest sum of predicted footprints admitted at once */
  int32_t peak_running;            /* most jobs running at once */
  int32_t slots;
} gkw_server_stats;
/* Statistics since creation or the last reset (reset != 0 clears them after reading). */
gkw_status gkw_server_stats_get(gkw_server* s, gkw_server_stats* out, int32_t reset);

/* Batched form: many independent graphs in one call, as one concatenated CSR.
 * `graph` is their disjoint union with global 0-based ids (graph g owns the
 * vertices [graph_ptr[g], graph_ptr[g+1]); no edge joins two graphs).
 * part_out[v] receives v's part id within its own graph, in [0, k[g]).
 * Graphs are scheduled largest first.  Returns GKW_OK if every graph was
 * partitioned, else the status of the first graph that failed (its index in
 * the message); status_out (may be NULL) gets each graph's status. */
typedef struct gkw_csr_batch {
  gkw_csr graph;             /* host memory; adjwgt / vwgt may be NULL */
  int32_t n_graphs;
  const int32_t* graph_ptr;  /* [n_graphs + 1] */
  const int32_t* k;          /* [n_graphs] */
  const double* eps;         /* [n_graphs], or NULL for opt->eps */
} gkw_csr_batch;

gkw_status gkw_partition_batch(gkw_server* s, const gkw_csr_batch* batch, const gkw_options* opt,
                               int32_t* part_out, int64_t* cut_out, int32_t* status_out);

#ifdef __cplusplus
}
#endif
#endif /* GKWAY_H_ */
