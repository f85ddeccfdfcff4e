/*
 * cpg.h -- C ABI of the B200-native critical path generator (libcpg_b200.so).
 *
 * The library reports the K lowest-cost source-to-sink paths of a timing DAG,
 * the operation of the reference gpu-cpg library's C++ class gpucpg::CpGen
 * (gpucpg/gpucpg.cuh:119-431).  The reference has no C ABI; each entry point
 * below names the CpGen member (or the part of report_paths) it replaces.
 * The header-only C++ shim include/gpucpg/cpgen.hpp rebuilds the CpGen surface
 * on top of these calls.
 *
 * Conventions: every call returns a cpg_status; nothing exits or throws across
 * the ABI; buffers passed in are copied (the caller keeps ownership); output
 * buffers belong to the caller.  One handle must not be used from two threads
 * at once; separate handles are independent.
 */
#ifndef CPG_B200_H
#define CPG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CPG_ABI_VERSION 3

/* Replaces exit(1) in cudaCheckErrors / checkError_t (gpucpg.cu:87-98,
 * 269-275) and the std::runtime_error throws of read_input (gpucpg.cu:457). */
typedef enum {
  CPG_OK = 0,
  CPG_ERR_INVALID = 1,   /* bad argument or graph */
  CPG_ERR_IO = 2,        /* file could not be read or parsed */
  CPG_ERR_OOM = 3,       /* device or host allocation failed */
  CPG_ERR_CAPACITY = 4,  /* a bounded buffer or the HBM budget was exceeded */
  CPG_ERR_TIMEOUT = 5,   /* a bounded device-side wait ran out */
  CPG_ERR_CUDA = 6,      /* CUDA runtime error */
  CPG_ERR_STATE = 7,     /* call out of order (e.g. no graph loaded) */
  CPG_ERR_NO_DEVICE = 8  /* no CUDA device / extension not usable */
} cpg_status;

/* Division used in the child-cost expression dist/10000.  The reference's
 * device code is compiled with --use_fast_math (CMakeLists.txt:38); REFERENCE
 * evaluates the same source expression under the same flag so the costs match
 * the reference's G-PathGen bit for bit.  IEEE uses round-to-nearest division,
 * matching the reference's host-side (SEQUENTIAL) arithmetic. */
typedef enum { CPG_DIV_REFERENCE = 0, CPG_DIV_IEEE = 1 } cpg_division;

/* Kahn step of the levelisation: CSR push with warp-aggregated enqueue, or the
 * BVSS bit-packed pull (binary AND-popc tensor-core tiles where dense enough,
 * scalar popc elsewhere).  AUTO picks by the measured frontier density. */
typedef enum {
  CPG_FRONTIER_AUTO = 0,
  CPG_FRONTIER_CSR = 1,
  CPG_FRONTIER_BVSS = 2
} cpg_frontier;

/* Which BVSS tiles go to the tensor cores (b1 AND-popc MMA).  DENSITY: a tile
 * whose frontier byte has at least min_bits bits and whose VSS holds more than
 * min_slices slices; the rest use scalar popc.  Both give identical counts. */
typedef enum {
  CPG_BVSS_TILES_DENSITY = 0,
  CPG_BVSS_TILES_TENSOR = 1,
  CPG_BVSS_TILES_SCALAR = 2
} cpg_bvss_tiles;

/* Root seeding.  REFERENCE reproduces G-PathGen's initial split
 * (gpucpg.cu:19136-19179): with R reachable sources, the split is the cost at
 * sorted index (size_t)(0.005f*R) and only the first (int)(0.005f*R+1) roots
 * at or below it (in source-id order) are kept, so on graphs with many tied
 * cheap sources some paths are never reported, exactly as in the reference.
 * ALL seeds every reachable source: the exact K cheapest paths.  The two
 * agree whenever the graph has a single source (e.g. a super-source). */
typedef enum { CPG_ROOTS_REFERENCE = 0, CPG_ROOTS_ALL = 1 } cpg_root_seeding;

typedef struct {
  int32_t device;           /* CUDA device ordinal */
  void* stream;             /* cudaStream_t to run on; NULL = handle-owned */
  int32_t division;         /* cpg_division */
  int32_t frontier;         /* cpg_frontier */
  int64_t hbm_budget_bytes; /* cap on per-query device memory; 0 = none */
  uint32_t spin_limit;      /* grid-barrier poll limit; 0 = default */
  int32_t root_seeding;     /* cpg_root_seeding */
  int32_t host_stepped;     /* 1: step the split raises from the host (one
                               kernel sequence per raise) instead of the
                               persistent device engine; for A/B checks */
  int32_t bvss_tiles;       /* cpg_bvss_tiles for the BVSS frontier */
  int32_t bvss_min_bits;    /* density test: frontier bits in the tile's byte
                               (0 = default 2) */
  int32_t bvss_min_slices;  /* density test: slices in the VSS (0 = default 32) */
  int32_t sfxt_level_sync;  /* 1: full suffix-tree builds step level by level
                               with a grid barrier per level instead of the
                               dataflow work queue; for A/B checks */
  int32_t sfxt_heap_warps;  /* dataflow build: warps per CTA (of 32) that only
                               insert chain heaps; 0 = the building warp does */
  int32_t sfxt_late_push;   /* dataflow build: 1 = a vertex's tails are
                               decremented after it is built instead of when
                               it is taken (A/B checks) */
  int32_t batch_caller_order; /* batched and served forms: 1 = keep the
                               callers' vertex order instead of renumbering
                               each graph in level order (A/B checks) */
  int32_t sfxt_heap_mode;   /* dataflow build: where chain heaps are inserted.
                               0 = chosen by size (a heap phase after every
                               build on large graphs, else by the building
                               warp right after each build), 1 = always by the
                               building warp, 2 = always in the heap phase */
  int32_t engine_ctas;      /* single queries: CTAs of the engine launch
                               (0 = chosen from k) */
  int32_t sfxt_claim_sets;  /* dataflow build: how warps take work-queue
                               slots.  0 = default (claimed, 8 sets), -1 =
                               static (warp w takes slots w, w + W, ...; A/B
                               checks), 1..16 = a free warp claims the next
                               slot of its set, the slots dealt round-robin
                               over that many sets */
} cpg_options;

typedef struct cpg_handle cpg_handle;
typedef struct cpg_dag cpg_dag;  /* a generated graph (see cpg_dag_generate) */

/* PfxtNode (gpucpg.cuh:74-107), same field order and 24-byte layout.
 * parent indexes the list returned by cpg_get_paths (-1 for a root, or when
 * the parent is not in the list); num_children is 0 as in G-PathGen. */
typedef struct {
  int32_t level;
  int32_t from;
  int32_t to;
  int32_t parent;
  int32_t num_children;
  float slack;
} cpg_path_node;

typedef struct {
  double sfxt_ms;          /* device time of the last SFXT build */
  double pfxt_ms;          /* device time of the last enumeration */
  double select_ms;        /* device time of the final select + sort + emit */
  int64_t paths_accepted;  /* paths materialised by the closure */
  int64_t items_generated; /* path-graph items written (accepted + pending) */
  int64_t pending_peak;    /* largest pending pile */
  int64_t bytes_reserved;  /* device bytes held for the last query */
  int32_t phases;          /* split raises */
  int32_t rounds;          /* closure rounds */
  int32_t levels;          /* SFXT levels */
  int32_t kernel_launches; /* kernels launched by the last levelize+report */
  float split;             /* final split (cost threshold) */
  int32_t frontier_used;   /* cpg_frontier actually used by the levelisation */
  int32_t retries;         /* query restarts after a bounded buffer overflowed */
  /* device time of the query engine by stage (ms): seed, decide, select,
   * promote, closure, output select, output sort, emit */
  float engine_stage_ms[8];
  int64_t bvss_tiles_tensor; /* BVSS tiles counted on the tensor cores */
  int64_t bvss_tiles_scalar; /* ... and with scalar popc */
  double bvss_bits_per_slice; /* measured density of the fan-out BVSS */
  double sfxt_kernel_ms;   /* the suffix-tree kernel alone (sfxt_ms adds the
                              counter reset and the deviation-row sorts) */
} cpg_stats;

/* ------------------------------------------------------------ lifecycle */
void cpg_options_init(cpg_options* opts);
/* CpGen::CpGen (gpucpg.cu:7400-7404). */
cpg_status cpg_create(cpg_handle** out, const cpg_options* opts);
/* CpGen::~CpGen. */
cpg_status cpg_destroy(cpg_handle* h);
const char* cpg_last_error(const cpg_handle* h);
const char* cpg_status_string(cpg_status s);
int32_t cpg_abi_version(void);

/* ------------------------------------------------------------ ingestion */
/* CpGen::read_input(filename, ignore_wgts) (gpucpg.cu:453-548). */
cpg_status cpg_load_text(cpg_handle* h, const char* path, int32_t ignore_wgts);
/* Same graph from an edge list in file order (no text round trip). */
cpg_status cpg_load_edges(cpg_handle* h, int32_t n, int32_t m,
                          const int32_t* src, const int32_t* dst,
                          const float* w);
/* Same graph from a fan-out CSR (_h_fanout_adjp/_adjncy/_wgts).  Returns once
 * the host-to-device copies have read the caller's buffers (they may be
 * reused at once).  The device graph (edge words, fan-in CSR, sources) is
 * then built on a least-priority stream the handle owns, and the first call
 * that uses the graph waits for it, so a caller streaming graphs through
 * several handles overlaps one handle's upload and build with another's
 * query.  A head outside [0, n) is reported by that first call
 * (CPG_ERR_INVALID, and the handle then holds no graph). */
cpg_status cpg_load_csr(cpg_handle* h, int32_t n, int32_t m,
                        const int32_t* adjp, const int32_t* adjncy,
                        const float* w);
/* CpGen::num_verts / num_edges (gpucpg.cu:286-292). */
int64_t cpg_num_verts(const cpg_handle* h);
int64_t cpg_num_edges(const cpg_handle* h);
/* Copy the fan-out CSR back (host buffers of n+1, m, m; any may be NULL). */
cpg_status cpg_get_csr(const cpg_handle* h, int32_t* adjp, int32_t* adjncy,
                       float* w);
/* Binary CSR file: int32 N, int32 M, int32 adjp[N+1], int32 adjncy[M],
 * float w[M] in host byte order (the layout of Graph::write_to_bin and
 * read_from_bin, gpucpg/graph.h:24-56), read on the host threads and checked
 * (size against the header, offsets rising from 0 to M, heads in range).
 * cpg_load_csr_bin stands for read_input + the CSR build on such a file;
 * cpg_write_csr_bin for CpGen::write_to_csr_bin (gpucpg.cuh:313-324), which
 * writes the adjacency where the offsets belong, so files it wrote fail the
 * offset check here. */
cpg_status cpg_load_csr_bin(cpg_handle* h, const char* path);
cpg_status cpg_write_csr_bin(const cpg_handle* h, const char* path);

/* Changes the handle's device-wait poll limit (cpg_options.spin_limit; 0 =
 * the default) for the calls that follow.  A wait that runs out returns
 * CPG_ERR_TIMEOUT and leaves the handle usable: the next call starts its
 * device work afresh.  The reference's waits are unbounded (the cooperative
 * loop's grid.sync(), gpucpg.cu:9152-9415); it has no such limit. */
cpg_status cpg_set_spin_limit(cpg_handle* h, uint32_t spin_limit);

/* Failure-injection hook for tests: from now on, every device buffer of a
 * handle, batch or server larger than max_bytes fails as out of device memory
 * (CPG_ERR_OOM) without calling cudaMalloc; 0 lifts the cap.  Process-wide.
 * The reference exits on any CUDA error instead (gpucpg.cu:87-98). */
void cpg_debug_fail_allocs_above(int64_t max_bytes);

/* ------------------------------------------------------------ suffix tree */
/* LEVELIZE_THEN_RELAX + update_successors_bu (gpucpg.cu:17642-17963,
 * 18421-18432): levels, fixed-point distances, successors and the sorted
 * deviation heaps.  Always recomputes. */
cpg_status cpg_levelize(cpg_handle* h);
/* Re-sample delays of fan-out edges (indices in CSR order).  Only the levels
 * at or above the lowest changed tail are recomputed at the next levelize. */
cpg_status cpg_update_delays(cpg_handle* h, int64_t count, const int32_t* eids,
                             const float* w);
/* Per-vertex distance (fixed point, INT32_MAX if unreachable), successor
 * (-1 at sinks) and reverse level (sinks 0, -1 if never levelled).  Host
 * buffers of n entries; any may be NULL.  Runs cpg_levelize if needed. */
cpg_status cpg_get_sfxt(cpg_handle* h, int32_t* dist, int32_t* succ,
                        int32_t* level);
int32_t cpg_num_levels(const cpg_handle* h);

/* ------------------------------------------------------------ prefix tree */
/* report_paths(k, ...) with LEVELIZE_THEN_RELAX and SHORT_LONG
 * (gpucpg.cu:16910-21366): the k smallest non-zero path costs, sorted
 * ascending, kept on the device until fetched.  Builds the suffix tree first
 * if it is not current.  Fewer than k paths are returned if fewer exist. */
cpg_status cpg_report_paths(cpg_handle* h, int64_t k);
/* report_paths on n handles (query i asks handles[i] for ks[i] paths), the
 * same as n cpg_report_paths calls; all queries are attempted and the first
 * failing status is returned (cpg_last_error of that handle says why).  For
 * many queries in one launch over side-by-side graphs, see cpg_batch_*. */
cpg_status cpg_report_paths_batch(cpg_handle* const* handles, const int64_t* ks, int32_t n);
/* get_slacks(k) (gpucpg.cu:21409-21420): copies min(k, available) costs. */
cpg_status cpg_get_costs(const cpg_handle* h, int64_t k, float* out,
                         int64_t* n_out);
/* get_pfxt_nodes(k) (gpucpg.cu:21422-21440). */
cpg_status cpg_get_paths(const cpg_handle* h, int64_t k, cpg_path_node* out,
                         int64_t* n_out);
/* Device pointer of the last result's costs (valid until the next report or
 * reset) and its length; lets callers keep results resident in HBM. */
cpg_status cpg_get_costs_device(const cpg_handle* h, const float** d_costs,
                                int64_t* n_out);
/* Full vertex sequence of result path i (0-based rank): walks the parent
 * links and suffix chains.  Writes at most cap vertices, *len = full length. */
cpg_status cpg_get_path_vertices(cpg_handle* h, int64_t i, int32_t* verts,
                                 int64_t cap, int64_t* len);
/* CpGen::reset() (gpucpg.cuh:211-250): drops results and the suffix tree,
 * keeps the graph. */
cpg_status cpg_reset(cpg_handle* h);
cpg_status cpg_get_stats(const cpg_handle* h, cpg_stats* out);
/* Synchronise the handle's stream. */
cpg_status cpg_sync(cpg_handle* h);

/* ------------------------------------------------------------ batched form */
/* Many independent queries (graph, k) answered together.  The graphs are
 * loaded side by side into one device graph; a step rebuilds the suffix
 * trees of all of them in one persistent launch and answers every query in
 * one persistent engine launch.  The step is captured once into a CUDA graph
 * and replayed.  Project-built form: the reference answers one query per
 * report_paths call and has no batched counterpart. */
typedef struct cpg_batch cpg_batch;

typedef struct {
  double step_ms;          /* device time of the last step (CUDA events) */
  double sfxt_ms;          /* part of step_ms spent in the suffix trees */
  int64_t paths_accepted;
  int32_t phases, rounds;
  int32_t graph_captured;  /* 1 when the step ran as a captured CUDA graph */
  int32_t retries;
  int64_t bytes_reserved;
  int32_t sfxt_ctas_per_sm;   /* launch shape chosen by cpg_batch_autotune */
  int32_t engine_ctas_per_sm;
  int32_t select_schedule;    /* 0: 11/11/10-bit radix digits, 1: 8/8/8/8 */
  int32_t sfxt_mode;          /* 0 dataflow (early push), 1 dataflow (late push), 2 level-synchronous */
  int32_t frontier_used;      /* cpg_frontier of the suffix-tree build */
  int32_t bvss_tiles;         /* cpg_bvss_tiles when the frontier is BVSS */
  int32_t tuned_candidates;   /* candidates timed by the last cpg_batch_autotune */
  int32_t pad;
} cpg_batch_stats;

cpg_status cpg_batch_create(cpg_batch** out, const cpg_options* opts);
cpg_status cpg_batch_destroy(cpg_batch* b);
const char* cpg_batch_last_error(const cpg_batch* b);
/* Append one graph (fan-out CSR, copied); *graph_id receives its index. */
cpg_status cpg_batch_add_graph(cpg_batch* b, int32_t n, int32_t m,
                               const int32_t* adjp, const int32_t* adjncy,
                               const float* w, int32_t* graph_id);
cpg_status cpg_batch_add_dag(cpg_batch* b, const cpg_dag* d, int32_t* graph_id);
/* Upload every graph added so far (one device graph). */
cpg_status cpg_batch_commit(cpg_batch* b);
/* Queries of the next steps: query i asks graph_ids[i] for ks[i] paths. */
cpg_status cpg_batch_set_queries(cpg_batch* b, int32_t nq,
                                 const int32_t* graph_ids, const int64_t* ks);
/* One step: rebuild the suffix trees (if rebuild_sfxt) and answer every
 * query.  The first step captures the CUDA graph; later steps replay it. */
cpg_status cpg_batch_run(cpg_batch* b, int32_t rebuild_sfxt);
/* Costs of query q from the last step (ascending, min(k, paths) of them). */
cpg_status cpg_batch_get_costs(const cpg_batch* b, int32_t q, float* out,
                               int64_t cap, int64_t* n_out);
cpg_status cpg_batch_get_stats(const cpg_batch* b, cpg_batch_stats* out);
/* Times candidate configurations over the set queries and keeps the fastest:
 * persistent grid sizes of the suffix-tree and engine kernels, the radix
 * digit schedule, the suffix-tree build mode and, when the side-by-side
 * graph's slices hold at least 1.5 heads on average (the BVSS density test),
 * the BVSS frontier with each tile policy.  Results are unchanged by any
 * choice. */
cpg_status cpg_batch_autotune(cpg_batch* b);

/* ------------------------------------------------------------ served form */
/* A C++ request loop over resident graphs.  Every graph's CSR and suffix tree
 * stay on the device; a query may carry delay updates for its graph, after
 * which only the affected levels of the suffix tree are rebuilt.  Queries
 * that arrive while a launch is running are admitted into the next one as
 * memory allows (predicted device footprint against hbm_budget_bytes), and
 * all admitted queries run together in one persistent engine launch
 * (continuous batching).  A query carrying updates starts a new launch, so
 * each query sees exactly the graph state of arrival order.  Project-built
 * form: no counterpart in the reference. */
typedef struct cpg_server cpg_server;

typedef struct {
  int32_t max_batch;          /* queries per engine launch (1 = one at a time) */
  int64_t hbm_budget_bytes;   /* admission budget for one launch; 0 = none */
  int32_t reserved[6];
} cpg_server_options;

typedef struct {
  int64_t completed;
  int64_t paths;              /* paths returned over completed queries */
  double p50_ms, p99_ms, mean_ms, max_ms;  /* submit -> result latency */
  double wall_s;              /* first submit -> last completion */
  double paths_per_s;         /* paths / wall_s */
  int64_t launches;           /* engine launches */
  int64_t sfxt_rebuilds;      /* incremental suffix-tree rebuilds */
  double busy_ms;             /* device time of all launches */
  int32_t max_batch_seen;
  int32_t reserved;
  double sfxt_ms;             /* device time of the suffix-tree rebuilds */
  int64_t retries;            /* launches rerun after a query buffer grew */
  int64_t pool_rebuilds;      /* full suffix-tree rebuilds after the heap pool filled */
  double max_step_ms;         /* longest loop step: updates, rebuild, launch, results */
  /* the longest of each part of a step, for diagnosis */
  double max_update_ms;       /* applying the admitted delay updates */
  double max_rebuild_ms;      /* the suffix-tree rebuild (incremental, or full after the pool filled) */
  double max_launch_ms;       /* the engine launch with its reruns after a buffer grew */
  double max_engine_ms;       /* the longest engine run on the GPU (CUDA events) */
  int64_t loop_allocs;        /* device or pinned buffers allocated inside the request
                                 loop (buffer growth); 0 while the admitted mix fits
                                 what cpg_server_start allocated */
} cpg_server_stats;

void cpg_server_options_init(cpg_server_options* o);
cpg_status cpg_server_create(cpg_server** out, const cpg_options* opts,
                             const cpg_server_options* sopts);
cpg_status cpg_server_destroy(cpg_server* s);
const char* cpg_server_last_error(const cpg_server* s);
cpg_status cpg_server_add_graph(cpg_server* s, int32_t n, int32_t m,
                                const int32_t* adjp, const int32_t* adjncy,
                                const float* w, int32_t* graph_id);
cpg_status cpg_server_add_dag(cpg_server* s, const cpg_dag* d, int32_t* graph_id);
/* Upload the graphs, build their suffix trees, start the request loop. */
cpg_status cpg_server_start(cpg_server* s);
/* Queue a query: k paths of graph_id after re-sampling n_updates delays
 * (edge ids in that graph's CSR order; may be 0).  Never blocks on the GPU. */
cpg_status cpg_server_submit(cpg_server* s, int32_t graph_id, int64_t k,
                             int32_t n_updates, const int32_t* eids,
                             const float* w, int64_t* ticket);
/* Wait (up to timeout_ms, < 0 = forever) for a ticket; copies up to cap
 * costs.  CPG_ERR_TIMEOUT if not done in time. */
cpg_status cpg_server_wait(cpg_server* s, int64_t ticket, float* out,
                           int64_t cap, int64_t* n_out, double* latency_ms,
                           int32_t timeout_ms);
/* Finish the queued work and stop the loop. */
cpg_status cpg_server_stop(cpg_server* s);
cpg_status cpg_server_get_stats(const cpg_server* s, cpg_server_stats* out);

/* ------------------------------------------------------------ top-K */
/* The k smallest non-zero values of a device array of path costs, ascending,
 * written to the device buffer d_out (room for k floats); *n_out receives
 * min(k, number of non-zero values).  This is the final step of report_paths
 * on its own: the reference sorts the whole short pile and drops zero-cost
 * nodes (gpucpg.cu:21323-21360); here a radix select finds the k-th value and
 * only the k survivors are radix-sorted.  Runs on `stream` (a cudaStream_t,
 * NULL for the default stream) and returns after the result is written.
 * Allocates and frees its own device scratch. */
cpg_status cpg_select_topk(const float* d_costs, int64_t n, int64_t k,
                           float* d_out, int64_t* n_out, void* stream);

/* Largest k cpg_select_topk_noalloc accepts. */
#define CPG_SELECT_TOPK_NOALLOC_MAX_K 262144

/* cpg_select_topk for callers that cannot allocate device memory: the same
 * k smallest non-zero costs, ascending, but its scratch is a fixed array
 * inside the library instead of cudaMalloc/cudaFree.  Meant for code that
 * runs where an allocation is not allowed or not affordable: between the
 * kernels of a pipeline whose other streams must keep running (cudaFree
 * synchronises the whole device), under a memory pool or budget that owns
 * every device byte, or in a process that has reserved all device memory up
 * front.  No counterpart in the reference, which allocates thrust vectors in
 * every report_paths call.
 *
 * Limits and rules:
 *  - k <= CPG_SELECT_TOPK_NOALLOC_MAX_K, else CPG_ERR_CAPACITY (nothing runs);
 *    n < 2^32.
 *  - The scratch (about 4.3 MiB) is reserved on every GPU that loads the
 *    library and kept until the process exits.
 *  - No call can run inside a stream capture: every call reads the count of
 *    non-zero costs back to the host partway through and synchronises
 *    `stream` before it returns.
 *  - The first call on a device looks up the scratch's device address (with
 *    that device current).  The address is kept for the life of the
 *    process: after cudaDeviceReset on that device the module is loaded
 *    again and the kept address is stale, so do not call this entry point
 *    across a device reset.
 *  - All calls share the one array: calls that overlap on the GPU (from two
 *    streams or threads at once) race and must be serialised by the caller.
 *  - Calls no cudaMalloc/cudaFree; returns after the result is written. */
cpg_status cpg_select_topk_noalloc(const float* d_costs, int64_t n, int64_t k,
                                   float* d_out, int64_t* n_out, void* stream);

/* ------------------------------------------------------------ BVSS */
/* Bit-vector slice sets (sigma = 8) of a row -> column relation, the
 * reference's HostBvss (gpucpg/tc_sfxt_bvss.cuh:17-31, tc_pfxt_bvss.cuh:7-25):
 * columns in intervals of 8, one slice (row, 8-bit mask) per row and interval,
 * slices packed 128 to a VSS (slice i in lane i % 32, chunk i / 32).  Built on
 * the host; the device copy is made on the first device call. */
typedef struct cpg_bvss cpg_bvss;

typedef struct {
  int32_t sigma;              /* 8 */
  int32_t slices_per_thread;  /* 4 */
  int32_t slice_capacity;     /* 128 */
  int32_t n_intervals;
  int32_t n_vss;
  int32_t n_rows;             /* rows the slices refer to */
  int64_t unpadded_slices;
  int64_t total_set_bits;
  double compression_ratio;   /* total_set_bits / (8 * unpadded_slices) */
} cpg_bvss_info;

typedef struct {
  int32_t device;
  void* stream;               /* cudaStream_t; NULL = the library's own */
  int32_t tiles;              /* cpg_bvss_tiles */
  int32_t min_bits;           /* density test (0 = default 2) */
  int32_t min_slices;         /* density test (0 = default 32) */
  int32_t half_slices;        /* skip the upper-half MMA of a VSS with at most
                                 this many slices (0 = default 64; the
                                 reference's shape dispatch) */
  uint32_t spin_limit;        /* grid-barrier polls; 0 = default */
  int32_t reserved[3];
} cpg_bvss_opts;

typedef struct {
  int32_t levels;             /* BFS levels holding a row (levels call) */
  int32_t pad;
  int64_t tiles_tensor;       /* VSS tiles counted on the tensor cores */
  int64_t tiles_scalar;       /* ... with scalar popc */
  int64_t mma_issued;         /* m8n8k128 b1 MMAs issued */
  double device_ms;
} cpg_bvss_run_stats;

void cpg_bvss_opts_init(cpg_bvss_opts* o);
/* Fan-out BVSS: rows are tail vertices, columns their heads
 * (build_bvss_from_fanout_csr, tc_sfxt_bvss.cuh:106-156).  With succs
 * non-NULL: the transposed deviation matrix A_dev, rows are heads v and
 * columns the tails u of edges u -> v with v != succs[u]
 * (build_adev_bvss_from_fanout_csr, tc_pfxt_bvss.cuh:117-175). */
cpg_status cpg_bvss_build(cpg_bvss** out, int32_t n, const int32_t* row_ptr,
                          const int32_t* col_idx, const int32_t* succs);
/* One slice per deviation d of source u: row d, column u
 * (build_adev_bvss_from_compact_deviation_offsets, tc_pfxt_bvss.cuh:177-226). */
cpg_status cpg_bvss_build_compact(cpg_bvss** out, int32_t n, const int32_t* deviation_offsets);
void cpg_bvss_destroy(cpg_bvss* b);
const char* cpg_bvss_last_error(const cpg_bvss* b);
cpg_status cpg_bvss_get_info(const cpg_bvss* b, cpg_bvss_info* info);
/* Copies the packed arrays; any NULL pointer is skipped.  Sizes:
 * real_ptrs n_intervals + 1, virtual_to_real and slice_counts n_vss,
 * row_ids 128 * n_vss, masks 32 * n_vss. */
cpg_status cpg_bvss_get_arrays(const cpg_bvss* b, int32_t* real_ptrs, int32_t* virtual_to_real,
                               uint8_t* slice_counts, int32_t* row_ids, uint32_t* masks);
/* Sorted columns of a row (decode_row_neighbors, tc_sfxt_bvss.cuh:158-183). */
cpg_status cpg_bvss_decode_row(const cpg_bvss* b, int32_t row, int32_t* out, int32_t cap,
                               int32_t* n_out);
/* 1 if the packed form holds exactly the distinct columns of every row of
 * the given CSR (verify_bvss_matches_csr / verify_adev_bvss_matches_csr),
 * 0 if not, negative on invalid input.  succs as in cpg_bvss_build. */
int32_t cpg_bvss_verify(const cpg_bvss* b, int32_t n, const int32_t* row_ptr,
                        const int32_t* col_idx, const int32_t* succs);
/* Pull BFS levels from the sinks over a fan-out BVSS: a row gets level L+1 the
 * first time one of its columns has level L; unreached rows get -1
 * (run_tc_bvss_pull_bfs_levels / run_scalar_bvss_pull_bfs_levels,
 * tc_sfxt_bvss.cuh:418-577; the tile choice is opts->tiles).  sinks = NULL
 * uses every row without columns.  levels: host array of n_rows. */
cpg_status cpg_bvss_levels(cpg_bvss* b, const cpg_bvss_opts* opts, const int32_t* sinks,
                           int32_t n_sinks, int32_t* levels, cpg_bvss_run_stats* stats);
/* Pairs (u, v) of an A_dev BVSS with u in the sources: every deviation edge
 * leaving the sources (discover_pairs_for_sources, tc_pfxt_bvss.cuh:582-636).
 * pairs: host array of 2 * max_pairs int32, sorted by (u, v) on return;
 * *n_pairs is the full count, CPG_ERR_CAPACITY when above max_pairs. */
cpg_status cpg_bvss_discover_pairs(cpg_bvss* b, const cpg_bvss_opts* opts,
                                   const int32_t* sources, int32_t n_sources, int32_t* pairs,
                                   int64_t max_pairs, int64_t* n_pairs,
                                   cpg_bvss_run_stats* stats);

/* ------------------------------------------------------------ generator */
/* Seeded levelised timing DAG in the reference's text format conventions:
 * explicit virtual super-source (id n_pins) and super-sink (id n_pins+1) with
 * zero-delay edges when add_virtual is set.  Host-only. */
typedef struct {
  uint64_t seed;
  int32_t n_pins;
  int32_t n_levels;
  int32_t n_first;        /* pins at level 0 */
  int32_t n_last;         /* pins at the last level */
  int32_t level_span;     /* edges go from level i to i+1..i+level_span */
  int32_t degree_kind;    /* 0: uniform {deg_lo..deg_hi}; 1: geometric */
  int32_t deg_lo, deg_hi;
  double deg_mean;        /* geometric mean (support 1, 2, ...) */
  int32_t deg_cap;
  int32_t weight_kind;    /* 0: fp32 uniform [w_lo, w_hi]; 1: integer */
  float w_lo, w_hi;
  int32_t iw_lo, iw_hi;
  int32_t add_virtual;
} cpg_gen_params;

void cpg_gen_params_init(cpg_gen_params* p);
cpg_status cpg_dag_generate(const cpg_gen_params* p, cpg_dag** out);
cpg_status cpg_dag_sizes(const cpg_dag* d, int32_t* n, int32_t* m);
cpg_status cpg_dag_edges(const cpg_dag* d, int32_t* src, int32_t* dst,
                         float* w);
cpg_status cpg_dag_write_text(const cpg_dag* d, const char* path);
/* Parse a graph in the reference's text format (the header line N, N vertex
 * name lines, then edge lines "u" -> "v"[, w];) into a host-side graph, in
 * parallel on the host threads.  Replaces the parsing half of
 * CpGen::read_input (gpucpg.cu:453-548); edges keep file order, blank lines
 * are skipped, and a malformed edge line fails with CPG_ERR_IO and its line
 * number in cpg_dag_last_error().  Host-only. */
cpg_status cpg_dag_read_text(const char* path, int32_t ignore_wgts, cpg_dag** out);
/* The binary CSR file above, to and from a host-side graph (rows keep the
 * edge order of the file).  Host-only. */
cpg_status cpg_dag_read_csr_bin(const char* path, cpg_dag** out);
cpg_status cpg_dag_write_csr_bin(const cpg_dag* d, const char* path);
/* Message of the last failing cpg_dag_* call on this thread. */
const char* cpg_dag_last_error(void);
cpg_status cpg_load_dag(cpg_handle* h, const cpg_dag* d);
void cpg_dag_free(cpg_dag* d);

#ifdef __cplusplus
}
#endif
#endif
