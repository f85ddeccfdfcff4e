// Internal declarations shared by the host orchestration (C++) and the CUDA
// translation units.  Nothing here is part of the public ABI (include/cpg.h).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cpg.h"

namespace cpg {

using Status = cpg_status;

// Fixed-point scale of the suffix distances: dist = sum of (int)(w * 10000.0f)
// (SCALE_UP, gpucpg/gpucpg.cuh:34).
constexpr int kScaleUp = 10000;

// ---------------------------------------------------------------- host graph
struct EdgeList {
  int32_t n = 0;
  std::vector<int32_t> src, dst;
  std::vector<float> w;
};

struct HostGraph {
  int32_t n = 0, m = 0;
  std::vector<int32_t> adjp, adj;  // fan-out CSR, rows in file order
  std::vector<float> w;
};

Status read_text_graph(const char* path, bool ignore_wgts, EdgeList& out,
                       std::string& err);
Status edges_to_csr(const EdgeList& el, HostGraph& g, std::string& err,
                    bool* grouped = nullptr);
Status generate_dag(const cpg_gen_params& p, EdgeList& out, std::string& err);
Status write_text_graph(const EdgeList& el, const char* path, std::string& err);
Status write_csr_bin(int32_t n, int32_t m, const int32_t* adjp, const int32_t* adj,
                     const float* w, const char* path, std::string& err);
Status read_csr_bin(const char* path, HostGraph& g, std::string& err);

// ---------------------------------------------------------------- device data
// One fan-out edge: head vertex and delay, loaded as one 8-byte word.
struct alignas(8) DevEdge {
  int32_t head;
  float w;
};

// One deviation ("sidetrack") edge (v, head) with head != succ[v]: the delay,
// the head's fixed-point distance and the sort key (its cost increase).  Each
// vertex's deviations are stored ascending by key in its own fan-out slots, so
// the list is also a binary min-heap (children 2j+1, 2j+2).
struct alignas(16) DevSidetrack {
  int32_t head;
  float w;
  int32_t dist_head;
  float key;
};

// Node of the persistent chain heap: the heap of vertex v holds, for every
// vertex u on v's suffix chain that has deviations, u's cheapest deviation.
// The heap of v shares every node but one root-to-leaf path with the heap of
// succ[v].  A node carries its element's whole record (the start of u's
// sorted deviation row, that deviation's head, delay and head distance, and
// u's distance), so a path search prices the element, and finds its row,
// from the node alone.  Heap order is (deviation_key of the record, vtx).
struct alignas(32) HeapNode {
  int32_t vtx;
  int32_t left;
  int32_t right;
  int32_t row;        // adjp[vtx]
  int32_t head;       // the cheapest deviation (entry 0 of the sorted row)
  float w;
  int32_t dist_head;
  int32_t dist_v;     // dist[vtx]
};

// Deviation rows are padded past the last edge by this many entries, so a
// search may load entry j of a row before checking j against the row's count
// (j <= 2 * count + 2 < 2 * the longest row).
constexpr int kDevPad = 2 * 16384 + 64;

// A path-graph item: the path "parent + the j-th deviation of vertex
// heap[node].vtx", or, when node <= -2, the root path that starts at source
// -(node + 2).  cost is the path's cost.
struct alignas(16) Item {
  float cost;
  int32_t parent;
  int32_t node;
  int32_t j;
};

struct GridBarrier {
  unsigned int count;
  unsigned int gen;
  int err;        // the status word as the last block to arrive found it
  int pad;
};

// Device error codes, written to a status word by kernels and mapped to
// cpg_status on the host.
enum DevErr : int {
  kDevOk = 0,
  kDevTimeout = 1,
  kDevCapacity = 2,
};

// Hot words sit on their own 128-byte lines: queue appends, the heap-pool
// cursor, the status word that waiting warps poll and the barrier do not
// contend for one L2 line.
constexpr int kMaxClaimSets = 16;
constexpr int kDefaultClaimSets = 8;

struct SfxtCounters {
  alignas(128) int tail;     // order[] / queue[] append cursor
  int act_n;                 // BVSS: act_list append cursor
  int level_end;             // tail and act_n snapshots taken at each level
  int act_end;               // barrier (adjacent: one two-word snapshot)
  alignas(128) int err;
  int levels;
  int sort_beg;              // order[] range whose deviation rows were rebuilt
  int sort_end;
  alignas(128) unsigned long long hnode_used;
  alignas(128) int n_long;   // rows left for the row-sort pass (long_rows[])
  // dataflow build: append cursors of the kSfxtQueues work queues, one line each
  alignas(128) int qtail[8][32];
  // dataflow build with claimed slots: claim[q][0] hands out the slots of
  // claim set q (slots q, q + S, q + 2S, ... for S = claim_sets)
  alignas(128) int claim[kMaxClaimSets][32];
  alignas(128) int sort_blocks;  // dataflow build: blocks whose level histogram is in
  int sort_ready;                // ... and the level offsets are scanned
  alignas(128) unsigned long long vss_tensor;  // BVSS tiles counted on the tensor cores
  unsigned long long vss_scalar;               // ... and with scalar popc
  alignas(128) GridBarrier bar;
};

// read back whole into the handle's 4 KiB pinned staging
static_assert(sizeof(SfxtCounters) <= 4096, "SfxtCounters outgrew the pinned staging");

struct SfxtParams {
  int32_t n;
  const int32_t* adjp;
  const DevEdge* edges;
  const int32_t* iadjp;
  const int32_t* iadj;
  int32_t* order;
  int32_t* lvlp;
  int32_t* level_of;
  int32_t* dist;
  int32_t* succ;
  int32_t* dev_cnt;
  DevSidetrack* dev;
  DevSidetrack* best;    // per vertex: its cheapest deviation (the heap element)
  int32_t* ht_root;
  int32_t* ht_size;
  HeapNode* hnodes;
  unsigned long long hnode_cap;
  unsigned long long* pool_mark;  // per level: heap nodes in use at its start
  int32_t* deps;
  const int32_t* big_off;  // big_tmp offset of big_rows[i]
  DevSidetrack* big_tmp;
  const int32_t* big_rows; // vertices with more than kSmemRow fan-out edges
  int32_t n_big_rows;
  int32_t big_row_cap;     // longest such row, rounded up to a power of two
  SfxtCounters* ctr;
  int32_t start_level;     // 0: full levelise + relax; > 0: relax from here
  int32_t known_levels;    // level count when start_level > 0
  unsigned int spin_limit;
  int32_t grid_limit;      // persistent CTAs (0: one per co-resident slot)
  // Incremental rebuild of some of several side-by-side graphs: vertex v is
  // rebuilt iff its level >= graph_from[vgraph[v]] (vgraph null: every vertex
  // of the rebuilt levels).  append_pool: new chain-heap nodes go after every
  // node in use instead of reusing the rebuilt levels' share of the pool.
  const int32_t* vgraph;
  const int32_t* graph_from;
  int32_t append_pool;
  // full CSR builds: dataflow work queue (n ints) unless level_sync is set
  int32_t* queue;
  int32_t* long_rows;      // rows over 64 edges, written unsorted (n ints)
  int32_t level_sync;
  int32_t heap_warps;      // dataflow: warps per CTA that only insert heaps (0: none)
  int32_t early_push;      // dataflow: push tails before the build, poll dl[]
  int32_t heap_phase;      // dataflow: chain heaps inserted after every build instead of
                           // by the building warp: 0 never, 1 on large graphs, 2 always
  unsigned long long* dl;  // dataflow: published (level << 32 | dist) per vertex
  int32_t claim_sets;      // dataflow: 0 = build warp w takes queue slots w, w + W, ...;
                           // S > 0 = a free warp claims the next slot of its claim set
  // Side-by-side graphs relabelled in level order (batched and served forms):
  // the caller's id of each vertex, for the successor tie-break; null when
  // the ids are the caller's
  const int32_t* orig_id;
  // BVSS pull for the Kahn step of a full build; used when bvss != 0
  int32_t bvss;
  const int32_t* bv_ptr;       // VSS range of each interval of 8 vertices
  const unsigned int* bv_masks;
  const int32_t* bv_rows;
  const uint8_t* bv_cnt;       // slices in each VSS
  const int32_t* bv_deps;      // distinct fan-out heads of each vertex
  unsigned int* fbits;         // frontier bitmap (n bits)
  unsigned int* iact;          // active-interval bitmap
  int32_t* act_list;           // active intervals, appended level after level
  int32_t mma_min_bits;        // density test of a tile, as BvssDispatch
  int32_t mma_min_slices;
  int32_t mma_mode;
};

// BVSS (bit-vector slice sets, sigma = 8) of a row -> column relation.
// Columns are grouped into intervals of 8; each row with columns in an
// interval contributes one slice (row, 8-bit mask).  An interval's slices, in
// row order, are packed 128 to a VSS: slice i of a VSS sits in lane i % 32,
// chunk i / 32, i.e. bits 8*chunk.. of masks[vss*32 + lane] and
// rows[vss*128 + lane*4 + chunk] (-1 pads).  The layout and the slice order
// are the reference's (gpucpg/tc_sfxt_bvss.cuh:17-31, 73-156).
struct HostBvss {
  int32_t n_rows = 0;              // vertex count of the graph
  int32_t n_intervals = 0, n_vss = 0;
  uint64_t unpadded_slices = 0, total_set_bits = 0;
  std::vector<int32_t> ptr;        // VSS range of each interval (n_intervals + 1)
  std::vector<int32_t> v2r;        // interval of each VSS
  std::vector<uint8_t> cnt;        // slices in each VSS
  std::vector<int32_t> rows;       // 128 per VSS
  std::vector<uint32_t> masks;     // 32 per VSS
  std::vector<int32_t> row_bits;   // distinct columns of each row
};
// Packs row -> columns given as a CSR over n rows with columns in [0, n).
Status pack_bvss(int32_t n, const int32_t* row_ptr, const int32_t* cols, HostBvss& out,
                 std::string& err);
// Packs one slice per (deviation, source) pair of a compact deviation CSR:
// row = deviation index, column = its source vertex
// (tc_pfxt_bvss.cuh:177-226).
Status pack_bvss_compact(int32_t n, const int32_t* dev_off, HostBvss& out, std::string& err);
// Sorted columns of one row, decoded from the packed form.
std::vector<int32_t> bvss_decode_row(const HostBvss& b, int32_t row);
// Average set bits per slice over the first `rows` rows of a CSR (the density
// test for the suffix tree's frontier choice).
double bvss_density_sample(int32_t n, const int32_t* row_ptr, const int32_t* cols,
                           int32_t rows);

// Device BVSS arrays.
struct DevBvss {
  int32_t n_rows, n_intervals, n_vss;
  const int32_t* ptr;
  const int32_t* v2r;
  const uint8_t* cnt;
  const int32_t* rows;
  const unsigned int* masks;
};
struct BvssDispatch {
  int32_t mode;            // 0 density test, 1 tensor cores always, 2 scalar always
  int32_t min_bits;        // density test: frontier byte has >= min_bits bits
  int32_t min_slices;      // ... and the VSS holds > min_slices slices
  int32_t half_slices;     // skip the upper-half MMA when slices <= this
};
struct BvssCounters {
  int err;
  int level;
  int qn[3];               // rotating queue sizes
  int pad;
  unsigned long long tiles_tensor, tiles_scalar, mma_issued;
  unsigned long long pairs;
  GridBarrier bar;
};
// Pull BFS levels from the sinks (min hops over fan-out edges), one
// persistent launch.  scratch: 3 frontier bitmaps + 3 queued-interval
// bitmaps + visited bitmap + 3 VSS queues (bvss_levels_scratch_words).
size_t bvss_levels_scratch_words(int32_t n, int32_t n_intervals, int32_t n_vss);
int launch_bvss_levels(const DevBvss& b, const int32_t* sinks, int32_t n_sinks,
                       int32_t* levels, unsigned int* scratch, BvssCounters* ctr,
                       BvssDispatch d, unsigned int spin_limit, int device, void* stream);
// Pairs (source u in the frontier, row v) of an A_dev BVSS.
size_t bvss_pairs_scratch_words(int32_t n_intervals, int32_t n_vss);
int launch_bvss_pairs(const DevBvss& b, const int32_t* sources, int32_t n_sources,
                      int32_t* pairs, long long max_pairs, unsigned int* scratch,
                      BvssCounters* ctr, BvssDispatch d, void* stream);

constexpr int kSfxtThreads = 1024;  // one block per SM: fewer grid-barrier arrivals
constexpr int kSmemRow = 256;  // deviation rows up to this length sort in smem

// Zero a build's counters on the device (capturable: no host copy).
int launch_init_sfxt_counters(SfxtCounters* c, const unsigned long long* pool_mark,
                              int start_level, int append_pool, void* stream);

// Launch the persistent SFXT kernel (cooperative) and the row sorts that
// follow it.  Returns a cudaError_t; *launches counts the kernels.
int launch_sfxt(const SfxtParams& p, int device, void* stream, int* grid_out,
                int* launches, void* ev_before = nullptr, void* ev_after = nullptr);

// ---------------------------------------------------------------- PFXT
struct PfxtCounters {
  int err;
  int pad0;
  unsigned long long paths;       // accepted paths (store cursor)
  unsigned long long frontier[3]; // rotating round counters
  unsigned long long pend_out;    // pending append cursor
  unsigned long long generated;
  int rounds;
  int pad1;
  GridBarrier bar;
};

struct PathStore {
  float* cost;
  int32_t* parent;
  int32_t* from;
  int32_t* to;
  int32_t* level;
  unsigned long long cap;
};

struct PfxtGraph {
  const int32_t* adjp;
  const int32_t* dist;
  const int32_t* dev_cnt;
  const DevSidetrack* dev;
  const int32_t* ht_root;
  const HeapNode* hnodes;
  int32_t division;  // cpg_division
};

struct ClosureParams {
  PfxtGraph g;
  PathStore ps;
  Item* front[2];
  unsigned long long front_cap;
  unsigned long long front_start;  // items already in front[0]
  Item* pend;                      // pending output
  unsigned long long pend_cap;
  float lim;                       // accept items with cost <= lim
  float tie;                       // accepted paths costing exactly this are
                                   // not expanded (NaN: expand all)
  PfxtCounters* ctr;
  unsigned int spin_limit;
};

int launch_closure(const ClosureParams& p, int device, void* stream,
                   int* grid_out);

// Seed root items for every source with a finite distance.
int launch_seed_roots(const int32_t* srcs, int32_t n_srcs, const int32_t* dist,
                      Item* pend, PfxtCounters* ctr, void* stream);

// Move pending items with cost <= lim into the frontier, the rest into
// pend_out.  Counts go to ctr->frontier[0] and ctr->pend_out.
int launch_promote(const Item* pend_in, unsigned long long n_in, float lim,
                   Item* front, unsigned long long front_cap, Item* pend_out,
                   unsigned long long pend_cap, PfxtCounters* ctr,
                   void* stream);

// ---------------------------------------------------------------- engine
// The persistent query engine (engine.cu) runs whole queries on the device:
// root seeding, every split raise, the closures, the final top-K select and
// the segmented sort, for any number of queries over one device graph, in
// one cooperative launch with no host round trip.
constexpr int kMaxQueries = 4096;   // Item.j carries the query id in 12 bits
constexpr int kJBits = 20;          // ... and the deviation index in 20 bits
constexpr unsigned kJMask = (1u << kJBits) - 1u;
constexpr int kSelBins = 2048;

struct EngineQuery {
  long long k;
  int src_beg, src_end;       // this query's sources in EngineParams::srcs
  int mode;                   // 0 idle, 1 grow, 2 final, 3 output select
  int done;
  float t, lim, tie, root_abs;
  unsigned int prefix;        // radix select state
  unsigned int coarse;        // growth phase split at a bin's upper edge
  unsigned long long krem;    // rank still wanted inside the prefix
  unsigned long long ksel;    // rank the select started from
  unsigned long long paths_nz, pend_nz, pend_n;     // maintained incrementally
  unsigned long long pend_next_n, pend_next_nz;      // the pile being written
  unsigned long long k_out, out_off, out_lt, out_eq;
  int phases;
  int pad;
  unsigned long long acc_prev, last_j;  // accepted before / promoted in the last growth phase
};

struct EngineCounters {
  alignas(128) int err;
  int active;
  int sel_paths;              // some query selects over accepted paths
  int err_stage;              // 1 + the first stage (barriers passed) with an error; 0 none
  int sel_stop;               // the select of this phase ended a pass early
  // append cursors, each on its own 128-byte line
  alignas(128) unsigned long long paths;
  alignas(128) unsigned long long frontier[3];
  alignas(128) unsigned long long pend_out;
  alignas(128) unsigned long long out_total;
  // single-query output: paths below and at the final split, and the key range
  alignas(128) unsigned long long out_below;
  alignas(128) unsigned long long out_at;
  alignas(128) unsigned int key_min, key_max;
  int rounds;
  int phases;
  int sorted_buf;             // which vals[] holds the sorted path indices
  int stopped;                // a one-CTA launch stopped at phase res_phase
  int res_phase, res_pin;     // the phase to resume and which pending pile is in
  unsigned long long res_paths, res_pend;
  // device time per stage (ns): 0 seed, 1 decide/bookkeeping, 2 select,
  // 3 promote, 4 closure, 5 output select, 6 output sort, 7 emit
  unsigned long long t_ns[8];
  alignas(128) GridBarrier bar;
};

struct EngineParams {
  PfxtGraph g;
  const int32_t* srcs;
  EngineQuery* q;
  int nq;
  int root_ref;               // reference G-PathGen root seeding
  PathStore ps;
  int32_t* pq;                // query of each accepted path
  Item* pend[2];
  unsigned long long pend_cap;
  Item* front[2];
  unsigned long long front_cap;
  unsigned int* hist;         // nq * kSelBins
  unsigned int* keys[2];
  unsigned int* qids[2];
  unsigned int* vals[2];
  unsigned long long out_cap;
  unsigned int* sort_hist;    // 256 * gridDim.x
  unsigned int* digit_tot;    // 256
  int32_t* rank_of;           // per accepted path, -1 if not reported
  float* out_cost;
  cpg_path_node* out_nodes;
  EngineCounters* ctr;
  unsigned int spin_limit;
  int grid_limit;             // persistent CTAs (0: one per co-resident slot)
  int grow_cap_k;             // cap a growth phase's promotion at K - accepted
  // Two launches for a single query: a one-CTA launch runs the phases while
  // the pending pile holds at most solo_stop items and stops there (state in
  // EngineCounters::res_*); the full launch (resume = 1) continues.
  unsigned long long solo_stop;
  int resume;
  int sel_passes;             // radix select digit schedule (sum of bits 32)
  int sel_shift[4];
  int sel_bits[4];
};

// Cooperative launch of the engine; *grid_out receives the grid size (the
// host sizes sort_hist as 256 * grid) for a given CTA limit (0: maximum).
int engine_grid(int device, int limit, int* grid_out);
int launch_engine(const EngineParams& p, int device, void* stream);
constexpr int kInlineQueries = 8;
int launch_set_queries(EngineQuery* dst, const EngineQuery* src, int nq, void* stream);

// ---------------------------------------------------------------- select/sort
size_t select_state_bytes();
// k-th smallest (1-based) value among the union of a (stride sa floats) and b
// (stride sb floats), zeros skipped if skip_zero.  *state receives the
// orderable key of that value (first 4 bytes) and its rank among equal keys
// (8-byte field at offset 8).  hist needs 2048 zeroed words.
int launch_select_kth(const float* a, unsigned long long na, unsigned sa,
                      const float* b, unsigned long long nb, unsigned sb,
                      unsigned long long k, int skip_zero, void* state,
                      unsigned int* hist, void* stream, int* launches);
// out[0] += #(x != 0 && key(x) <= *t_key), out[1] += #(x != 0).
int launch_count_le(const float* a, unsigned long long n, unsigned stride_f,
                    const unsigned int* t_key, unsigned long long* out,
                    void* stream);
// Sorted emission of the k smallest non-zero accepted paths (state from
// launch_select_kth over the accepted costs with k).  keys/vals: 2k words;
// hist: 256*ceil(k/2048) words; rank_of: n_paths; cnt: 2 words.
int launch_emit_topk(const PathStore& ps, unsigned long long n_paths,
                     const void* state, unsigned long long k,
                     unsigned int* keys, unsigned int* vals, unsigned int* hist,
                     unsigned long long* cnt, int32_t* rank_of, float* out_cost,
                     cpg_path_node* out_nodes, void* stream, int* launches);

// Host copies of the orderable float key map (device versions live in
// device_common.cuh).
float key_float_host(unsigned int k);
unsigned int float_key_host(float f);

// Device-side graph build from an uploaded fan-out CSR (graph_build.cu).
size_t build_scratch_words(int32_t n);
int launch_build_graph(const int32_t* adjp, const int32_t* adj, const float* w,
                       int32_t n, int64_t m, DevEdge* edges, int32_t* iadjp,
                       int32_t* iadj, int32_t* srcs, int32_t* n_srcs,
                       int32_t* scratch, void* stream);

// Standalone top-K of a device cost array (select_sort.cu).
struct TopkScratch {
  unsigned int* hist;             // 2048 words, zero on entry and on exit
  void* state;                    // select state, 16 bytes
  unsigned long long* counts;     // 2 words
  unsigned int* tkey;             // 1 word
  unsigned int* keys;             // 2*k words
  unsigned int* vals;             // 2*k words
  unsigned int* sort_hist;        // topk_sort_hist_words(k) words
  unsigned long long* cnt;        // 2 words
};
size_t topk_sort_hist_words(unsigned long long k);
int launch_topk_costs(const float* costs, unsigned long long n, unsigned long long k,
                      const TopkScratch& s, float* out, unsigned long long* n_out,
                      void* stream);

// Scatter new delays into the device fan-out edges.
int launch_scatter_delays(DevEdge* edges, const int32_t* eids, const float* w,
                          int64_t count, void* stream);

}  // namespace cpg
