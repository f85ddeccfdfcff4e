// C ABI and host orchestration of the critical path generator.
//
// Host side of the reference's CpGen::report_paths (gpucpg/gpucpg.cu:
// 16910-21366) for LEVELIZE_THEN_RELAX + SHORT_LONG: the graph and its suffix
// tree stay resident on the device across queries; each query raises a cost
// split until at least K non-zero paths cost <= split (the reference's
// SHORT_LONG stopping rule, 19134-20850), then selects and sorts the K
// cheapest.  Device work is in sfxt.cu, pfxt.cu and select_sort.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cpg_internal.hpp"

using namespace cpg;

namespace {

struct DevMem {
  void* p = nullptr;
  size_t bytes = 0;
};

constexpr unsigned int kDefaultSpinLimit = 1u << 24;
// the handle's pinned staging of counters and small tables
constexpr size_t kPinnedBytes = 4096;
// single queries: pending items up to which one CTA runs a phase
constexpr unsigned long long kEngSoloStop = 4096;
enum { kRetry = 1000 };  // internal: a bounded buffer overflowed, grow and rerun
constexpr int32_t kMaxRow = 16384;  // longest deviation row the row sort takes

}  // namespace

struct cpg_handle {
  cpg_options opts{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;

  // graph
  bool has_graph = false;
  bool build_pending = false;  // cpg_load_csr: the graph's first use waits for its device build
  // ... which starts at once on this least-priority stream (build_done marks
  // its end; the source count and head check land in pinned_build)
  cudaStream_t build_stream = nullptr;
  cudaEvent_t build_done = nullptr;
  int32_t* pinned_build = nullptr;
  bool build_launched = false;
  HostGraph g;          // n, m and the fan-out row offsets only
  int32_t n_srcs = 0;
  int32_t max_outdeg = 0;
  int64_t big_total = 0;
  int32_t big_rows = 0, big_cap = 1;
  DevMem d_adjp, d_edges, d_iadjp, d_iadj, d_srcs, d_big_off, d_big_tmp,
      d_big_rows;
  // several side-by-side graphs (batched and served forms): delay updates
  // rebuild only the changed graphs, from each one's lowest changed level
  bool multi_graph = false;
  std::vector<int32_t> graph_voff;  // first vertex of each graph
  std::vector<int32_t> graph_from;  // per graph: lowest changed level (INT32_MAX: clean)
  DevMem d_vgraph, d_graph_from, d_upd, d_queue, d_dl, d_long;
  // side-by-side graphs relabelled in level order by cpg_batch_commit: the
  // caller's id of each vertex (device) and the new position of each of the
  // caller's edges (host, for delay updates); empty otherwise
  bool relabeled = false;
  std::vector<int32_t> emap;
  DevMem d_orig_id;
  // BVSS form of the fan-out CSR, for the pull Kahn step
  bool use_bvss = false;
  double bvss_bps = 0;  // set bits per slice (sampled, or exact once built)
  DevMem d_bv_ptr, d_bv_masks, d_bv_rows, d_bv_cnt, d_bv_deps, d_fbits, d_iact, d_act_list;

  // suffix tree
  bool sfxt_valid = false;
  int32_t levels = 0;
  int32_t dirty_level = -1;  // lowest level whose delays changed
  std::vector<int32_t> h_level_of, h_succ;
  bool h_sfxt_cached = false;
  bool h_levels_cached = false;  // levels depend on the graph, not on delays
  DevMem d_order, d_lvlp, d_level_of, d_dist, d_succ, d_dev_cnt, d_dev,
      d_ht_root, d_ht_size, d_hnodes, d_pool_mark, d_deps, d_sctr, d_best;
  unsigned long long hnode_cap = 0;

  // query
  unsigned long long cap_paths = 0, cap_front = 0, cap_pend = 0;
  DevMem d_pcost, d_pparent, d_pfrom, d_pto, d_plevel, d_front0, d_front1,
      d_pend0, d_pend1, d_pctr, d_selstate, d_selhist, d_counts, d_keys,
      d_vals, d_sorthist, d_cnt, d_rank, d_out_cost, d_out_nodes, d_pq, d_qids,
      d_ehist, d_esort, d_equery, d_ectr;
  size_t sorted_vals_off = 0;  // where the sorted path indices start in d_vals
  int64_t n_result = 0;
  int64_t pool_rebuilds = 0;  // full suffix-tree rebuilds after the heap pool filled
  // engine counters of the last launch that overflowed (valid while set)
  bool overflow_known = false;
  unsigned long long overflow_paths = 0, overflow_pend = 0;
  unsigned long long n_paths = 0;
  bool result_valid = false;

  // launch shape (chosen by the batch autotuner; 0 = maximum co-resident)
  int sfxt_grid_limit = 0;
  int engine_grid_limit = 0;
  int sel_schedule = 0;  // 0: 11/11/10-bit select digits, 1: 8/8/8/8

  // staging
  void* pinned = nullptr;
  // pinned ring for large host-to-device uploads (kStageSlots x kStageChunk)
  char* stage = nullptr;
  cudaEvent_t stage_ev[4] = {};
  int stage_next = 0;
  cudaEvent_t ev[8] = {};  // [6], [7]: around the suffix-tree kernel alone
  cpg_stats stats{};
};

namespace {

Status fail(cpg_handle* h, Status s, const std::string& msg) {
  if (h) h->err = msg;
  return s;
}

Status cuda_fail(cpg_handle* h, int e, const char* what) {
  const cudaError_t ce = static_cast<cudaError_t>(e);
  if (ce == cudaErrorMemoryAllocation)
    return fail(h, CPG_ERR_OOM, std::string(what) + ": out of device memory");
  return fail(h, CPG_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(ce));
}

#define CK(expr, what)                                   \
  do {                                                   \
    const int _e = static_cast<int>(expr);               \
    if (_e != cudaSuccess) return cuda_fail(h, _e, what); \
  } while (0)

// Failure injection (cpg_debug_fail_allocs_above): device buffers larger
// than this fail as out of memory without reaching cudaMalloc; 0 = off.
std::atomic<int64_t> g_alloc_cap{0};
// Allocations made by the calling thread (device buffers and the server's
// pinned staging); the server loop reports the ones made inside it.
thread_local int64_t t_allocs = 0;

cudaError_t ensure(DevMem& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return cudaSuccess;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  const int64_t cap = g_alloc_cap.load(std::memory_order_relaxed);
  if (cap > 0 && bytes > static_cast<size_t>(cap)) return cudaErrorMemoryAllocation;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e == cudaSuccess) {
    b.bytes = bytes;
    ++t_allocs;
  }
  return e;
}

// ensure() for per-query buffers, whose size follows K and the batch: grows
// to at least twice the old size, so a stream of growing queries reallocates
// (and, with cudaFree, waits for the device) only a logarithmic number of times.
cudaError_t ensure_grow(DevMem& b, size_t bytes) {
  if (b.bytes >= bytes) return cudaSuccess;
  const size_t want = b.bytes ? std::max(bytes, 2 * b.bytes) : bytes;
  if (ensure(b, want) == cudaSuccess) return cudaSuccess;
  cudaGetLastError();
  return ensure(b, bytes);  // the doubled size did not fit: the size asked for
}

void release(DevMem& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

template <typename T>
T* P(DevMem& b) {
  return static_cast<T*>(b.p);
}

Status check_handle(cpg_handle* h) {
  if (!h) return CPG_ERR_INVALID;
  return CPG_OK;
}

// Host-to-device copy of a caller's (pageable) buffer.  Pageable copies run
// at about a fifth of the link's pinned rate, so large ones go through a
// pinned ring: host threads copy one chunk into a free slot while the copy
// engine moves the previous ones.  Small copies go directly.
constexpr size_t kStageChunk = size_t{16} << 20;
constexpr int kStageSlots = 4;
constexpr size_t kStageMin = size_t{8} << 20;

Status upload_h2d(cpg_handle* h, void* dst, const void* src, size_t bytes) {
  cudaStream_t s = h->stream;
  cudaPointerAttributes attr{};
  const bool pinned_src = cudaPointerGetAttributes(&attr, src) == cudaSuccess &&
                          attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  if (bytes < kStageMin || pinned_src) {  // pinned sources copy at full rate as they are
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "H2D");
    return CPG_OK;
  }
  if (!h->stage) {
    void* p = nullptr;
    CK(cudaMallocHost(&p, kStageChunk * kStageSlots), "pinned staging");
    h->stage = static_cast<char*>(p);
    for (auto& e : h->stage_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  }
  const int threads = std::max(1, std::min(8, static_cast<int>(std::thread::hardware_concurrency())));
  for (size_t off = 0; off < bytes; off += kStageChunk) {
    const size_t len = std::min(kStageChunk, bytes - off);
    const int slot = h->stage_next;
    h->stage_next = (slot + 1) % kStageSlots;
    CK(cudaEventSynchronize(h->stage_ev[slot]), "staging slot");  // its last copy is done
    char* stg = h->stage + static_cast<size_t>(slot) * kStageChunk;
    const char* from = static_cast<const char*>(src) + off;
    const size_t part = (len + threads - 1) / threads;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int t = 0; t < threads; ++t) {
      const size_t b = static_cast<size_t>(t) * part;
      if (b < len) std::memcpy(stg + b, from + b, std::min(part, len - b));
    }
    CK(cudaMemcpyAsync(static_cast<char*>(dst) + off, stg, len, cudaMemcpyHostToDevice, s), "H2D");
    CK(cudaEventRecord(h->stage_ev[slot], s), "event");
  }
  return CPG_OK;
}

// Density at which the BVSS pull takes over the Kahn step: with b set bits
// per slice the pull issues one atomic per slice where the CSR push issues
// one per edge, so it pays from about two heads per interval on.
constexpr double kBvssAutoBits = 2.0;

// Frontier choice for the Kahn step, and the BVSS build when it is used.
Status setup_bvss(cpg_handle* h, int32_t n, const int32_t* adjp, const int32_t* adj) {
  h->use_bvss = false;
  const int32_t mode = h->opts.frontier;
  if (mode == CPG_FRONTIER_CSR || n == 0) {
    h->bvss_bps = 0;
    return CPG_OK;
  }
  if (mode == CPG_FRONTIER_AUTO) {
    h->bvss_bps = bvss_density_sample(n, adjp, adj, 4096);
    if (h->bvss_bps < kBvssAutoBits) return CPG_OK;
  }
  HostBvss b;
  Status st = pack_bvss(n, adjp, adj, b, h->err);
  if (st != CPG_OK) return st;
  h->bvss_bps = b.unpadded_slices ? static_cast<double>(b.total_set_bits) /
                                        static_cast<double>(b.unpadded_slices)
                                  : 0.0;
  const size_t fw = (static_cast<size_t>(n) + 31) / 32;
  const size_t iw = (static_cast<size_t>(b.n_intervals) + 31) / 32;
  CK(ensure(h->d_bv_ptr, b.ptr.size() * 4), "alloc BVSS");
  CK(ensure(h->d_bv_masks, std::max<size_t>(b.masks.size(), 1) * 4), "alloc BVSS");
  CK(ensure(h->d_bv_rows, std::max<size_t>(b.rows.size(), 1) * 4), "alloc BVSS");
  CK(ensure(h->d_bv_cnt, std::max<size_t>(b.cnt.size(), 1)), "alloc BVSS");
  CK(ensure(h->d_bv_deps, b.row_bits.size() * 4), "alloc BVSS");
  CK(ensure(h->d_fbits, 2 * fw * 4), "alloc BVSS");
  CK(ensure(h->d_iact, 2 * iw * 4), "alloc BVSS");
  CK(ensure(h->d_act_list, static_cast<size_t>(n) * 4 + 4), "alloc BVSS");
  CK(cudaMemcpy(h->d_bv_ptr.p, b.ptr.data(), b.ptr.size() * 4, cudaMemcpyHostToDevice), "H2D BVSS");
  if (b.n_vss) {
    CK(cudaMemcpy(h->d_bv_masks.p, b.masks.data(), b.masks.size() * 4, cudaMemcpyHostToDevice), "H2D BVSS");
    CK(cudaMemcpy(h->d_bv_rows.p, b.rows.data(), b.rows.size() * 4, cudaMemcpyHostToDevice), "H2D BVSS");
    CK(cudaMemcpy(h->d_bv_cnt.p, b.cnt.data(), b.cnt.size(), cudaMemcpyHostToDevice), "H2D BVSS");
  }
  CK(cudaMemcpy(h->d_bv_deps.p, b.row_bits.data(), b.row_bits.size() * 4, cudaMemcpyHostToDevice), "H2D BVSS");
  h->use_bvss = true;
  return CPG_OK;
}

// Upload a fan-out CSR and build the rest of the graph on the device: edge
// words, fan-in CSR and source list.  The host keeps only the row offsets.
Status finish_graph(cpg_handle* h);
Status start_graph_build(cpg_handle* h);

// Uploads a fan-out CSR and builds the device graph from it.  defer: return
// once the copies have read the caller's buffers, with the build started on
// the handle's least-priority stream; the graph's first use (ready_graph)
// waits for it.  A caller streaming uploads through several handles then
// overlaps this one's copies and build with another's query.
Status upload_graph(cpg_handle* h, int32_t n, int32_t m, const int32_t* adjp,
                    const int32_t* adj, const float* w, bool defer = false) {
  if (n < 0 || m < 0 || !adjp || (m > 0 && (!adj || !w)))
    return fail(h, CPG_ERR_INVALID, "null CSR buffer");
  if (adjp[0] != 0 || adjp[n] != m)
    return fail(h, CPG_ERR_INVALID, "CSR offsets must start at 0 and end at m");
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  if (h->build_launched) {
    // an earlier upload's build still reads the staging and writes the graph
    CK(cudaEventSynchronize(h->build_done), "graph build");
    h->build_launched = false;
  }
  h->build_pending = false;
  h->has_graph = false;
  h->multi_graph = false;  // cpg_batch_commit sets it after the upload
  h->relabeled = false;    // so does it this
  h->emap.clear();
  h->graph_voff.clear();
  h->graph_from.clear();
  const size_t nn = static_cast<size_t>(n), mm = static_cast<size_t>(m);
  CK(ensure(h->d_adjp, (nn + 1) * 4), "alloc adjp");
  CK(ensure(h->d_edges, mm * sizeof(DevEdge)), "alloc edges");
  CK(ensure(h->d_iadjp, (nn + 1) * 4), "alloc iadjp");
  CK(ensure(h->d_iadj, mm * 4), "alloc iadj");
  CK(ensure(h->d_srcs, nn * 4 + 8), "alloc srcs");
  // suffix tree storage (the deviation array doubles as upload staging)
  CK(ensure(h->d_order, nn * 4), "alloc order");
  CK(ensure(h->d_queue, (nn + 64) * 4), "alloc queue");
  CK(ensure(h->d_long, nn * 4 + 4), "alloc row list");
  CK(ensure(h->d_dl, nn * 8 + 8), "alloc queue");
  CK(ensure(h->d_lvlp, (nn + 2) * 4), "alloc lvlp");
  CK(ensure(h->d_level_of, nn * 4), "alloc level_of");
  CK(ensure(h->d_dist, nn * 4), "alloc dist");
  CK(ensure(h->d_succ, nn * 4), "alloc succ");
  CK(ensure(h->d_dev_cnt, nn * 4), "alloc dev_cnt");
  CK(ensure(h->d_dev, (mm + kDevPad) * sizeof(DevSidetrack)), "alloc deviations");
  CK(ensure(h->d_best, nn * sizeof(DevSidetrack) + 16), "alloc deviations");
  CK(ensure(h->d_ht_root, nn * 4), "alloc ht_root");
  CK(ensure(h->d_ht_size, nn * 4), "alloc ht_size");
  CK(ensure(h->d_pool_mark, (nn + 2) * 8), "alloc pool_mark");
  CK(ensure(h->d_deps, std::max(nn, build_scratch_words(n)) * 4), "alloc deps");
  CK(ensure(h->d_sctr, sizeof(SfxtCounters)), "alloc sfxt counters");
  // ~10 path-copied nodes per vertex, plus the warps' private pool chunks
  // (64 nodes per warp of the dataflow build, 32 warps per SM)
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
  const unsigned long long want = nn * 10ull + 1024 + 64ull * 32 * static_cast<unsigned>(sms);
  if (h->hnode_cap < want) {
    h->hnode_cap = want;
    release(h->d_hnodes);
  }
  CK(ensure(h->d_hnodes, h->hnode_cap * sizeof(HeapNode)), "alloc chain heaps");
  cudaStream_t s = h->stream;
  int32_t* stage_adj = reinterpret_cast<int32_t*>(h->d_dev.p);
  float* stage_w = reinterpret_cast<float*>(stage_adj + mm);
  // the copies start first; the host checks below overlap them
  {
    Status st = upload_h2d(h, h->d_adjp.p, adjp, (nn + 1) * 4);
    if (st == CPG_OK && m) st = upload_h2d(h, stage_adj, adj, mm * 4);
    if (st == CPG_OK && m) st = upload_h2d(h, stage_w, w, mm * 4);
    if (st != CPG_OK) return st;
  }
  int32_t max_deg = 0, bad = 0;
#pragma omp parallel for reduction(max : max_deg) reduction(| : bad) schedule(static)
  for (int32_t v = 0; v < n; ++v) {
    const int32_t d = adjp[v + 1] - adjp[v];
    bad |= d < 0;
    max_deg = std::max(max_deg, d);
  }
  if (bad || max_deg > kMaxRow) {
    cudaStreamSynchronize(s);  // the copies still read the caller's buffers
    return fail(h, CPG_ERR_INVALID, bad ? "CSR offsets must be non-decreasing"
                                        : "out-degree above 16384 is not supported");
  }
  // heads are range-checked on the device while the graph is built
  {
    Status st = setup_bvss(h, n, adjp, adj);
    if (st != CPG_OK) {
      cudaStreamSynchronize(s);
      return st;
    }
  }
  h->g.n = n;
  h->g.m = m;
  h->g.adjp.assign(adjp, adjp + n + 1);
  h->g.adj.clear();
  h->g.w.clear();
  h->max_outdeg = max_deg;
  // rows too long for the shared-memory row sort (none in most graphs)
  std::vector<int32_t> big_off, big_rows;
  int64_t big_total = 0;
  int32_t big_cap = 1;
  if (max_deg > kSmemRow) {
    for (int32_t v = 0; v < n; ++v) {
      const int32_t od = adjp[v + 1] - adjp[v];
      if (od > kSmemRow) {
        big_off.push_back(static_cast<int32_t>(big_total));  // big_tmp offset of row i
        big_total += od;
        big_rows.push_back(v);
        while (big_cap < od) big_cap <<= 1;
      }
    }
  }
  h->big_total = big_total;
  h->big_rows = static_cast<int32_t>(big_rows.size());
  h->big_cap = big_cap;
  CK(ensure(h->d_big_rows, big_rows.size() * 4), "alloc big rows");
  CK(ensure(h->d_big_tmp, static_cast<size_t>(big_total) * sizeof(DevSidetrack)),
     "alloc big rows");
  CK(ensure(h->d_big_off, big_rows.size() * 4), "alloc big_off");
  if (!big_rows.empty()) {
    CK(cudaMemcpyAsync(h->d_big_off.p, big_off.data(), big_off.size() * 4, cudaMemcpyHostToDevice, s), "H2D big_off");
    CK(cudaMemcpyAsync(h->d_big_rows.p, big_rows.data(), big_rows.size() * 4, cudaMemcpyHostToDevice, s), "H2D big rows");
  }
  h->has_graph = true;
  h->sfxt_valid = false;
  h->h_sfxt_cached = false;
  h->h_levels_cached = false;
  h->dirty_level = -1;
  h->result_valid = false;
  h->n_result = 0;
  if (defer) {
    // the copies read the caller's buffers (and big_off / big_rows above)
    CK(cudaStreamSynchronize(s), "upload");
    h->build_pending = true;
    return start_graph_build(h);
  }
  return finish_graph(h);
}

// The device graph build of an upload (edge words, fan-in CSR, sources) from
// the staged adjacency and delays, and the head range check.
// Enqueues the device graph build on stream s; its source count and head
// check (two ints) go to hn.
Status enqueue_graph_build(cpg_handle* h, cudaStream_t s, int32_t* hn) {
  const int32_t n = h->g.n, m = h->g.m;
  const size_t nn = static_cast<size_t>(n), mm = static_cast<size_t>(m);
  int32_t* stage_adj = reinterpret_cast<int32_t*>(h->d_dev.p);
  float* stage_w = reinterpret_cast<float*>(stage_adj + mm);
  int32_t* nsrc_dev = P<int32_t>(h->d_srcs) + nn;
  CK(launch_build_graph(P<int32_t>(h->d_adjp), stage_adj, stage_w, n, m,
                        P<DevEdge>(h->d_edges), P<int32_t>(h->d_iadjp),
                        P<int32_t>(h->d_iadj), P<int32_t>(h->d_srcs), nsrc_dev,
                        P<int32_t>(h->d_deps), s), "build graph");
  CK(cudaMemcpyAsync(hn, nsrc_dev, 8, cudaMemcpyDeviceToHost, s), "D2H sources");
  return CPG_OK;
}

// Starts a deferred upload's build on the handle's least-priority stream, so
// it runs on whatever SMs the other streams leave idle (another handle's
// query, say); the graph's first use waits for it.
Status start_graph_build(cpg_handle* h) {
  if (!h->build_stream) {
    int least = 0, greatest = 0;
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
    CK(cudaStreamCreateWithPriority(&h->build_stream, cudaStreamNonBlocking, least),
       "build stream");
    CK(cudaEventCreateWithFlags(&h->build_done, cudaEventDisableTiming), "event");
    void* pb = nullptr;
    CK(cudaMallocHost(&pb, 64), "pinned");
    h->pinned_build = static_cast<int32_t*>(pb);
  }
  Status st = enqueue_graph_build(h, h->build_stream, h->pinned_build);
  if (st != CPG_OK) return st;
  CK(cudaEventRecord(h->build_done, h->build_stream), "event");
  h->build_launched = true;
  return CPG_OK;
}

// The host side of a build: the head check, the source count and order.
Status complete_graph_build(cpg_handle* h, const int32_t* hn) {
  if (hn[1] != 0) {
    h->has_graph = false;
    return fail(h, CPG_ERR_INVALID, "edge head out of range");
  }
  h->n_srcs = *hn;
  // sources in vertex-id order, as the reference's _srcs list (gpucpg.cu:
  // 531-533): G-PathGen's root seeding keeps the first roots in that order
  if (h->n_srcs > 1) {
    std::vector<int32_t> srcs(h->n_srcs);
    CK(cudaMemcpy(srcs.data(), h->d_srcs.p, srcs.size() * 4, cudaMemcpyDeviceToHost), "D2H sources");
    std::sort(srcs.begin(), srcs.end());
    CK(cudaMemcpy(h->d_srcs.p, srcs.data(), srcs.size() * 4, cudaMemcpyHostToDevice), "H2D sources");
  }
  return CPG_OK;
}

Status finish_graph(cpg_handle* h) {
  h->build_pending = false;
  h->build_launched = false;
  int32_t* hn = static_cast<int32_t*>(h->pinned);
  Status st = enqueue_graph_build(h, h->stream, hn);
  if (st != CPG_OK) return st;
  CK(cudaStreamSynchronize(h->stream), "upload");
  return complete_graph_build(h, hn);
}

// A loaded graph, built on the device: the build of a deferred upload, begun
// on the build stream, is waited for here (or run here if it was not begun).
Status ready_graph(cpg_handle* h) {
  if (!h->has_graph) return fail(h, CPG_ERR_STATE, "no graph loaded");
  if (!h->build_pending) return CPG_OK;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  if (!h->build_launched) return finish_graph(h);
  h->build_pending = false;
  h->build_launched = false;
  CK(cudaEventSynchronize(h->build_done), "graph build");
  return complete_graph_build(h, h->pinned_build);
}

Status load_edgelist(cpg_handle* h, const EdgeList& el) {
  HostGraph g;
  bool grouped = false;
  Status st = edges_to_csr(el, g, h->err, &grouped);
  if (st != CPG_OK) return st;
  // a list grouped by tail is its own adjacency
  return grouped ? upload_graph(h, g.n, g.m, g.adjp.data(), el.dst.data(), el.w.data())
                 : upload_graph(h, g.n, g.m, g.adjp.data(), g.adj.data(), g.w.data());
}

SfxtParams sfxt_params(cpg_handle* h, int32_t start_level) {
  SfxtParams p{};
  p.n = h->g.n;
  p.adjp = P<int32_t>(h->d_adjp);
  p.edges = P<DevEdge>(h->d_edges);
  p.iadjp = P<int32_t>(h->d_iadjp);
  p.iadj = P<int32_t>(h->d_iadj);
  p.order = P<int32_t>(h->d_order);
  p.lvlp = P<int32_t>(h->d_lvlp);
  p.level_of = P<int32_t>(h->d_level_of);
  p.dist = P<int32_t>(h->d_dist);
  p.succ = P<int32_t>(h->d_succ);
  p.dev_cnt = P<int32_t>(h->d_dev_cnt);
  p.dev = P<DevSidetrack>(h->d_dev);
  p.best = P<DevSidetrack>(h->d_best);
  p.ht_root = P<int32_t>(h->d_ht_root);
  p.ht_size = P<int32_t>(h->d_ht_size);
  p.hnodes = P<HeapNode>(h->d_hnodes);
  p.hnode_cap = h->hnode_cap;
  p.pool_mark = P<unsigned long long>(h->d_pool_mark);
  p.deps = P<int32_t>(h->d_deps);
  p.big_off = P<int32_t>(h->d_big_off);
  p.big_tmp = P<DevSidetrack>(h->d_big_tmp);
  p.big_rows = P<int32_t>(h->d_big_rows);
  p.n_big_rows = h->big_rows;
  p.big_row_cap = h->big_cap;
  p.ctr = P<SfxtCounters>(h->d_sctr);
  p.start_level = start_level;
  p.known_levels = h->levels;
  p.spin_limit = h->opts.spin_limit ? h->opts.spin_limit : kDefaultSpinLimit;
  p.grid_limit = h->sfxt_grid_limit;
  p.queue = P<int32_t>(h->d_queue);
  p.long_rows = P<int32_t>(h->d_long);
  p.level_sync = h->opts.sfxt_level_sync == 1;
  p.heap_warps = std::min(std::max(h->opts.sfxt_heap_warps, 0), 16);
  p.early_push = h->opts.sfxt_late_push != 1 && p.heap_warps == 0;
  p.heap_phase = p.heap_warps > 0 ? 0 : h->opts.sfxt_heap_mode == 1 ? 0
               : h->opts.sfxt_heap_mode == 2 ? 2 : 1;
  p.dl = P<unsigned long long>(h->d_dl);
  p.claim_sets = h->opts.sfxt_claim_sets < 0 ? 0
               : h->opts.sfxt_claim_sets == 0 ? kDefaultClaimSets
               : std::min(h->opts.sfxt_claim_sets, kMaxClaimSets);
  p.orig_id = h->relabeled ? P<int32_t>(h->d_orig_id) : nullptr;
  if (start_level > 0) {
    // a dataflow build allocates heap nodes out of level order, so rebuilt
    // levels take fresh nodes; a pool overflow falls back to a full build
    p.append_pool = 1;
    if (h->multi_graph) {
      p.vgraph = P<int32_t>(h->d_vgraph);
      p.graph_from = P<int32_t>(h->d_graph_from);
    }
  }
  if (h->use_bvss) {
    p.bvss = 1;
    p.bv_ptr = P<int32_t>(h->d_bv_ptr);
    p.bv_masks = P<unsigned int>(h->d_bv_masks);
    p.bv_rows = P<int32_t>(h->d_bv_rows);
    p.bv_cnt = P<uint8_t>(h->d_bv_cnt);
    p.bv_deps = P<int32_t>(h->d_bv_deps);
    p.fbits = P<unsigned int>(h->d_fbits);
    p.iact = P<unsigned int>(h->d_iact);
    p.act_list = P<int32_t>(h->d_act_list);
    p.mma_mode = h->opts.bvss_tiles;
    p.mma_min_bits = h->opts.bvss_min_bits > 0 ? h->opts.bvss_min_bits : 2;
    p.mma_min_slices = h->opts.bvss_min_slices > 0 ? h->opts.bvss_min_slices : 32;
  }
  return p;
}

// Device work of one suffix-tree build, asynchronous and capturable.
Status enqueue_sfxt(cpg_handle* h, int32_t start_level, int* launches,
                    bool kernel_events = false) {
  cudaStream_t s = h->stream;
  if (h->multi_graph && start_level > 0)
    CK(cudaMemcpyAsync(h->d_graph_from.p, h->graph_from.data(), h->graph_from.size() * 4,
                       cudaMemcpyHostToDevice, s), "H2D changed levels");
  CK(launch_init_sfxt_counters(P<SfxtCounters>(h->d_sctr), P<unsigned long long>(h->d_pool_mark),
                               start_level, start_level > 0, s),
     "sfxt counters");
  if (h->use_bvss && start_level == 0) {
    // the pull leaves the bitmaps clear; a build cut short by an error may not
    CK(cudaMemsetAsync(h->d_fbits.p, 0, h->d_fbits.bytes, s), "memset");
    CK(cudaMemsetAsync(h->d_iact.p, 0, h->d_iact.bytes, s), "memset");
  }
  int grid = 0;
  CK(launch_sfxt(sfxt_params(h, start_level), h->device, s, &grid, launches,
                 kernel_events ? h->ev[6] : nullptr, kernel_events ? h->ev[7] : nullptr),
     "sfxt launch");
  *launches += 1;
  return CPG_OK;
}

// Reads the build's counters back; kRetry when the heap pool overflowed.
int finish_sfxt(cpg_handle* h, int32_t start_level) {
  SfxtCounters* out = static_cast<SfxtCounters*>(h->pinned);
  CK(cudaMemcpyAsync(out, h->d_sctr.p, sizeof(SfxtCounters), cudaMemcpyDeviceToHost, h->stream),
     "D2H sfxt counters");
  CK(cudaStreamSynchronize(h->stream), "sfxt");
  if (out->err == kDevTimeout)
    return fail(h, CPG_ERR_TIMEOUT, "suffix tree: grid barrier wait ran out");
  if (out->err == kDevCapacity) return kRetry;
  if (start_level == 0) {
    h->levels = out->levels;
    h->h_levels_cached = false;
  }
  h->stats.levels = h->levels;
  if (start_level == 0) {
    h->stats.frontier_used = h->use_bvss ? CPG_FRONTIER_BVSS : CPG_FRONTIER_CSR;
    h->stats.bvss_tiles_tensor = static_cast<int64_t>(out->vss_tensor);
    h->stats.bvss_tiles_scalar = static_cast<int64_t>(out->vss_scalar);
  }
  h->stats.bvss_bits_per_slice = h->bvss_bps;
  h->sfxt_valid = true;
  h->h_sfxt_cached = false;
  h->dirty_level = -1;
  std::fill(h->graph_from.begin(), h->graph_from.end(), INT32_MAX);
  return CPG_OK;
}

Status grow_heap_pool(cpg_handle* h) {
  release(h->d_hnodes);
  h->hnode_cap *= 2;
  CK(ensure(h->d_hnodes, h->hnode_cap * sizeof(HeapNode)), "alloc chain heaps");
  return CPG_OK;
}

Status run_sfxt(cpg_handle* h, int32_t start_level) {
  cudaStream_t s = h->stream;
  for (int attempt = 0; attempt < 8; ++attempt) {
    CK(cudaEventRecord(h->ev[0], s), "event");
    int launches = 0;
    Status st = enqueue_sfxt(h, start_level, &launches, true);
    if (st != CPG_OK) return st;
    CK(cudaEventRecord(h->ev[1], s), "event");
    h->stats.kernel_launches += launches;
    const int r = finish_sfxt(h, start_level);
    float ms = 0.f, kms = 0.f;
    cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
    cudaEventElapsedTime(&kms, h->ev[6], h->ev[7]);
    h->stats.sfxt_ms = ms;
    h->stats.sfxt_kernel_ms = kms;
    if (r == kRetry) {
      // chain heaps outgrew their pool.  Incremental builds append to the
      // pool, so first rebuild from scratch (which compacts it); grow only
      // if a full build overflows.
      h->pool_rebuilds += 1;
      if (start_level == 0) {
        st = grow_heap_pool(h);
        if (st != CPG_OK) return st;
      }
      start_level = 0;
      continue;
    }
    return static_cast<Status>(r);
  }
  return fail(h, CPG_ERR_CAPACITY, "suffix tree: chain heap pool cannot grow");
}

Status cache_sfxt_host(cpg_handle* h) {
  if (h->h_sfxt_cached) return CPG_OK;
  const size_t n = h->g.n;
  h->h_level_of.resize(n);
  h->h_succ.resize(n);
  if (n) {
    CK(cudaMemcpy(h->h_level_of.data(), h->d_level_of.p, n * 4, cudaMemcpyDeviceToHost), "D2H levels");
    CK(cudaMemcpy(h->h_succ.data(), h->d_succ.p, n * 4, cudaMemcpyDeviceToHost), "D2H succ");
  }
  h->h_sfxt_cached = true;
  return CPG_OK;
}

// Host copy of the reverse levels (kept across delay updates).
Status ensure_levels_host(cpg_handle* h) {
  if (h->h_levels_cached) return CPG_OK;
  const size_t n = h->g.n;
  h->h_level_of.resize(n);
  if (n)
    CK(cudaMemcpy(h->h_level_of.data(), h->d_level_of.p, n * 4, cudaMemcpyDeviceToHost), "D2H levels");
  h->h_levels_cached = true;
  return CPG_OK;
}

Status ensure_sfxt(cpg_handle* h) {
  {
    Status st = ready_graph(h);
    if (st != CPG_OK) return st;
  }
  if (h->sfxt_valid) return CPG_OK;
  if (h->dirty_level > 0 && h->levels > 0)
    return run_sfxt(h, h->dirty_level);
  return run_sfxt(h, 0);
}

struct Counts {
  unsigned long long le, nz;
};

Status counts(cpg_handle* h, const float* a, unsigned long long n, unsigned stride,
              unsigned int t_key, Counts& out) {
  cudaStream_t s = h->stream;
  unsigned long long* dc = P<unsigned long long>(h->d_counts);
  unsigned int* tk = reinterpret_cast<unsigned int*>(dc + 2);
  CK(cudaMemsetAsync(dc, 0, 16, s), "memset counts");
  CK(cudaMemcpyAsync(tk, &t_key, 4, cudaMemcpyHostToDevice, s), "H2D key");
  CK(launch_count_le(a, n, stride, tk, dc, s), "count");
  h->stats.kernel_launches += 1;
  unsigned long long* hc = static_cast<unsigned long long*>(h->pinned);
  CK(cudaMemcpyAsync(hc, dc, 16, cudaMemcpyDeviceToHost, s), "D2H counts");
  CK(cudaStreamSynchronize(s), "counts");
  out.le = hc[0];
  out.nz = hc[1];
  return CPG_OK;
}

Status select_kth(cpg_handle* h, const float* a, unsigned long long na,
                  unsigned sa, const float* b, unsigned long long nb,
                  unsigned sb, unsigned long long k, int skip_zero,
                  float& value) {
  cudaStream_t s = h->stream;
  int launches = 0;
  CK(launch_select_kth(a, na, sa, b, nb, sb, k, skip_zero, h->d_selstate.p,
                       P<unsigned int>(h->d_selhist), s, &launches),
     "select");
  h->stats.kernel_launches += launches;
  unsigned int* hk = static_cast<unsigned int*>(h->pinned);
  CK(cudaMemcpyAsync(hk, h->d_selstate.p, 4, cudaMemcpyDeviceToHost, s), "D2H select");
  CK(cudaStreamSynchronize(s), "select");
  value = key_float_host(*hk);
  return CPG_OK;
}

float margin_of(float t, float root_abs) {
  const float a = std::max(std::max(std::fabs(t), root_abs), 1.0f);
  return a * 0x1p-16f;
}


// Capacities for the rerun after an engine launch overflowed.  The launch's
// counters kept counting past the ends, so a path store or pending pile that
// overflowed grows to 1.5x what it was asked to hold (at least twice its
// size); when neither did (the frontier or another buffer did), or the
// counters are unknown, every pile grows 4x.  Growing only what overflowed
// keeps the reallocation, which waits for the device, small.
void grow_caps(cpg_handle* h) {
  bool grown = false;
  if (h->overflow_known) {
    if (h->overflow_paths > h->cap_paths) {
      h->cap_paths = std::max(2 * h->cap_paths, h->overflow_paths + h->overflow_paths / 2);
      grown = true;
    }
    if (h->overflow_pend > h->cap_pend) {
      h->cap_pend = std::max(2 * h->cap_pend, h->overflow_pend + h->overflow_pend / 2);
      grown = true;
    }
  }
  if (!grown) {
    h->cap_paths *= 4;
    h->cap_front *= 4;
    h->cap_pend *= 4;
  }
  h->overflow_known = false;
}

Status alloc_query(cpg_handle* h, unsigned long long k) {
  const size_t cp = h->cap_paths, cf = h->cap_front, cpd = h->cap_pend;
  const size_t need =
      cp * 20 + 2 * cf * sizeof(Item) + 2 * cpd * sizeof(Item) + k * 4 * 4 +
      cp * 4 + k * (4 + sizeof(cpg_path_node)) + 256 * ((k + 2047) / 2048) * 4;
  if (h->opts.hbm_budget_bytes > 0 &&
      static_cast<int64_t>(need) > h->opts.hbm_budget_bytes)
    return fail(h, CPG_ERR_CAPACITY, "query needs more device memory than hbm_budget_bytes");
  h->stats.bytes_reserved = static_cast<int64_t>(need);
  CK(ensure_grow(h->d_pcost, cp * 4), "alloc paths");
  CK(ensure_grow(h->d_pparent, cp * 4), "alloc paths");
  CK(ensure_grow(h->d_pfrom, cp * 4), "alloc paths");
  CK(ensure_grow(h->d_pto, cp * 4), "alloc paths");
  CK(ensure_grow(h->d_plevel, cp * 4), "alloc paths");
  CK(ensure_grow(h->d_front0, cf * sizeof(Item)), "alloc frontier");
  CK(ensure_grow(h->d_front1, cf * sizeof(Item)), "alloc frontier");
  CK(ensure_grow(h->d_pend0, cpd * sizeof(Item)), "alloc pending");
  CK(ensure_grow(h->d_pend1, cpd * sizeof(Item)), "alloc pending");
  CK(ensure_grow(h->d_pctr, sizeof(PfxtCounters)), "alloc counters");
  CK(ensure_grow(h->d_selstate, 64), "alloc select");
  CK(ensure_grow(h->d_selhist, 2048 * 4), "alloc select");
  CK(ensure_grow(h->d_counts, 64), "alloc counts");
  CK(ensure_grow(h->d_keys, 2 * k * 4), "alloc sort");
  CK(ensure_grow(h->d_vals, 2 * k * 4), "alloc sort");
  CK(ensure_grow(h->d_sorthist, 256 * ((k + 2047) / 2048) * 4), "alloc sort");
  CK(ensure_grow(h->d_cnt, 16), "alloc sort");
  CK(ensure_grow(h->d_rank, cp * 4), "alloc rank");
  CK(ensure_grow(h->d_out_cost, k * 4), "alloc output");
  CK(ensure_grow(h->d_out_nodes, k * sizeof(cpg_path_node)), "alloc output");
  CK(cudaMemsetAsync(h->d_selhist.p, 0, 2048 * 4, h->stream), "memset hist");
  return CPG_OK;
}

PathStore path_store(cpg_handle* h) {
  PathStore ps;
  ps.cost = P<float>(h->d_pcost);
  ps.parent = P<int32_t>(h->d_pparent);
  ps.from = P<int32_t>(h->d_pfrom);
  ps.to = P<int32_t>(h->d_pto);
  ps.level = P<int32_t>(h->d_plevel);
  ps.cap = h->cap_paths;
  return ps;
}

Status read_pctr(cpg_handle* h, PfxtCounters& c) {
  PfxtCounters* hc = static_cast<PfxtCounters*>(h->pinned);
  CK(cudaMemcpyAsync(hc, h->d_pctr.p, sizeof(PfxtCounters), cudaMemcpyDeviceToHost, h->stream), "D2H counters");
  CK(cudaStreamSynchronize(h->stream), "counters");
  c = *hc;
  return CPG_OK;
}

// One attempt at a query with the current capacities.  Returns kRetry when a
// bounded buffer overflowed.
int try_query(cpg_handle* h, unsigned long long k) {
  Status st = alloc_query(h, k);
  if (st != CPG_OK) return st;
  cudaStream_t s = h->stream;
  PfxtCounters zero{};
  CK(cudaMemcpyAsync(h->d_pctr.p, &zero, sizeof(zero), cudaMemcpyHostToDevice, s), "H2D counters");
  PfxtCounters* dctr = P<PfxtCounters>(h->d_pctr);
  Item* pend_in = P<Item>(h->d_pend0);
  Item* pend_out = P<Item>(h->d_pend1);
  CK(launch_seed_roots(P<int32_t>(h->d_srcs), h->n_srcs,
                       P<int32_t>(h->d_dist), pend_in, dctr, s), "seed roots");
  h->stats.kernel_launches += 1;
  PfxtCounters c{};
  st = read_pctr(h, c);
  if (st != CPG_OK) return st;
  unsigned long long n_pend = c.pend_out;
  if (n_pend > h->cap_pend) return kRetry;
  // roots back on the host, in source-id order, for the seeding rule
  float root_abs = 0.f;
  {
    std::vector<Item> roots(n_pend);
    if (n_pend)
      CK(cudaMemcpy(roots.data(), pend_in, n_pend * sizeof(Item), cudaMemcpyDeviceToHost), "D2H roots");
    std::sort(roots.begin(), roots.end(),
              [](const Item& a, const Item& b) { return a.node > b.node; });
    if (h->opts.root_seeding == CPG_ROOTS_REFERENCE && !roots.empty()) {
      // G-PathGen's initial split (gpucpg.cu:19136-19179): split = cost at
      // sorted index (size_t)(0.005f*R); the short pile keeps only the first
      // (int)(0.005f*R + 1) roots at or below it
      const float perc = 0.005f;
      const size_t r = roots.size();
      std::vector<float> sorted(r);
      for (size_t i = 0; i < r; ++i) sorted[i] = roots[i].cost;
      std::sort(sorted.begin(), sorted.end());
      const float split = sorted[static_cast<size_t>(perc * r)];
      const int n_short = static_cast<int>(perc * r + 1);
      std::vector<Item> kept;
      int seen = 0;
      for (const Item& it : roots) {
        if (it.cost > split) kept.push_back(it);
        else if (seen < n_short) {
          ++seen;
          kept.push_back(it);
        }
      }
      roots.swap(kept);
      n_pend = roots.size();
      if (n_pend)
        CK(cudaMemcpy(pend_in, roots.data(), n_pend * sizeof(Item), cudaMemcpyHostToDevice), "H2D roots");
    }
    for (const Item& r : roots) root_abs = std::max(root_abs, std::fabs(r.cost));
  }
  unsigned long long n_paths = 0;
  const float* pcost = P<float>(h->d_pcost);
  const float* pend_cost_in = reinterpret_cast<const float*>(pend_in);
  float t = 0.f;
  int phases = 0;
  CK(cudaEventRecord(h->ev[2], s), "event");
  while (n_pend > 0) {
    Counts cp{}, cq{};
    pend_cost_in = reinterpret_cast<const float*>(pend_in);
    st = counts(h, pcost, n_paths, 1, 0xffffffffu, cp);
    if (st != CPG_OK) return st;
    st = counts(h, pend_cost_in, n_pend, 4, 0xffffffffu, cq);
    if (st != CPG_OK) return st;
    float lim, tie = std::nanf("");
    bool final_phase = false;
    if (cp.nz >= k) {
      // enough known candidates: the k-th smallest of paths and pending is
      // >= the answer's k-th cost, so one more closure finishes the query.
      // Paths costing exactly t are reported but not expanded.
      st = select_kth(h, pcost, n_paths, 1, pend_cost_in, n_pend, 4, k, 1, t);
      if (st != CPG_OK) return st;
      lim = t + margin_of(t, root_abs);
      tie = t;
      final_phase = true;
    } else {
      // too few known: grow geometrically by count.  Promoting the j cheapest
      // pending items (j ~ four times the accepted paths, at most half the
      // pile) keeps the split away
      // from expensive outliers, whose closure could be exponentially large;
      // accepting only costs strictly below the j-th keeps a tie group at
      // that cost for a later phase.
      const unsigned long long j = std::min<unsigned long long>(
          (n_pend + 1) / 2, std::max<unsigned long long>(64, 4 * (n_paths + 1)));
      st = select_kth(h, pend_cost_in, n_pend, 4, nullptr, 0, 1, j, 0, t);
      if (st != CPG_OK) return st;
      const float below = std::nextafter(t, -INFINITY);
      Counts lt{};
      st = counts(h, pend_cost_in, n_pend, 4, float_key_host(below), lt);
      if (st != CPG_OK) return st;
      // zeros are not counted by counts(); a zero-cost minimum promotes as is
      lim = (lt.le > 0) ? below : t;
    }
    // promote pending items under the split, then close over the frontier
    CK(cudaMemsetAsync(&dctr->frontier[0], 0, 3 * sizeof(unsigned long long), s), "memset");
    CK(cudaMemsetAsync(&dctr->pend_out, 0, sizeof(unsigned long long), s), "memset");
    CK(launch_promote(pend_in, n_pend, lim, P<Item>(h->d_front0), h->cap_front,
                      pend_out, h->cap_pend, dctr, s), "promote");
    ClosureParams cpar{};
    cpar.g.adjp = P<int32_t>(h->d_adjp);
    cpar.g.dist = P<int32_t>(h->d_dist);
    cpar.g.dev_cnt = P<int32_t>(h->d_dev_cnt);
    cpar.g.dev = P<DevSidetrack>(h->d_dev);
    cpar.g.ht_root = P<int32_t>(h->d_ht_root);
    cpar.g.hnodes = P<HeapNode>(h->d_hnodes);
    cpar.g.division = h->opts.division;
    cpar.ps = path_store(h);
    cpar.front[0] = P<Item>(h->d_front0);
    cpar.front[1] = P<Item>(h->d_front1);
    cpar.front_cap = h->cap_front;
    cpar.pend = pend_out;
    cpar.pend_cap = h->cap_pend;
    cpar.lim = lim;
    cpar.tie = tie;
    cpar.ctr = dctr;
    cpar.spin_limit = h->opts.spin_limit ? h->opts.spin_limit : kDefaultSpinLimit;
    int grid = 0;
    CK(launch_closure(cpar, h->device, s, &grid), "closure launch");
    h->stats.kernel_launches += 2;
    st = read_pctr(h, c);
    if (st != CPG_OK) return st;
    ++phases;
    if (c.err == kDevTimeout)
      return fail(h, CPG_ERR_TIMEOUT, "prefix tree: grid barrier wait ran out");
    if (c.err == kDevCapacity || c.paths > h->cap_paths || c.pend_out > h->cap_pend)
      return kRetry;
    n_paths = c.paths;
    n_pend = c.pend_out;
    std::swap(pend_in, pend_out);
    h->stats.pending_peak = std::max<int64_t>(h->stats.pending_peak, n_pend);
    if (final_phase) break;
  }
  CK(cudaEventRecord(h->ev[3], s), "event");
  // final: the k smallest non-zero accepted costs, sorted
  Counts all{};
  st = counts(h, pcost, n_paths, 1, 0xffffffffu, all);
  if (st != CPG_OK) return st;
  const unsigned long long k_out = std::min<unsigned long long>(k, all.nz);
  CK(cudaEventRecord(h->ev[4], s), "event");
  if (k_out > 0) {
    float kth = 0.f;
    st = select_kth(h, pcost, n_paths, 1, nullptr, 0, 1, k_out, 1, kth);
    if (st != CPG_OK) return st;
    int launches = 0;
    CK(launch_emit_topk(path_store(h), n_paths, h->d_selstate.p, k_out,
                        P<unsigned int>(h->d_keys), P<unsigned int>(h->d_vals),
                        P<unsigned int>(h->d_sorthist),
                        P<unsigned long long>(h->d_cnt), P<int32_t>(h->d_rank),
                        P<float>(h->d_out_cost),
                        P<cpg_path_node>(h->d_out_nodes), s, &launches),
       "emit");
    h->stats.kernel_launches += launches;
  }
  CK(cudaEventRecord(h->ev[5], s), "event");
  CK(cudaStreamSynchronize(s), "query");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]);
  h->stats.pfxt_ms = ms;
  cudaEventElapsedTime(&ms, h->ev[4], h->ev[5]);
  h->stats.select_ms = ms;
  h->stats.paths_accepted = static_cast<int64_t>(n_paths);
  h->stats.items_generated = static_cast<int64_t>(n_paths + n_pend);
  h->stats.phases = phases;
  h->stats.rounds = c.rounds;
  h->stats.split = t;
  h->n_paths = n_paths;
  h->n_result = static_cast<int64_t>(k_out);
  h->result_valid = true;
  return CPG_OK;
}

// ---- query engine: prepare (allocate, upload the query table), enqueue
// (asynchronous and capturable: memsets and one cooperative launch) and
// finish (read counters back, map errors).

// Buffers for nq queries whose K sum to k_total.
Status engine_prepare(cpg_handle* h, const std::vector<EngineQuery>& qs,
                      unsigned long long k_total) {
  Status st = alloc_query(h, k_total);
  if (st != CPG_OK) return st;
  int grid = 0;
  CK(engine_grid(h->device, h->engine_grid_limit, &grid), "engine occupancy");
  const size_t nq = qs.size();
  CK(ensure_grow(h->d_pq, h->cap_paths * 4), "alloc paths");
  CK(ensure_grow(h->d_qids, 2 * k_total * 4), "alloc sort");
  CK(ensure_grow(h->d_ehist, nq * static_cast<size_t>(kSelBins) * 4), "alloc select");
  CK(ensure_grow(h->d_esort, (256 * static_cast<size_t>(grid) + 256) * 4), "alloc sort");
  CK(ensure_grow(h->d_equery, nq * sizeof(EngineQuery)), "alloc queries");
  CK(ensure_grow(h->d_ectr, sizeof(EngineCounters)), "alloc counters");
  if (nq <= static_cast<size_t>(kInlineQueries)) {
    // no host-to-device copy: a large upload on another stream would hold it
    CK(launch_set_queries(P<EngineQuery>(h->d_equery), qs.data(), static_cast<int>(nq), h->stream),
       "queries");
    h->stats.kernel_launches += 1;
    return CPG_OK;
  }
  CK(cudaMemcpyAsync(h->d_equery.p, qs.data(), nq * sizeof(EngineQuery),
                     cudaMemcpyHostToDevice, h->stream), "H2D queries");
  CK(cudaStreamSynchronize(h->stream), "H2D queries");
  return CPG_OK;
}

// solo_stop > 0 (single queries): a one-CTA launch runs the phases while the
// pending pile holds at most solo_stop items, then the launch on the handle's
// CTA count resumes where it stopped (or finds the query answered and
// returns).  *launches receives the number of launches.
Status engine_enqueue(cpg_handle* h, int nq, unsigned long long k_total,
                      unsigned long long solo_stop = 0, int* launches = nullptr) {
  cudaStream_t s = h->stream;
  int grid = 0;
  CK(engine_grid(h->device, h->engine_grid_limit, &grid), "engine occupancy");
  CK(cudaMemsetAsync(h->d_ectr.p, 0, sizeof(EngineCounters), s), "memset");
  CK(cudaMemsetAsync(h->d_ehist.p, 0, static_cast<size_t>(nq) * kSelBins * 4, s), "memset");
  // every output slot is written by the compaction; zero-filling keeps a path
  // index in range even if selection and compaction ever disagreed
  CK(cudaMemsetAsync(h->d_vals.p, 0, 2 * k_total * 4, s), "memset");
  EngineParams p{};
  p.g.adjp = P<int32_t>(h->d_adjp);
  p.g.dist = P<int32_t>(h->d_dist);
  p.g.dev_cnt = P<int32_t>(h->d_dev_cnt);
  p.g.dev = P<DevSidetrack>(h->d_dev);
  p.g.ht_root = P<int32_t>(h->d_ht_root);
  p.g.hnodes = P<HeapNode>(h->d_hnodes);
  p.g.division = h->opts.division;
  p.srcs = P<int32_t>(h->d_srcs);
  p.q = P<EngineQuery>(h->d_equery);
  p.nq = nq;
  p.root_ref = h->opts.root_seeding == CPG_ROOTS_REFERENCE;
  p.ps = path_store(h);
  p.pq = P<int32_t>(h->d_pq);
  p.pend[0] = P<Item>(h->d_pend0);
  p.pend[1] = P<Item>(h->d_pend1);
  p.pend_cap = h->cap_pend;
  p.front[0] = P<Item>(h->d_front0);
  p.front[1] = P<Item>(h->d_front1);
  p.front_cap = h->cap_front;
  p.hist = P<unsigned int>(h->d_ehist);
  p.keys[0] = P<unsigned int>(h->d_keys);
  p.keys[1] = P<unsigned int>(h->d_keys) + k_total;
  p.qids[0] = P<unsigned int>(h->d_qids);
  p.qids[1] = P<unsigned int>(h->d_qids) + k_total;
  p.vals[0] = P<unsigned int>(h->d_vals);
  p.vals[1] = P<unsigned int>(h->d_vals) + k_total;
  p.out_cap = k_total;
  p.sort_hist = P<unsigned int>(h->d_esort);
  p.digit_tot = P<unsigned int>(h->d_esort) + 256 * static_cast<size_t>(grid);
  p.rank_of = P<int32_t>(h->d_rank);
  p.out_cost = P<float>(h->d_out_cost);
  p.out_nodes = P<cpg_path_node>(h->d_out_nodes);
  p.ctr = P<EngineCounters>(h->d_ectr);
  p.spin_limit = h->opts.spin_limit ? h->opts.spin_limit : kDefaultSpinLimit;
  p.grid_limit = h->engine_grid_limit;
  p.grow_cap_k = 1;
  if (h->sel_schedule == 1) {  // four 8-bit digits
    p.sel_passes = 4;
    for (int i = 0; i < 4; ++i) {
      p.sel_shift[i] = 24 - 8 * i;
      p.sel_bits[i] = 8;
    }
  } else {                     // 11 + 11 + 10 bits
    p.sel_passes = 3;
    p.sel_shift[0] = 21; p.sel_bits[0] = 11;
    p.sel_shift[1] = 10; p.sel_bits[1] = 11;
    p.sel_shift[2] = 0;  p.sel_bits[2] = 10;
  }
  if (solo_stop > 0 && grid > 1) {
    EngineParams a = p;
    a.grid_limit = 1;
    a.solo_stop = solo_stop;
    CK(launch_engine(a, h->device, s), "engine launch");
    p.resume = 1;
    CK(launch_engine(p, h->device, s), "engine launch");
    if (launches) *launches = 2;
    return CPG_OK;
  }
  CK(launch_engine(p, h->device, s), "engine launch");
  if (launches) *launches = 1;
  return CPG_OK;
}

// Counters and the per-query table back on the host.  kRetry on overflow.
int engine_finish(cpg_handle* h, std::vector<EngineQuery>& qout, EngineCounters& c,
                  unsigned long long k_total) {
  const size_t nq = qout.size();
  char* hb = static_cast<char*>(h->pinned);
  // a few queries' table comes back with the counters, in one pinned copy
  constexpr size_t kQoff = (sizeof(EngineCounters) + 127) & ~size_t{127};
  const bool inline_q = kQoff + nq * sizeof(EngineQuery) <= kPinnedBytes;
  CK(cudaMemcpyAsync(hb, h->d_ectr.p, sizeof(EngineCounters), cudaMemcpyDeviceToHost,
                     h->stream), "D2H counters");
  if (inline_q)
    CK(cudaMemcpyAsync(hb + kQoff, h->d_equery.p, nq * sizeof(EngineQuery),
                       cudaMemcpyDeviceToHost, h->stream), "D2H queries");
  CK(cudaStreamSynchronize(h->stream), "engine");
  std::memcpy(&c, hb, sizeof(c));
  if (c.err == kDevTimeout)
    return fail(h, CPG_ERR_TIMEOUT, "query engine: grid barrier wait ran out");
  if (c.err == kDevCapacity) {
    h->overflow_known = true;
    h->overflow_paths = c.paths;
    h->overflow_pend = c.pend_out;
    return kRetry;
  }
  if (inline_q)
    std::memcpy(qout.data(), hb + kQoff, nq * sizeof(EngineQuery));
  else
    CK(cudaMemcpy(qout.data(), h->d_equery.p, nq * sizeof(EngineQuery), cudaMemcpyDeviceToHost),
       "D2H queries");
  h->stats.paths_accepted = static_cast<int64_t>(c.paths);
  h->stats.items_generated = static_cast<int64_t>(c.paths + c.pend_out);
  h->stats.pending_peak = static_cast<int64_t>(c.pend_out);
  h->stats.phases = c.phases;
  h->stats.rounds = c.rounds;
  for (int i = 0; i < 8; ++i) h->stats.engine_stage_ms[i] = static_cast<float>(c.t_ns[i] * 1e-6);
  h->n_paths = c.paths;
  h->sorted_vals_off = c.sorted_buf ? k_total : 0;
  return CPG_OK;
}

// One query through the engine.  Returns kRetry when a bounded buffer
// overflowed.
int engine_query(cpg_handle* h, unsigned long long k) {
  // CTAs of the engine launch: the option, else chosen from K (a small
  // query's phases are bound by barrier latency, and one CTA's grid barrier
  // is a block barrier)
  // (measured on the 20,000-pin and 1M-pin graphs: one CTA is fastest up to
  // K of about 2,000 -- 0.33 against 0.61 ms at K = 1,000 -- eight around
  // K = 1e4, then about K / 3,000, up to one per SM at K = 1e6)
  int ctas = h->opts.engine_ctas;
  if (ctas <= 0) {
    if (k <= 2000) ctas = 1;
    else if (k <= 20000) ctas = 8;
    else ctas = static_cast<int>(std::min<unsigned long long>(std::max<unsigned long long>(k / 3000, 16), 1u << 20));
  }
  h->engine_grid_limit = ctas;  // engine_grid caps it at the co-resident CTAs
  std::vector<EngineQuery> qs(1);
  qs[0].k = static_cast<long long>(k);
  qs[0].src_beg = 0;
  qs[0].src_end = h->n_srcs;
  Status st = engine_prepare(h, qs, k);
  if (st != CPG_OK) return st;
  cudaStream_t s = h->stream;
  CK(cudaEventRecord(h->ev[2], s), "event");
  // the first phases move a few thousand items at most: one CTA runs them
  // on block barriers, the full launch takes over once the pile is larger
  int launches = 0;
  st = engine_enqueue(h, 1, k, kEngSoloStop, &launches);
  if (st != CPG_OK) return st;
  CK(cudaEventRecord(h->ev[3], s), "event");
  h->stats.kernel_launches += launches;
  EngineCounters c;
  const int r = engine_finish(h, qs, c, k);
  if (r != CPG_OK) return r;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]);
  h->stats.pfxt_ms = ms;
  h->stats.select_ms = 0.0;
  h->stats.split = qs[0].t;
  h->n_result = static_cast<int64_t>(qs[0].k_out);
  h->result_valid = true;
  return CPG_OK;
}

}  // namespace

float cpg::key_float_host(unsigned int k) {
  unsigned int u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

unsigned int cpg::float_key_host(float f) {
  unsigned int u;
  std::memcpy(&u, &f, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// ====================================================================== ABI

extern "C" {

int32_t cpg_abi_version(void) { return CPG_ABI_VERSION; }

const char* cpg_status_string(cpg_status s) {
  switch (s) {
    case CPG_OK: return "ok";
    case CPG_ERR_INVALID: return "invalid argument";
    case CPG_ERR_IO: return "i/o error";
    case CPG_ERR_OOM: return "out of memory";
    case CPG_ERR_CAPACITY: return "capacity exceeded";
    case CPG_ERR_TIMEOUT: return "device wait timed out";
    case CPG_ERR_CUDA: return "cuda error";
    case CPG_ERR_STATE: return "bad call order";
    case CPG_ERR_NO_DEVICE: return "no cuda device";
  }
  return "unknown";
}

void cpg_options_init(cpg_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->division = CPG_DIV_REFERENCE;
  o->frontier = CPG_FRONTIER_AUTO;
}

cpg_status cpg_create(cpg_handle** out, const cpg_options* opts) {
  if (!out) return CPG_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CPG_ERR_NO_DEVICE;
  }
  cpg_handle* h = new (std::nothrow) cpg_handle();
  if (!h) return CPG_ERR_OOM;
  if (opts) h->opts = *opts;
  else cpg_options_init(&h->opts);
  if (h->opts.division != CPG_DIV_REFERENCE && h->opts.division != CPG_DIV_IEEE) {
    delete h;
    return CPG_ERR_INVALID;
  }
  h->device = h->opts.device;
  if (h->device < 0 || h->device >= ndev) {
    delete h;
    return CPG_ERR_INVALID;
  }
  if (cudaSetDevice(h->device) != cudaSuccess) {
    delete h;
    return CPG_ERR_CUDA;
  }
  if (h->opts.stream) {
    h->stream = static_cast<cudaStream_t>(h->opts.stream);
  } else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete h;
      return CPG_ERR_CUDA;
    }
    h->own_stream = true;
  }
  if (cudaMallocHost(&h->pinned, kPinnedBytes) != cudaSuccess) {
    if (h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
    return CPG_ERR_OOM;
  }
  for (auto& e : h->ev) cudaEventCreate(&e);
  *out = h;
  return CPG_OK;
}

cpg_status cpg_destroy(cpg_handle* h) {
  if (!h) return CPG_ERR_INVALID;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  if (h->build_stream) cudaStreamSynchronize(h->build_stream);  // a graph build still running
  DevMem* all[] = {&h->d_adjp, &h->d_edges, &h->d_iadjp, &h->d_iadj, &h->d_srcs,
                   &h->d_big_off, &h->d_big_tmp, &h->d_big_rows, &h->d_order, &h->d_lvlp,
                   &h->d_level_of, &h->d_dist, &h->d_succ, &h->d_dev_cnt,
                   &h->d_dev, &h->d_best, &h->d_ht_root, &h->d_ht_size, &h->d_hnodes,
                   &h->d_pool_mark, &h->d_deps, &h->d_sctr, &h->d_pcost,
                   &h->d_pparent, &h->d_pfrom, &h->d_pto, &h->d_plevel,
                   &h->d_front0, &h->d_front1, &h->d_pend0, &h->d_pend1,
                   &h->d_pctr, &h->d_selstate, &h->d_selhist, &h->d_counts,
                   &h->d_keys, &h->d_vals, &h->d_sorthist, &h->d_cnt,
                   &h->d_rank, &h->d_out_cost, &h->d_out_nodes, &h->d_pq,
                   &h->d_qids, &h->d_ehist, &h->d_esort, &h->d_equery, &h->d_ectr,
                   &h->d_bv_ptr, &h->d_bv_masks, &h->d_bv_rows, &h->d_bv_cnt,
                   &h->d_bv_deps, &h->d_fbits, &h->d_iact, &h->d_act_list,
                   &h->d_vgraph, &h->d_graph_from, &h->d_upd, &h->d_queue, &h->d_dl,
                   &h->d_long, &h->d_orig_id};
  for (DevMem* b : all) release(*b);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->pinned) cudaFreeHost(h->pinned);
  if (h->build_stream) {
    cudaStreamDestroy(h->build_stream);
    cudaEventDestroy(h->build_done);
    cudaFreeHost(h->pinned_build);
  }
  if (h->stage) {
    cudaFreeHost(h->stage);
    for (auto& e : h->stage_ev)
      if (e) cudaEventDestroy(e);
  }
  if (h->own_stream) cudaStreamDestroy(h->stream);
  delete h;
  return CPG_OK;
}

const char* cpg_last_error(const cpg_handle* h) {
  return h ? h->err.c_str() : "null handle";
}

cpg_status cpg_load_text(cpg_handle* h, const char* path, int32_t ignore_wgts) {
  if (check_handle(h) != CPG_OK || !path) return CPG_ERR_INVALID;
  EdgeList el;
  Status st = read_text_graph(path, ignore_wgts != 0, el, h->err);
  if (st != CPG_OK) return st;
  return load_edgelist(h, el);
}

cpg_status cpg_load_csr_bin(cpg_handle* h, const char* path) {
  if (check_handle(h) != CPG_OK || !path) return CPG_ERR_INVALID;
  HostGraph g;
  Status st = read_csr_bin(path, g, h->err);
  if (st != CPG_OK) return st;
  return upload_graph(h, g.n, g.m, g.adjp.data(), g.adj.data(), g.w.data());
}

cpg_status cpg_write_csr_bin(const cpg_handle* h, const char* path) {
  if (!h || !path) return CPG_ERR_INVALID;
  if (!h->has_graph) return CPG_ERR_STATE;
  const int32_t n = h->g.n, m = h->g.m;
  std::vector<int32_t> adjp(static_cast<size_t>(n) + 1), adj(static_cast<size_t>(m));
  std::vector<float> w(static_cast<size_t>(m));
  Status st = cpg_get_csr(h, adjp.data(), adj.data(), w.data());
  if (st != CPG_OK) return st;
  cpg_handle* hm = const_cast<cpg_handle*>(h);
  return write_csr_bin(n, m, adjp.data(), adj.data(), w.data(), path, hm->err);
}

cpg_status cpg_load_edges(cpg_handle* h, int32_t n, int32_t m,
                          const int32_t* src, const int32_t* dst,
                          const float* w) {
  if (check_handle(h) != CPG_OK || n < 0 || m < 0) return CPG_ERR_INVALID;
  if (m > 0 && (!src || !dst || !w)) return fail(h, CPG_ERR_INVALID, "null edge buffer");
  EdgeList el;
  el.n = n;
  el.src.assign(src, src + m);
  el.dst.assign(dst, dst + m);
  el.w.assign(w, w + m);
  return load_edgelist(h, el);
}

cpg_status cpg_load_csr(cpg_handle* h, int32_t n, int32_t m,
                        const int32_t* adjp, const int32_t* adjncy,
                        const float* w) {
  if (check_handle(h) != CPG_OK) return CPG_ERR_INVALID;
  return upload_graph(h, n, m, adjp, adjncy, w, true);
}

int64_t cpg_num_verts(const cpg_handle* h) { return h && h->has_graph ? h->g.n : 0; }
int64_t cpg_num_edges(const cpg_handle* h) { return h && h->has_graph ? h->g.m : 0; }

cpg_status cpg_get_csr(const cpg_handle* hc, int32_t* adjp, int32_t* adjncy,
                       float* w) {
  cpg_handle* h = const_cast<cpg_handle*>(hc);
  if (!h) return CPG_ERR_INVALID;
  if (!h->has_graph) return CPG_ERR_STATE;
  {
    Status st = ready_graph(h);
    if (st != CPG_OK) return st;
  }
  if (adjp) std::memcpy(adjp, h->g.adjp.data(), (h->g.n + 1) * 4);
  if ((adjncy || w) && h->g.m) {
    std::vector<DevEdge> e(h->g.m);
    CK(cudaMemcpy(e.data(), h->d_edges.p, e.size() * sizeof(DevEdge), cudaMemcpyDeviceToHost), "D2H edges");
    for (int32_t i = 0; i < h->g.m; ++i) {
      if (adjncy) adjncy[i] = e[i].head;
      if (w) w[i] = e[i].w;
    }
  }
  return CPG_OK;
}

cpg_status cpg_levelize(cpg_handle* h) {
  if (check_handle(h) != CPG_OK) return CPG_ERR_INVALID;
  if (!h->has_graph) return fail(h, CPG_ERR_STATE, "no graph loaded");
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  h->stats.kernel_launches = 0;
  h->sfxt_valid = false;
  return ensure_sfxt(h);
}

cpg_status cpg_set_spin_limit(cpg_handle* h, uint32_t spin_limit) {
  if (check_handle(h) != CPG_OK) return CPG_ERR_INVALID;
  h->opts.spin_limit = spin_limit;
  return CPG_OK;
}

void cpg_debug_fail_allocs_above(int64_t max_bytes) {
  g_alloc_cap.store(max_bytes > 0 ? max_bytes : 0, std::memory_order_relaxed);
}

cpg_status cpg_update_delays(cpg_handle* h, int64_t count, const int32_t* eids,
                             const float* w) {
  if (check_handle(h) != CPG_OK || count < 0) return CPG_ERR_INVALID;
  {
    Status st = ready_graph(h);
    if (st != CPG_OK) return st;
  }
  if (count == 0) return CPG_OK;
  if (!eids || !w) return fail(h, CPG_ERR_INVALID, "null delay buffer");
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  // a relabelled graph stores the caller's edges at new positions
  std::vector<int32_t> mapped;
  if (!h->emap.empty()) {
    mapped.resize(static_cast<size_t>(count));
    for (int64_t i = 0; i < count; ++i) {
      const int32_t e = eids[i];
      if (e < 0 || e >= h->g.m) return fail(h, CPG_ERR_INVALID, "edge id out of range");
      mapped[i] = h->emap[e];
    }
    eids = mapped.data();
  }
  int32_t lowest = INT32_MAX;
  const bool have_levels = h->sfxt_valid || h->dirty_level > 0;
  if (have_levels) {
    Status st = ensure_levels_host(h);
    if (st != CPG_OK) return st;
  }
  // tail of each fan-out edge, by binary search over the CSR offsets
  for (int64_t i = 0; i < count; ++i) {
    const int32_t e = eids[i];
    if (e < 0 || e >= h->g.m) return fail(h, CPG_ERR_INVALID, "edge id out of range");
  }
  for (int64_t i = 0; have_levels && i < count; ++i) {
    const auto it = std::upper_bound(h->g.adjp.begin(), h->g.adjp.end(), eids[i]);
    const int32_t tail = static_cast<int32_t>(it - h->g.adjp.begin()) - 1;
    const int32_t lv = h->h_level_of[tail];
    if (lv < 0) continue;
    lowest = std::min(lowest, lv);
    if (h->multi_graph) {
      const size_t g = static_cast<size_t>(
          std::upper_bound(h->graph_voff.begin(), h->graph_voff.end(), tail) -
          h->graph_voff.begin() - 1);
      h->graph_from[g] = std::min(h->graph_from[g], lv);
    }
  }
  // staging kept by the handle: no allocation (and no device-wide
  // synchronisation) per update
  CK(ensure_grow(h->d_upd, static_cast<size_t>(count) * 8), "alloc delay update");
  int32_t* up_e = P<int32_t>(h->d_upd);
  float* up_w = reinterpret_cast<float*>(up_e + count);
  CK(cudaMemcpyAsync(up_e, eids, count * 4, cudaMemcpyHostToDevice, h->stream), "H2D eids");
  CK(cudaMemcpyAsync(up_w, w, count * 4, cudaMemcpyHostToDevice, h->stream), "H2D delays");
  CK(launch_scatter_delays(P<DevEdge>(h->d_edges), up_e, up_w, count, h->stream),
     "scatter delays");
  CK(cudaStreamSynchronize(h->stream), "scatter delays");
  // incremental rebuild from the lowest changed level (levels never change
  // with delays); without levels a full rebuild follows
  if (have_levels && lowest != INT32_MAX && lowest >= 1)
    h->dirty_level = h->dirty_level > 0 ? std::min(h->dirty_level, lowest) : lowest;
  else if (!(have_levels && lowest == INT32_MAX))
    h->dirty_level = -1;
  h->sfxt_valid = false;
  h->h_sfxt_cached = false;
  h->result_valid = false;
  return CPG_OK;
}

cpg_status cpg_get_sfxt(cpg_handle* h, int32_t* dist, int32_t* succ,
                        int32_t* level) {
  if (check_handle(h) != CPG_OK) return CPG_ERR_INVALID;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  Status st = ensure_sfxt(h);
  if (st != CPG_OK) return st;
  const size_t n = h->g.n;
  if (n == 0) return CPG_OK;
  if (dist) CK(cudaMemcpy(dist, h->d_dist.p, n * 4, cudaMemcpyDeviceToHost), "D2H dist");
  if (succ) CK(cudaMemcpy(succ, h->d_succ.p, n * 4, cudaMemcpyDeviceToHost), "D2H succ");
  if (level) CK(cudaMemcpy(level, h->d_level_of.p, n * 4, cudaMemcpyDeviceToHost), "D2H level");
  return CPG_OK;
}

int32_t cpg_num_levels(const cpg_handle* h) { return h ? h->levels : 0; }

cpg_status cpg_report_paths_batch(cpg_handle* const* handles, const int64_t* ks, int32_t n) {
  if (n < 0 || (n > 0 && (!handles || !ks))) return CPG_ERR_INVALID;
  cpg_status first = CPG_OK;
  for (int32_t i = 0; i < n; ++i) {
    const cpg_status st = cpg_report_paths(handles[i], ks[i]);
    if (st != CPG_OK && first == CPG_OK) first = st;
  }
  return first;
}

cpg_status cpg_report_paths(cpg_handle* h, int64_t k) {
  if (check_handle(h) != CPG_OK || k < 0) return CPG_ERR_INVALID;
  if (!h->has_graph) return fail(h, CPG_ERR_STATE, "no graph loaded");
  if (k > (int64_t{1} << 30)) return fail(h, CPG_ERR_INVALID, "k too large");
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  if (!h->sfxt_valid) h->stats.kernel_launches = 0;
  Status st = ensure_sfxt(h);
  if (st != CPG_OK) return st;
  h->result_valid = false;
  h->n_result = 0;
  h->stats.pending_peak = 0;
  h->stats.phases = 0;
  h->stats.rounds = 0;
  h->stats.retries = 0;
  if (k == 0) {
    h->result_valid = true;
    return CPG_OK;
  }
  const unsigned long long uk = static_cast<unsigned long long>(k);
  const unsigned long long nsrc = static_cast<unsigned long long>(h->n_srcs);
  h->cap_paths = std::max(h->cap_paths, std::max<unsigned long long>(4 * uk, 1 << 16) + nsrc);
  h->cap_front = std::max(h->cap_front, std::max<unsigned long long>(2 * uk, 1 << 16));
  h->cap_pend = std::max(h->cap_pend, std::max<unsigned long long>(8 * uk, 1 << 17) + nsrc);
  const bool host_stepped = h->opts.host_stepped == 1;
  for (int attempt = 0; attempt < 10; ++attempt) {
    const int r = host_stepped ? try_query(h, uk) : engine_query(h, uk);
    if (r == kRetry) {
      // a bounded pile overflowed: grow 4x while device memory allows (a tie
      // wall of equal-cost paths can need far more than K of them)
      h->stats.retries += 1;
      size_t free_b = 0, total_b = 0;
      cudaMemGetInfo(&free_b, &total_b);
      const size_t held = static_cast<size_t>(h->stats.bytes_reserved);
      const size_t next = 4 * held;
      if (next > held + free_b * 9 / 10) break;
      grow_caps(h);
      continue;
    }
    return static_cast<cpg_status>(r);
  }
  return fail(h, CPG_ERR_CAPACITY, "prefix tree buffers cannot grow further");
}

cpg_status cpg_get_costs(const cpg_handle* hc, int64_t k, float* out,
                         int64_t* n_out) {
  cpg_handle* h = const_cast<cpg_handle*>(hc);
  if (!h || k < 0) return CPG_ERR_INVALID;
  if (!h->result_valid) return fail(h, CPG_ERR_STATE, "no result");
  const int64_t n = std::min(k, h->n_result);
  if (n_out) *n_out = n;
  if (n > 0) {
    if (!out) return fail(h, CPG_ERR_INVALID, "null output");
    CK(cudaMemcpy(out, h->d_out_cost.p, n * 4, cudaMemcpyDeviceToHost), "D2H costs");
  }
  return CPG_OK;
}

cpg_status cpg_get_paths(const cpg_handle* hc, int64_t k, cpg_path_node* out,
                         int64_t* n_out) {
  cpg_handle* h = const_cast<cpg_handle*>(hc);
  if (!h || k < 0) return CPG_ERR_INVALID;
  if (!h->result_valid) return fail(h, CPG_ERR_STATE, "no result");
  const int64_t n = std::min(k, h->n_result);
  if (n_out) *n_out = n;
  if (n > 0) {
    if (!out) return fail(h, CPG_ERR_INVALID, "null output");
    CK(cudaMemcpy(out, h->d_out_nodes.p, n * sizeof(cpg_path_node), cudaMemcpyDeviceToHost), "D2H paths");
  }
  return CPG_OK;
}

cpg_status cpg_get_costs_device(const cpg_handle* h, const float** d_costs,
                                int64_t* n_out) {
  if (!h || !d_costs) return CPG_ERR_INVALID;
  if (!h->result_valid) return CPG_ERR_STATE;
  *d_costs = static_cast<const float*>(h->d_out_cost.p);
  if (n_out) *n_out = h->n_result;
  return CPG_OK;
}

cpg_status cpg_get_path_vertices(cpg_handle* h, int64_t i, int32_t* verts,
                                 int64_t cap, int64_t* len) {
  if (check_handle(h) != CPG_OK || i < 0 || cap < 0) return CPG_ERR_INVALID;
  if (!h->result_valid || i >= h->n_result) return fail(h, CPG_ERR_STATE, "no such result");
  Status st = cache_sfxt_host(h);
  if (st != CPG_OK) return st;
  unsigned int idx = 0;
  CK(cudaMemcpy(&idx, P<unsigned int>(h->d_vals) + h->sorted_vals_off + i, 4,
                cudaMemcpyDeviceToHost), "D2H index");
  // deviations from the leaf back to the root
  std::vector<std::pair<int32_t, int32_t>> devs;
  int32_t cur = static_cast<int32_t>(idx), src = -1;
  for (int guard = 0; guard < (1 << 24); ++guard) {
    int32_t par = 0, from = 0, to = 0;
    CK(cudaMemcpy(&par, P<int32_t>(h->d_pparent) + cur, 4, cudaMemcpyDeviceToHost), "D2H path");
    CK(cudaMemcpy(&from, P<int32_t>(h->d_pfrom) + cur, 4, cudaMemcpyDeviceToHost), "D2H path");
    CK(cudaMemcpy(&to, P<int32_t>(h->d_pto) + cur, 4, cudaMemcpyDeviceToHost), "D2H path");
    if (par < 0) {
      src = to;
      break;
    }
    devs.emplace_back(from, to);
    cur = par;
  }
  std::reverse(devs.begin(), devs.end());
  std::vector<int32_t> seq;
  int32_t v = src;
  size_t d = 0;
  while (v >= 0) {
    seq.push_back(v);
    if (d < devs.size() && devs[d].first == v) {
      v = devs[d].second;
      ++d;
    } else {
      v = h->h_succ[v];
    }
    if (seq.size() > static_cast<size_t>(h->g.n) + 1)
      return fail(h, CPG_ERR_STATE, "path walk did not terminate");
  }
  if (len) *len = static_cast<int64_t>(seq.size());
  if (verts) {
    const int64_t c = std::min<int64_t>(cap, seq.size());
    std::memcpy(verts, seq.data(), c * 4);
  }
  return CPG_OK;
}

cpg_status cpg_reset(cpg_handle* h) {
  if (check_handle(h) != CPG_OK) return CPG_ERR_INVALID;
  h->sfxt_valid = false;
  h->h_sfxt_cached = false;
  h->dirty_level = -1;
  h->result_valid = false;
  h->n_result = 0;
  h->stats = cpg_stats{};
  return CPG_OK;
}

cpg_status cpg_get_stats(const cpg_handle* h, cpg_stats* out) {
  if (!h || !out) return CPG_ERR_INVALID;
  *out = h->stats;
  return CPG_OK;
}

cpg_status cpg_sync(cpg_handle* h) {
  if (check_handle(h) != CPG_OK) return CPG_ERR_INVALID;
  CK(cudaStreamSynchronize(h->stream), "sync");
  return CPG_OK;
}

// ---------------------------------------------------------------- top-K

cpg_status cpg_select_topk(const float* d_costs, int64_t n, int64_t k, float* d_out,
                           int64_t* n_out, void* stream) {
  if (n < 0 || k < 0 || !n_out || (n > 0 && !d_costs) || (k > 0 && !d_out))
    return CPG_ERR_INVALID;
  *n_out = 0;
  if (n == 0 || k == 0) return CPG_OK;
  if (n > (int64_t{1} << 32) - 1 || k > (int64_t{1} << 31))
    return CPG_ERR_INVALID;
  const unsigned long long kk = static_cast<unsigned long long>(std::min(k, n));
  const size_t words = 2048 + 4 + 2 + 1 + 4 * kk + topk_sort_hist_words(kk) + 4;
  void* buf = nullptr;
  if (cudaMalloc(&buf, words * 4 + 64) != cudaSuccess) {
    cudaGetLastError();
    return CPG_ERR_OOM;
  }
  char* b = static_cast<char*>(buf);
  TopkScratch sc;
  sc.hist = reinterpret_cast<unsigned int*>(b);
  sc.state = b + 2048 * 4;
  sc.counts = reinterpret_cast<unsigned long long*>(b + 2048 * 4 + 16);
  sc.cnt = sc.counts + 2;
  sc.tkey = reinterpret_cast<unsigned int*>(sc.cnt + 2);
  sc.keys = sc.tkey + 4;
  sc.vals = sc.keys + 2 * kk;
  sc.sort_hist = sc.vals + 2 * kk;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(sc.hist, 0, 2048 * 4, s);
  unsigned long long got = 0;
  if (e == cudaSuccess)
    e = static_cast<cudaError_t>(launch_topk_costs(d_costs, static_cast<unsigned long long>(n),
                                                   kk, sc, d_out, &got, s));
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(buf);
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? CPG_ERR_OOM : CPG_ERR_CUDA;
  *n_out = static_cast<int64_t>(got);
  return CPG_OK;
}

// ---------------------------------------------------------------- batched form

struct cpg_dag {
  EdgeList el;
};

// message of the last failing host-side graph call on this thread
static std::string& dag_err() {
  static thread_local std::string e;
  return e;
}

struct cpg_batch {
  cpg_handle* h = nullptr;          // owns the side-by-side device graph
  std::string err;
  // graphs added so far, as one fan-out CSR
  std::vector<int32_t> adjp{0}, adj;
  std::vector<float> w;
  std::vector<int32_t> voff{0};     // first vertex of each graph
  bool committed = false;
  std::vector<int32_t> src_beg, src_end;  // per graph: its sources in d_srcs
  // the committed graph, relabelled in level order (what the device holds)
  std::vector<int32_t> padjp, padj;
  // queries
  std::vector<EngineQuery> qs;
  unsigned long long k_total = 0;
  std::vector<EngineQuery> qout;
  bool have_result = false;
  // the captured step
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int captured_rebuild = -1;        // rebuild flag of the captured graph
  bool prepared = false;
  cpg_batch_stats stats{};
};

namespace {

// Side-by-side graphs in level order.  Within each graph's id range the
// vertices are renumbered by (suffix-tree level, caller id): sinks are level
// 0, any other vertex one more than its highest head.  One level of the
// side-by-side graph is then one contiguous block per graph, so a build step
// reads and writes per-vertex words packed together instead of one DRAM burst
// per 4-byte word.  Rows keep their edge order.  A vertex on a cycle gets no
// level and goes last; the device build then reports the cycle.
struct LevelOrder {
  std::vector<int32_t> orig;        // new id -> caller id
  std::vector<int32_t> adjp, adj;   // the relabelled CSR
  std::vector<float> w;
  std::vector<int32_t> emap;        // caller edge position -> new edge position
};

void relabel_by_level(const std::vector<int32_t>& voff, const std::vector<int32_t>& adjp,
                      const std::vector<int32_t>& adj, const std::vector<float>& w,
                      LevelOrder& lo) {
  const int32_t n = voff.back();
  const size_t m = adj.size();
  const int ng = static_cast<int>(voff.size()) - 1;
  std::vector<int32_t> perm(static_cast<size_t>(n));
  lo.orig.assign(static_cast<size_t>(n), 0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int g = 0; g < ng; ++g) {
    const int32_t v0 = voff[g], nv = voff[g + 1] - voff[g];
    const int32_t e0 = adjp[v0], e1 = adjp[v0 + nv];
    // fan-in lists of the graph
    std::vector<int32_t> ip(static_cast<size_t>(nv) + 1, 0), iadj(static_cast<size_t>(e1 - e0));
    for (int32_t e = e0; e < e1; ++e) ++ip[adj[e] - v0 + 1];
    for (int32_t i = 0; i < nv; ++i) ip[i + 1] += ip[i];
    std::vector<int32_t> cur(ip.begin(), ip.end() - 1);
    for (int32_t i = 0; i < nv; ++i)
      for (int32_t e = adjp[v0 + i]; e < adjp[v0 + i + 1]; ++e) iadj[cur[adj[e] - v0]++] = i;
    // Kahn from the sinks: a vertex's level is final when its last head is done
    std::vector<int32_t> lvl(static_cast<size_t>(nv), -1), left(static_cast<size_t>(nv)), q;
    q.reserve(static_cast<size_t>(nv));
    for (int32_t i = 0; i < nv; ++i) {
      left[i] = adjp[v0 + i + 1] - adjp[v0 + i];
      if (left[i] == 0) {
        lvl[i] = 0;
        q.push_back(i);
      }
    }
    int32_t top = 0;
    for (size_t x = 0; x < q.size(); ++x) {
      const int32_t u = q[x];
      top = std::max(top, lvl[u]);
      for (int32_t j = ip[u]; j < ip[u + 1]; ++j) {
        const int32_t t = iadj[j];
        lvl[t] = std::max(lvl[t], lvl[u] + 1);
        if (--left[t] == 0) q.push_back(t);
      }
    }
    // stable counting sort by level (caller-id order within a level; no level last)
    std::vector<int32_t> at(static_cast<size_t>(top) + 3, 0);
    auto bucket = [&](int32_t i) { return lvl[i] >= 0 && left[i] == 0 ? lvl[i] : top + 1; };
    for (int32_t i = 0; i < nv; ++i) ++at[bucket(i) + 1];
    for (int32_t b = 0; b <= top + 1; ++b) at[b + 1] += at[b];
    for (int32_t i = 0; i < nv; ++i) {
      const int32_t pos = at[bucket(i)]++;
      perm[v0 + i] = v0 + pos;
      lo.orig[v0 + pos] = v0 + i;
    }
  }
  lo.adjp.assign(static_cast<size_t>(n) + 1, 0);
  for (int32_t v = 0; v < n; ++v) {
    const int32_t o = lo.orig[v];
    lo.adjp[v + 1] = lo.adjp[v] + (adjp[o + 1] - adjp[o]);
  }
  lo.adj.resize(m);
  lo.w.resize(m);
  lo.emap.resize(m);
#pragma omp parallel for schedule(static)
  for (int32_t v = 0; v < n; ++v) {
    const int32_t o = lo.orig[v];
    for (int32_t j = 0; j < adjp[o + 1] - adjp[o]; ++j) {
      const int32_t e = adjp[o] + j, f = lo.adjp[v] + j;
      lo.adj[f] = perm[adj[e]];
      lo.w[f] = w[e];
      lo.emap[e] = f;
    }
  }
}

void batch_drop_graph(cpg_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->captured_rebuild = -1;
}

Status batch_fail(cpg_batch* b, Status s, const std::string& msg) {
  b->err = msg;
  return s;
}

// Enqueue one step on the handle's stream (capturable).
Status batch_enqueue(cpg_batch* b, bool rebuild) {
  cpg_handle* h = b->h;
  int launches = 0;
  if (rebuild) {
    Status st = enqueue_sfxt(h, 0, &launches);
    if (st != CPG_OK) return st;
  }
  return engine_enqueue(h, static_cast<int>(b->qs.size()), b->k_total);
}

// Capture the step into a CUDA graph; on any capture error the step runs as
// plain launches instead (graph_captured = 0).
void batch_capture(cpg_batch* b, bool rebuild) {
  batch_drop_graph(b);
  cudaStream_t s = b->h->stream;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  const Status st = batch_enqueue(b, rebuild);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  if (st != CPG_OK || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return;
  }
  if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
    cudaGraphDestroy(g);
    b->exec = nullptr;
    cudaGetLastError();
    return;
  }
  b->graph = g;
  b->captured_rebuild = rebuild ? 1 : 0;
}

// One step with the current capacities.  kRetry on overflow.
int batch_step(cpg_batch* b, bool rebuild) {
  cpg_handle* h = b->h;
  cudaStream_t s = h->stream;
  if (!b->prepared) {
    Status st = engine_prepare(h, b->qs, b->k_total);
    if (st != CPG_OK) return st;
    b->prepared = true;
    batch_drop_graph(b);
  }
  if (b->captured_rebuild != (rebuild ? 1 : 0)) batch_capture(b, rebuild);
  CK(cudaEventRecord(h->ev[4], s), "event");
  if (b->exec) {
    CK(cudaGraphLaunch(b->exec, s), "graph launch");
  } else {
    Status st = batch_enqueue(b, rebuild);
    if (st != CPG_OK) return st;
  }
  CK(cudaEventRecord(h->ev[5], s), "event");
  if (rebuild) {
    const int r = finish_sfxt(h, 0);
    if (r == kRetry) {
      Status st = grow_heap_pool(h);
      if (st != CPG_OK) return st;
      batch_drop_graph(b);
      return kRetry;
    }
    if (r != CPG_OK) return r;
  }
  b->qout = b->qs;
  EngineCounters c;
  const int r = engine_finish(h, b->qout, c, b->k_total);
  if (r == kRetry) {
    b->prepared = false;
    return kRetry;
  }
  if (r != CPG_OK) return r;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev[4], h->ev[5]);
  b->stats.step_ms = ms;
  b->stats.sfxt_ms = 0.0;
  b->stats.paths_accepted = static_cast<int64_t>(c.paths);
  b->stats.phases = c.phases;
  b->stats.rounds = c.rounds;
  b->stats.graph_captured = b->exec ? 1 : 0;
  b->stats.bytes_reserved = h->stats.bytes_reserved;
  b->have_result = true;
  return CPG_OK;
}

}  // namespace

extern "C" {

cpg_status cpg_batch_create(cpg_batch** out, const cpg_options* opts) {
  if (!out) return CPG_ERR_INVALID;
  *out = nullptr;
  cpg_batch* b = new (std::nothrow) cpg_batch();
  if (!b) return CPG_ERR_OOM;
  const cpg_status st = cpg_create(&b->h, opts);
  if (st != CPG_OK) {
    delete b;
    return st;
  }
  *out = b;
  return CPG_OK;
}

cpg_status cpg_batch_destroy(cpg_batch* b) {
  if (!b) return CPG_ERR_INVALID;
  batch_drop_graph(b);
  if (b->h) cpg_destroy(b->h);
  delete b;
  return CPG_OK;
}

const char* cpg_batch_last_error(const cpg_batch* b) {
  if (!b) return "null batch";
  return b->err.empty() ? cpg_last_error(b->h) : b->err.c_str();
}

cpg_status cpg_batch_add_graph(cpg_batch* b, int32_t n, int32_t m, const int32_t* adjp,
                               const int32_t* adjncy, const float* w, int32_t* graph_id) {
  if (!b || n < 0 || m < 0 || !adjp || (m > 0 && (!adjncy || !w))) return CPG_ERR_INVALID;
  if (adjp[0] != 0 || adjp[n] != m)
    return batch_fail(b, CPG_ERR_INVALID, "CSR offsets must start at 0 and end at m");
  const int64_t base_v = b->voff.back();
  const int64_t base_e = static_cast<int64_t>(b->adj.size());
  if (base_v + n > INT32_MAX - 2 || base_e + m > INT32_MAX - 1)
    return batch_fail(b, CPG_ERR_CAPACITY, "batch exceeds 32-bit vertex or edge ids");
  for (int32_t v = 0; v < n; ++v) b->adjp.push_back(static_cast<int32_t>(base_e + adjp[v + 1]));
  for (int32_t e = 0; e < m; ++e) {
    if (adjncy[e] < 0 || adjncy[e] >= n)
      return batch_fail(b, CPG_ERR_INVALID, "edge head out of range");
    b->adj.push_back(static_cast<int32_t>(base_v + adjncy[e]));
  }
  b->w.insert(b->w.end(), w, w + m);
  b->voff.push_back(static_cast<int32_t>(base_v + n));
  if (graph_id) *graph_id = static_cast<int32_t>(b->voff.size() - 2);
  b->committed = false;
  return CPG_OK;
}

cpg_status cpg_batch_add_dag(cpg_batch* b, const cpg_dag* d, int32_t* graph_id) {
  if (!b || !d) return CPG_ERR_INVALID;
  HostGraph g;
  std::string err;
  Status st = edges_to_csr(d->el, g, err);
  if (st != CPG_OK) return batch_fail(b, st, err);
  return cpg_batch_add_graph(b, g.n, g.m, g.adjp.data(), g.adj.data(), g.w.data(), graph_id);
}

cpg_status cpg_batch_commit(cpg_batch* b) {
  if (!b) return CPG_ERR_INVALID;
  cpg_handle* h = b->h;
  const int32_t n = b->voff.back();
  // each graph relabelled in level order (invisible to the caller: the batch
  // returns costs, the successor tie-break and the root order use caller ids,
  // delay updates name the caller's edges)
  LevelOrder lo;
  if (h->opts.batch_caller_order == 1) {
    lo.orig.resize(static_cast<size_t>(n));
    for (int32_t v = 0; v < n; ++v) lo.orig[v] = v;
    lo.adjp = b->adjp;
    lo.adj = b->adj;
    lo.w = b->w;
  } else {
    relabel_by_level(b->voff, b->adjp, b->adj, b->w, lo);
  }
  Status st = upload_graph(h, n, static_cast<int32_t>(lo.adj.size()), lo.adjp.data(),
                           lo.adj.data(), lo.w.data());
  if (st != CPG_OK) return st;
  CK(ensure(h->d_orig_id, std::max<size_t>(lo.orig.size(), 1) * 4), "alloc caller ids");
  if (n) CK(cudaMemcpy(h->d_orig_id.p, lo.orig.data(), lo.orig.size() * 4, cudaMemcpyHostToDevice),
            "H2D caller ids");
  h->relabeled = h->opts.batch_caller_order != 1;
  h->emap.swap(lo.emap);
  // sources of each graph: a contiguous run of the id-sorted source list
  std::vector<int32_t> srcs(h->n_srcs);
  if (h->n_srcs)
    CK(cudaMemcpy(srcs.data(), h->d_srcs.p, srcs.size() * 4, cudaMemcpyDeviceToHost), "D2H sources");
  const size_t ng = b->voff.size() - 1;
  b->src_beg.assign(ng, 0);
  b->src_end.assign(ng, 0);
  for (size_t g = 0; g < ng; ++g) {
    b->src_beg[g] = static_cast<int32_t>(
        std::lower_bound(srcs.begin(), srcs.end(), b->voff[g]) - srcs.begin());
    b->src_end[g] = static_cast<int32_t>(
        std::lower_bound(srcs.begin(), srcs.end(), b->voff[g + 1]) - srcs.begin());
    // within a graph, roots are seeded in caller-id order (gpucpg.cu:531-533)
    std::sort(srcs.begin() + b->src_beg[g], srcs.begin() + b->src_end[g],
              [&](int32_t a, int32_t c) { return lo.orig[a] < lo.orig[c]; });
  }
  if (h->n_srcs > 1)
    CK(cudaMemcpy(h->d_srcs.p, srcs.data(), srcs.size() * 4, cudaMemcpyHostToDevice), "H2D sources");
  b->padjp.swap(lo.adjp);
  b->padj.swap(lo.adj);
  // per-vertex graph ids for incremental rebuilds of single graphs
  h->multi_graph = true;
  h->graph_voff = b->voff;
  h->graph_from.assign(ng, INT32_MAX);
  {
    std::vector<int32_t> vg(static_cast<size_t>(n));
    for (size_t g = 0; g < ng; ++g)
      std::fill(vg.begin() + b->voff[g], vg.begin() + b->voff[g + 1], static_cast<int32_t>(g));
    CK(ensure(h->d_vgraph, std::max<size_t>(vg.size(), 1) * 4), "alloc graph ids");
    CK(ensure(h->d_graph_from, std::max<size_t>(ng, 1) * 4), "alloc graph ids");
    if (n)
      CK(cudaMemcpy(h->d_vgraph.p, vg.data(), vg.size() * 4, cudaMemcpyHostToDevice), "H2D graph ids");
  }
  b->committed = true;
  b->prepared = false;
  batch_drop_graph(b);
  return CPG_OK;
}

cpg_status cpg_batch_set_queries(cpg_batch* b, int32_t nq, const int32_t* graph_ids,
                                 const int64_t* ks) {
  if (!b || nq <= 0 || !graph_ids || !ks) return CPG_ERR_INVALID;
  if (!b->committed) return batch_fail(b, CPG_ERR_STATE, "commit the graphs first");
  if (nq > kMaxQueries) return batch_fail(b, CPG_ERR_CAPACITY, "more than 4096 queries");
  const int32_t ng = static_cast<int32_t>(b->voff.size() - 1);
  std::vector<EngineQuery> qs(nq);
  unsigned long long tot = 0;
  for (int32_t i = 0; i < nq; ++i) {
    if (graph_ids[i] < 0 || graph_ids[i] >= ng || ks[i] < 0 || ks[i] > (int64_t{1} << 30))
      return batch_fail(b, CPG_ERR_INVALID, "bad query");
    qs[i] = EngineQuery{};
    qs[i].k = ks[i];
    qs[i].src_beg = b->src_beg[graph_ids[i]];
    qs[i].src_end = b->src_end[graph_ids[i]];
    tot += static_cast<unsigned long long>(ks[i]);
  }
  if (tot > (1ull << 31)) return batch_fail(b, CPG_ERR_CAPACITY, "sum of k above 2^31");
  b->qs.swap(qs);
  b->k_total = tot ? tot : 1;
  cpg_handle* h = b->h;
  h->cap_paths = std::max<unsigned long long>(4 * b->k_total, 1 << 16) + h->n_srcs;
  h->cap_front = std::max<unsigned long long>(2 * b->k_total, 1 << 16);
  h->cap_pend = std::max<unsigned long long>(8 * b->k_total, 1 << 17) + h->n_srcs;
  b->prepared = false;
  b->have_result = false;
  return CPG_OK;
}

cpg_status cpg_batch_run(cpg_batch* b, int32_t rebuild_sfxt) {
  if (!b) return CPG_ERR_INVALID;
  if (b->qs.empty()) return batch_fail(b, CPG_ERR_STATE, "no queries set");
  cpg_handle* h = b->h;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  bool rebuild = rebuild_sfxt != 0 || !h->sfxt_valid;
  b->stats.retries = 0;
  for (int attempt = 0; attempt < 10; ++attempt) {
    const int r = batch_step(b, rebuild);
    if (r == kRetry) {
      b->stats.retries += 1;
      size_t free_b = 0, total_b = 0;
      cudaMemGetInfo(&free_b, &total_b);
      const size_t held = static_cast<size_t>(h->stats.bytes_reserved);
      if (4 * held > held + free_b * 9 / 10) break;
      grow_caps(h);
      b->prepared = false;
      rebuild = true;
      continue;
    }
    return static_cast<cpg_status>(r);
  }
  return batch_fail(b, CPG_ERR_CAPACITY, "batch buffers cannot grow further");
}

cpg_status cpg_batch_get_costs(const cpg_batch* bc, int32_t q, float* out, int64_t cap,
                               int64_t* n_out) {
  cpg_batch* b = const_cast<cpg_batch*>(bc);
  if (!b || q < 0 || cap < 0) return CPG_ERR_INVALID;
  if (!b->have_result || q >= static_cast<int32_t>(b->qout.size()))
    return batch_fail(b, CPG_ERR_STATE, "no result for that query");
  cpg_handle* h = b->h;
  const EngineQuery& Q = b->qout[q];
  const int64_t n = std::min<int64_t>(cap, static_cast<int64_t>(Q.k_out));
  if (n_out) *n_out = static_cast<int64_t>(Q.k_out) < cap ? static_cast<int64_t>(Q.k_out) : cap;
  if (n > 0) {
    if (!out) return CPG_ERR_INVALID;
    CK(cudaMemcpy(out, P<float>(h->d_out_cost) + Q.out_off, n * 4, cudaMemcpyDeviceToHost),
       "D2H costs");
  }
  return CPG_OK;
}

cpg_status cpg_batch_get_stats(const cpg_batch* b, cpg_batch_stats* out) {
  if (!b || !out) return CPG_ERR_INVALID;
  *out = b->stats;
  out->sfxt_ctas_per_sm = b->h->sfxt_grid_limit;
  out->engine_ctas_per_sm = b->h->engine_grid_limit;
  out->select_schedule = b->h->sel_schedule;
  out->sfxt_mode = b->h->opts.sfxt_level_sync == 1 ? 2 : (b->h->opts.sfxt_late_push == 1 ? 1 : 0);
  out->frontier_used = b->h->use_bvss ? CPG_FRONTIER_BVSS : CPG_FRONTIER_CSR;
  out->bvss_tiles = b->h->opts.bvss_tiles;
  return CPG_OK;
}

cpg_status cpg_batch_autotune(cpg_batch* b) {
  if (!b) return CPG_ERR_INVALID;
  if (b->qs.empty()) return batch_fail(b, CPG_ERR_STATE, "no queries set");
  cpg_handle* h = b->h;
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device), "attribute");
  // The BVSS frontier is a candidate only when its slices are dense enough
  // to have a chance; it is built once, from the host CSR, when it is.
  const bool try_bvss = h->use_bvss || h->bvss_bps >= 1.5 ||
                        bvss_density_sample(b->voff.back(), b->padjp.data(), b->padj.data(), 4096) >= 1.5;
  if (try_bvss && !h->use_bvss) {
    const int32_t keep = h->opts.frontier;
    h->opts.frontier = CPG_FRONTIER_BVSS;
    Status st = setup_bvss(h, b->voff.back(), b->padjp.data(), b->padj.data());
    h->opts.frontier = keep;
    if (st != CPG_OK) return static_cast<cpg_status>(st);
    h->use_bvss = false;  // built; each candidate below turns it on or off
  }
  struct Cand {
    int sfxt, engine, sched, mode, bvss, tiles;
  };
  std::vector<Cand> cands = {{0, 0, 0, 0, 0, 0}, {0, 0, 1, 0, 0, 0}, {sms / 2, 0, 0, 0, 0, 0},
                             {0, sms / 2, 0, 0, 0, 0}, {sms / 2, sms / 2, 0, 0, 0, 0},
                             {0, 0, 0, 1, 0, 0}, {0, 0, 0, 2, 0, 0}};
  if (try_bvss)
    for (int t = 0; t < 3; ++t) cands.push_back({0, 0, 0, 2, 1, t});
  auto apply = [&](const Cand& c) {
    h->sfxt_grid_limit = c.sfxt;
    h->engine_grid_limit = c.engine;
    h->sel_schedule = c.sched;
    h->opts.sfxt_late_push = c.mode == 1;
    h->opts.sfxt_level_sync = c.mode == 2;
    h->use_bvss = c.bvss != 0;
    h->opts.bvss_tiles = c.tiles;
    b->prepared = false;  // sort scratch depends on the engine grid
    batch_drop_graph(b);
  };
  double best = 1e30;
  Cand pick = cands[0];
  for (const Cand& c : cands) {
    apply(c);
    cpg_status st = cpg_batch_run(b, 1);
    if (st != CPG_OK) return st;
    double t = 0;
    for (int i = 0; i < 2; ++i) {
      st = cpg_batch_run(b, 1);
      if (st != CPG_OK) return st;
      t += b->stats.step_ms;
    }
    if (t < best) {
      best = t;
      pick = c;
    }
  }
  apply(pick);
  b->stats.tuned_candidates = static_cast<int32_t>(cands.size());
  return CPG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- served form

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Predicted device bytes of one query of k paths: path store, frontier and
// pending piles, sort buffers and outputs at the engine's initial sizing.
// Paths the server's piles are sized for at start (see cpg_server_start).
constexpr unsigned long long kServerPresizePaths = 4ull << 20;

int64_t predicted_bytes(int64_t k) {
  const int64_t kk = std::max<int64_t>(k, 1);
  return 4 * kk * 24 + 4 * kk * 16 + 16 * kk * 16 + 6 * kk * 4 + kk * 28 + (64 << 10);
}

struct ServerReq {
  int64_t ticket;
  int32_t graph;
  int64_t k;
  std::vector<int32_t> eids;  // union edge ids
  std::vector<float> w;
  double t_submit;
};

struct ServerResult {
  std::vector<float> costs;
  double latency_ms = 0;
  Status status = CPG_OK;
  bool done = false;
};

}  // namespace

struct cpg_server {
  cpg_batch* b = nullptr;
  cpg_server_options so{};
  std::string err;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<ServerReq> queue;
  std::unordered_map<int64_t, ServerResult> results;
  int64_t next_ticket = 0;
  bool running = false, stopping = false;
  // statistics
  std::vector<double> lat_ms;
  int64_t paths = 0, launches = 0, rebuilds = 0, retries = 0, pool_rebuilds = 0;
  double busy_ms = 0, sfxt_ms = 0, first_submit = -1, last_done = 0, max_step_ms = 0;
  double max_update_ms = 0, max_rebuild_ms = 0, max_launch_ms = 0, max_engine_ms = 0;
  int32_t max_batch_seen = 0;
  int64_t loop_allocs = 0;  // allocations made inside the request loop
  // pinned staging of a launch's costs (grown geometrically, kept): one fast
  // copy from the device, one copy into the results
  float* pin_out = nullptr;
  size_t pin_cap = 0;
};

namespace {

// One engine launch over the admitted queries.  Returns kRetry on overflow.
int server_launch(cpg_server* sv, const std::vector<ServerReq>& batch,
                  std::vector<std::vector<float>>& out) {
  cpg_batch* b = sv->b;
  cpg_handle* h = b->h;
  std::vector<EngineQuery> qs(batch.size());
  unsigned long long k_total = 0;
  for (size_t i = 0; i < batch.size(); ++i) {
    qs[i] = EngineQuery{};
    qs[i].k = batch[i].k;
    qs[i].src_beg = b->src_beg[batch[i].graph];
    qs[i].src_end = b->src_end[batch[i].graph];
    k_total += static_cast<unsigned long long>(batch[i].k);
  }
  if (k_total == 0) k_total = 1;
  h->cap_paths = std::max<unsigned long long>(h->cap_paths, std::max<unsigned long long>(4 * k_total, 1 << 16) + h->n_srcs);
  h->cap_front = std::max<unsigned long long>(h->cap_front, std::max<unsigned long long>(2 * k_total, 1 << 16));
  h->cap_pend = std::max<unsigned long long>(h->cap_pend, std::max<unsigned long long>(8 * k_total, 1 << 17) + h->n_srcs);
  Status st = engine_prepare(h, qs, k_total);
  if (st != CPG_OK) return st;
  cudaStream_t s = h->stream;
  CK(cudaEventRecord(h->ev[4], s), "event");
  st = engine_enqueue(h, static_cast<int>(qs.size()), k_total);
  if (st != CPG_OK) return st;
  CK(cudaEventRecord(h->ev[5], s), "event");
  EngineCounters c;
  const int r = engine_finish(h, qs, c, k_total);
  if (r != CPG_OK) return r;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev[4], h->ev[5]);
  sv->busy_ms += ms;
  sv->max_engine_ms = std::max(sv->max_engine_ms, static_cast<double>(ms));
  sv->launches += 1;
  // all outputs in one copy into the pinned staging, then split per query
  unsigned long long total = 0;
  for (const EngineQuery& q : qs) total = std::max(total, q.out_off + q.k_out);
  if (total > sv->pin_cap) {
    if (sv->pin_out) cudaFreeHost(sv->pin_out);
    sv->pin_out = nullptr;
    const size_t want = std::max<size_t>(total, 2 * sv->pin_cap);
    if (cudaMallocHost(&sv->pin_out, want * 4) != cudaSuccess) {
      sv->pin_out = nullptr;
      sv->pin_cap = 0;
      cudaGetLastError();
      return fail(h, CPG_ERR_OOM, "pinned staging of the costs");
    }
    ++t_allocs;
    sv->pin_cap = want;
  }
  if (total) {
    CK(cudaMemcpyAsync(sv->pin_out, h->d_out_cost.p, total * 4, cudaMemcpyDeviceToHost, s),
       "D2H costs");
    CK(cudaStreamSynchronize(s), "D2H costs");
  }
  out.resize(qs.size());
  for (size_t i = 0; i < qs.size(); ++i)
    out[i].assign(sv->pin_out + qs[i].out_off, sv->pin_out + qs[i].out_off + qs[i].k_out);
  return CPG_OK;
}

void server_loop(cpg_server* sv) {
  cpg_handle* h = sv->b->h;
  cudaSetDevice(h->device);
  for (;;) {
    std::vector<ServerReq> batch;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->cv_work.wait(lk, [&] { return sv->stopping || !sv->queue.empty(); });
      if (sv->queue.empty()) break;  // stopping and drained
      // Admit in arrival order, up to max_batch queries whose predicted
      // footprint fits the budget.  Delay updates are applied before the
      // launch, so an update joins only if no admitted query reads its
      // graph; otherwise it waits for the next launch, and so does every
      // later request on that graph (a graph's requests keep their order),
      // while requests on other graphs behind it are still admitted.
      const size_t max_batch = static_cast<size_t>(std::max(1, sv->so.max_batch));
      const size_t window = 4 * max_batch;
      int64_t used = 0;
      std::vector<char> graph_read(sv->b->voff.size(), 0), blocked(sv->b->voff.size(), 0);
      for (size_t i = 0; i < sv->queue.size() && i < window && batch.size() < max_batch;) {
        ServerReq& r = sv->queue[i];
        if (blocked[r.graph] || (!r.eids.empty() && graph_read[r.graph])) {
          blocked[r.graph] = 1;
          ++i;
          continue;
        }
        const int64_t need = predicted_bytes(r.k);
        if (!batch.empty() && sv->so.hbm_budget_bytes > 0 && used + need > sv->so.hbm_budget_bytes)
          break;
        used += need;
        graph_read[r.graph] = 1;
        batch.push_back(std::move(r));
        sv->queue.erase(sv->queue.begin() + static_cast<std::ptrdiff_t>(i));
      }
    }
    const double t_step = now_s();
    const int64_t pool_before = h->pool_rebuilds;
    const int64_t allocs_before = t_allocs;
    Status st = CPG_OK;
    bool updated = false;
    for (const ServerReq& r : batch) {
      if (r.eids.empty() || st != CPG_OK) continue;
      st = cpg_update_delays(h, static_cast<int64_t>(r.eids.size()), r.eids.data(), r.w.data());
      updated = true;
    }
    const double t_upd = now_s();
    if (st == CPG_OK && updated) {
      st = ensure_sfxt(h);  // incremental: levels at or above the lowest change
      sv->rebuilds += 1;
      sv->sfxt_ms += h->stats.sfxt_ms;
    }
    const double t_sfxt = now_s();
    std::vector<std::vector<float>> out;
    for (int attempt = 0; st == CPG_OK && attempt < 10; ++attempt) {
      const int r = server_launch(sv, batch, out);
      if (r == kRetry) {
        grow_caps(h);
        sv->retries += 1;
        continue;
      }
      st = static_cast<Status>(r);
      break;
    }
    const double t = now_s();
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->max_batch_seen = std::max<int32_t>(sv->max_batch_seen, static_cast<int32_t>(batch.size()));
      sv->max_step_ms = std::max(sv->max_step_ms, (t - t_step) * 1e3);
      sv->max_update_ms = std::max(sv->max_update_ms, (t_upd - t_step) * 1e3);
      sv->max_rebuild_ms = std::max(sv->max_rebuild_ms, (t_sfxt - t_upd) * 1e3);
      sv->max_launch_ms = std::max(sv->max_launch_ms, (t - t_sfxt) * 1e3);
      sv->pool_rebuilds += h->pool_rebuilds - pool_before;
      sv->loop_allocs += t_allocs - allocs_before;
      for (size_t i = 0; i < batch.size(); ++i) {
        ServerResult& res = sv->results[batch[i].ticket];
        res.status = st;
        if (st == CPG_OK && i < out.size()) {
          res.costs = std::move(out[i]);
          sv->paths += static_cast<int64_t>(res.costs.size());
        }
        res.latency_ms = (t - batch[i].t_submit) * 1e3;
        res.done = true;
        sv->lat_ms.push_back(res.latency_ms);
      }
      sv->last_done = t;
      if (st != CPG_OK) sv->err = cpg_last_error(h);
    }
    sv->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

void cpg_server_options_init(cpg_server_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->max_batch = 256;
  o->hbm_budget_bytes = 150ll << 30;
}

cpg_status cpg_server_create(cpg_server** out, const cpg_options* opts,
                             const cpg_server_options* sopts) {
  if (!out) return CPG_ERR_INVALID;
  *out = nullptr;
  cpg_server* sv = new (std::nothrow) cpg_server();
  if (!sv) return CPG_ERR_OOM;
  if (sopts) sv->so = *sopts;
  else cpg_server_options_init(&sv->so);
  const cpg_status st = cpg_batch_create(&sv->b, opts);
  if (st != CPG_OK) {
    delete sv;
    return st;
  }
  *out = sv;
  return CPG_OK;
}

cpg_status cpg_server_stop(cpg_server* sv) {
  if (!sv) return CPG_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stopping = true;
  }
  sv->cv_work.notify_all();
  if (sv->th.joinable()) sv->th.join();
  sv->running = false;
  return CPG_OK;
}

cpg_status cpg_server_destroy(cpg_server* sv) {
  if (!sv) return CPG_ERR_INVALID;
  cpg_server_stop(sv);
  if (sv->pin_out) cudaFreeHost(sv->pin_out);
  if (sv->b) cpg_batch_destroy(sv->b);
  delete sv;
  return CPG_OK;
}

const char* cpg_server_last_error(const cpg_server* sv) {
  if (!sv) return "null server";
  return sv->err.empty() ? cpg_batch_last_error(sv->b) : sv->err.c_str();
}

cpg_status cpg_server_add_graph(cpg_server* sv, int32_t n, int32_t m, const int32_t* adjp,
                                const int32_t* adjncy, const float* w, int32_t* graph_id) {
  if (!sv || sv->running) return CPG_ERR_INVALID;
  return cpg_batch_add_graph(sv->b, n, m, adjp, adjncy, w, graph_id);
}

cpg_status cpg_server_add_dag(cpg_server* sv, const cpg_dag* d, int32_t* graph_id) {
  if (!sv || sv->running) return CPG_ERR_INVALID;
  return cpg_batch_add_dag(sv->b, d, graph_id);
}

cpg_status cpg_server_start(cpg_server* sv) {
  if (!sv || sv->running) return CPG_ERR_INVALID;
  cpg_status st = cpg_batch_commit(sv->b);
  if (st != CPG_OK) return st;
  st = cpg_levelize(sv->b->h);
  if (st != CPG_OK) return st;
  // The engine's path and item piles, sized once for a launch answering
  // kServerPresizePaths paths (about 1.7 GB at 4 M; less under a smaller
  // admission budget), and allocated here with the tables of max_batch
  // queries and the pinned cost staging.  Growing a pile mid-stream
  // reallocates it and reruns the launch, and an allocation in the loop
  // stalls every query queued behind it: those steps set the tail latency.
  {
    cpg_handle* h = sv->b->h;
    unsigned long long pre = kServerPresizePaths;
    if (sv->so.hbm_budget_bytes > 0)
      pre = std::min<unsigned long long>(
          pre, static_cast<unsigned long long>(sv->so.hbm_budget_bytes) / (8 * 512));
    const unsigned long long ns = static_cast<unsigned long long>(h->n_srcs);
    // engine_prepare sizes the piles from the handle's capacities; if it
    // fails they go back to what they were, so a later start or batch call
    // does not retry the same oversized growth
    const unsigned long long old_paths = h->cap_paths, old_front = h->cap_front,
                             old_pend = h->cap_pend;
    h->cap_paths = std::max(h->cap_paths, 4 * pre + ns);
    h->cap_front = std::max(h->cap_front, 2 * pre);
    h->cap_pend = std::max(h->cap_pend, 8 * pre + ns);
    const std::vector<EngineQuery> none(static_cast<size_t>(std::max(1, sv->so.max_batch)));
    const Status ws = engine_prepare(h, none, pre);
    if (ws != CPG_OK) {
      h->cap_paths = old_paths;
      h->cap_front = old_front;
      h->cap_pend = old_pend;
      sv->err = cpg_last_error(h);
      return static_cast<cpg_status>(ws);
    }
    // the delay-update staging, for a request that re-samples every edge of
    // the largest graph
    size_t max_edges = 1;
    const cpg_batch* b = sv->b;
    for (size_t g = 0; g + 1 < b->voff.size(); ++g)
      max_edges = std::max<size_t>(
          max_edges, static_cast<size_t>(b->adjp[b->voff[g + 1]] - b->adjp[b->voff[g]]));
    CK(ensure_grow(h->d_upd, max_edges * 8), "alloc delay update");
    if (!sv->pin_out) {
      if (cudaMallocHost(&sv->pin_out, pre * 4) == cudaSuccess) {
        sv->pin_cap = pre;
      } else {
        sv->pin_out = nullptr;  // the loop allocates it when first needed
        cudaGetLastError();
      }
    }
  }
  sv->stopping = false;
  sv->running = true;
  sv->th = std::thread(server_loop, sv);
  return CPG_OK;
}

cpg_status cpg_server_submit(cpg_server* sv, int32_t graph_id, int64_t k, int32_t n_updates,
                             const int32_t* eids, const float* w, int64_t* ticket) {
  if (!sv || !ticket || k < 0 || n_updates < 0 || (n_updates > 0 && (!eids || !w)))
    return CPG_ERR_INVALID;
  if (!sv->running) return CPG_ERR_STATE;
  cpg_batch* b = sv->b;
  const int32_t ng = static_cast<int32_t>(b->voff.size() - 1);
  if (graph_id < 0 || graph_id >= ng || k > (int64_t{1} << 30)) return CPG_ERR_INVALID;
  ServerReq r;
  r.graph = graph_id;
  r.k = k;
  const int32_t e0 = b->adjp[b->voff[graph_id]];
  const int32_t e1 = b->adjp[b->voff[graph_id + 1]];
  r.eids.reserve(n_updates);
  for (int32_t i = 0; i < n_updates; ++i) {
    if (eids[i] < 0 || e0 + eids[i] >= e1) return CPG_ERR_INVALID;
    r.eids.push_back(e0 + eids[i]);
  }
  r.w.assign(w, w + n_updates);
  r.t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    r.ticket = sv->next_ticket++;
    *ticket = r.ticket;
    if (sv->first_submit < 0) sv->first_submit = r.t_submit;
    sv->results[r.ticket] = ServerResult{};
    sv->queue.push_back(std::move(r));
  }
  sv->cv_work.notify_one();
  return CPG_OK;
}

cpg_status cpg_server_wait(cpg_server* sv, int64_t ticket, float* out, int64_t cap,
                           int64_t* n_out, double* latency_ms, int32_t timeout_ms) {
  if (!sv || cap < 0) return CPG_ERR_INVALID;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->results.find(ticket);
  if (it == sv->results.end()) return CPG_ERR_INVALID;
  auto ready = [&] { return sv->results[ticket].done; };
  if (timeout_ms < 0) {
    sv->cv_done.wait(lk, ready);
  } else if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return CPG_ERR_TIMEOUT;
  }
  ServerResult res = std::move(sv->results[ticket]);
  sv->results.erase(ticket);
  if (res.status != CPG_OK) return res.status;
  const int64_t n = std::min<int64_t>(cap, static_cast<int64_t>(res.costs.size()));
  if (n > 0 && out) std::memcpy(out, res.costs.data(), n * 4);
  if (n_out) *n_out = n;
  if (latency_ms) *latency_ms = res.latency_ms;
  return CPG_OK;
}

cpg_status cpg_server_get_stats(const cpg_server* svc, cpg_server_stats* out) {
  cpg_server* sv = const_cast<cpg_server*>(svc);
  if (!sv || !out) return CPG_ERR_INVALID;
  std::lock_guard<std::mutex> lk(sv->mu);
  *out = cpg_server_stats{};
  std::vector<double> l = sv->lat_ms;
  std::sort(l.begin(), l.end());
  out->completed = static_cast<int64_t>(l.size());
  out->paths = sv->paths;
  if (!l.empty()) {
    auto q = [&](double f) {
      const size_t i = std::min(l.size() - 1, static_cast<size_t>(std::ceil(f * l.size())) - 1);
      return l[i];
    };
    out->p50_ms = q(0.50);
    out->p99_ms = q(0.99);
    double sum = 0;
    for (double x : l) sum += x;
    out->mean_ms = sum / l.size();
    out->max_ms = l.back();
  }
  out->wall_s = sv->first_submit >= 0 ? sv->last_done - sv->first_submit : 0;
  out->paths_per_s = out->wall_s > 0 ? sv->paths / out->wall_s : 0;
  out->launches = sv->launches;
  out->sfxt_rebuilds = sv->rebuilds;
  out->busy_ms = sv->busy_ms;
  out->max_batch_seen = sv->max_batch_seen;
  out->sfxt_ms = sv->sfxt_ms;
  out->retries = sv->retries;
  out->pool_rebuilds = sv->pool_rebuilds;
  out->max_step_ms = sv->max_step_ms;
  out->max_update_ms = sv->max_update_ms;
  out->max_rebuild_ms = sv->max_rebuild_ms;
  out->max_launch_ms = sv->max_launch_ms;
  out->max_engine_ms = sv->max_engine_ms;
  out->loop_allocs = sv->loop_allocs;
  return CPG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- generator


void cpg_gen_params_init(cpg_gen_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->seed = 1;
  p->n_pins = 20000;
  p->n_levels = 60;
  p->n_first = 64;
  p->n_last = 64;
  p->level_span = 3;
  p->degree_kind = 0;
  p->deg_lo = 1;
  p->deg_hi = 4;
  p->deg_mean = 20.0;
  p->deg_cap = 256;
  p->weight_kind = 0;
  p->w_lo = 0.1f;
  p->w_hi = 10.0f;
  p->iw_lo = 1;
  p->iw_hi = 100;
  p->add_virtual = 1;
}

cpg_status cpg_dag_generate(const cpg_gen_params* p, cpg_dag** out) {
  if (!p || !out) return CPG_ERR_INVALID;
  cpg_dag* d = new (std::nothrow) cpg_dag();
  if (!d) return CPG_ERR_OOM;
  Status st = generate_dag(*p, d->el, dag_err());
  if (st != CPG_OK) {
    delete d;
    return st;
  }
  *out = d;
  return CPG_OK;
}

cpg_status cpg_dag_sizes(const cpg_dag* d, int32_t* n, int32_t* m) {
  if (!d) return CPG_ERR_INVALID;
  if (n) *n = d->el.n;
  if (m) *m = static_cast<int32_t>(d->el.src.size());
  return CPG_OK;
}

cpg_status cpg_dag_edges(const cpg_dag* d, int32_t* src, int32_t* dst, float* w) {
  if (!d) return CPG_ERR_INVALID;
  const size_t m = d->el.src.size();
  if (src) std::memcpy(src, d->el.src.data(), m * 4);
  if (dst) std::memcpy(dst, d->el.dst.data(), m * 4);
  if (w) std::memcpy(w, d->el.w.data(), m * 4);
  return CPG_OK;
}

cpg_status cpg_dag_read_text(const char* path, int32_t ignore_wgts, cpg_dag** out) {
  if (!path || !out) {
    dag_err() = "null argument";
    return CPG_ERR_INVALID;
  }
  cpg_dag* d = new (std::nothrow) cpg_dag();
  if (!d) return CPG_ERR_OOM;
  Status st = read_text_graph(path, ignore_wgts != 0, d->el, dag_err());
  if (st != CPG_OK) {
    delete d;
    return st;
  }
  *out = d;
  return CPG_OK;
}

cpg_status cpg_dag_read_csr_bin(const char* path, cpg_dag** out) {
  if (!path || !out) {
    dag_err() = "null argument";
    return CPG_ERR_INVALID;
  }
  HostGraph g;
  Status st = read_csr_bin(path, g, dag_err());
  if (st != CPG_OK) return st;
  cpg_dag* d = new (std::nothrow) cpg_dag();
  if (!d) return CPG_ERR_OOM;
  d->el.n = g.n;
  d->el.src.resize(static_cast<size_t>(g.m));
  for (int32_t v = 0; v < g.n; ++v)
    std::fill(d->el.src.begin() + g.adjp[v], d->el.src.begin() + g.adjp[v + 1], v);
  d->el.dst = std::move(g.adj);
  d->el.w = std::move(g.w);
  *out = d;
  return CPG_OK;
}

cpg_status cpg_dag_write_csr_bin(const cpg_dag* d, const char* path) {
  if (!d || !path) return CPG_ERR_INVALID;
  HostGraph g;
  Status st = edges_to_csr(d->el, g, dag_err());
  if (st != CPG_OK) return st;
  return write_csr_bin(g.n, g.m, g.adjp.data(), g.adj.data(), g.w.data(), path, dag_err());
}

const char* cpg_dag_last_error(void) { return dag_err().c_str(); }

cpg_status cpg_dag_write_text(const cpg_dag* d, const char* path) {
  if (!d || !path) return CPG_ERR_INVALID;
  return write_text_graph(d->el, path, dag_err());
}

cpg_status cpg_load_dag(cpg_handle* h, const cpg_dag* d) {
  if (check_handle(h) != CPG_OK || !d) return CPG_ERR_INVALID;
  return load_edgelist(h, d->el);
}

void cpg_dag_free(cpg_dag* d) { delete d; }

}  // extern "C"
