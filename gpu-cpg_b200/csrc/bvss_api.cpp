// C ABI of the BVSS component: host builders, decode / verify, and the two
// device operations (pull BFS levels, deviation pair discovery).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "cpg_internal.hpp"

using namespace cpg;

namespace {

constexpr unsigned int kBvssSpinLimit = 1u << 24;

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
};

cudaError_t grow(Buf& b, size_t bytes) {
  if (bytes <= b.bytes && b.p) return cudaSuccess;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  cudaError_t e = cudaMalloc(&b.p, std::max<size_t>(bytes, 16));
  if (e == cudaSuccess) b.bytes = std::max<size_t>(bytes, 16);
  return e;
}

}  // namespace

struct cpg_bvss {
  HostBvss hb;
  bool adev = false;
  std::string err;
  int device = -1;  // device holding the copy below
  Buf d_ptr, d_v2r, d_cnt, d_rows, d_masks, d_scratch, d_ctr, d_io, d_out;
};

namespace {

Status bfail(cpg_bvss* b, Status s, const std::string& msg) {
  if (b) b->err = msg;
  return s;
}

#define BCK(expr, what)                                                        \
  do {                                                                         \
    const cudaError_t _e = (expr);                                             \
    if (_e != cudaSuccess) {                                                   \
      cudaGetLastError();                                                      \
      return bfail(b, _e == cudaErrorMemoryAllocation ? CPG_ERR_OOM : CPG_ERR_CUDA, \
                   std::string(what) + ": " + cudaGetErrorString(_e));         \
    }                                                                          \
  } while (0)

Status upload(cpg_bvss* b, int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return bfail(b, CPG_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return bfail(b, CPG_ERR_INVALID, "bad device ordinal");
  BCK(cudaSetDevice(device), "cudaSetDevice");
  if (b->device == device) return CPG_OK;
  Buf* all[] = {&b->d_ptr, &b->d_v2r, &b->d_cnt, &b->d_rows, &b->d_masks,
                &b->d_scratch, &b->d_ctr, &b->d_io, &b->d_out};
  for (Buf* x : all) {
    if (x->p) cudaFree(x->p);
    *x = Buf{};
  }
  const HostBvss& h = b->hb;
  BCK(grow(b->d_ptr, h.ptr.size() * 4), "alloc BVSS");
  BCK(grow(b->d_v2r, h.v2r.size() * 4), "alloc BVSS");
  BCK(grow(b->d_cnt, h.cnt.size()), "alloc BVSS");
  BCK(grow(b->d_rows, h.rows.size() * 4), "alloc BVSS");
  BCK(grow(b->d_masks, h.masks.size() * 4), "alloc BVSS");
  BCK(grow(b->d_ctr, sizeof(BvssCounters)), "alloc BVSS");
  BCK(cudaMemcpy(b->d_ptr.p, h.ptr.data(), h.ptr.size() * 4, cudaMemcpyHostToDevice), "H2D BVSS");
  if (h.n_vss) {
    BCK(cudaMemcpy(b->d_v2r.p, h.v2r.data(), h.v2r.size() * 4, cudaMemcpyHostToDevice), "H2D BVSS");
    BCK(cudaMemcpy(b->d_cnt.p, h.cnt.data(), h.cnt.size(), cudaMemcpyHostToDevice), "H2D BVSS");
    BCK(cudaMemcpy(b->d_rows.p, h.rows.data(), h.rows.size() * 4, cudaMemcpyHostToDevice), "H2D BVSS");
    BCK(cudaMemcpy(b->d_masks.p, h.masks.data(), h.masks.size() * 4, cudaMemcpyHostToDevice), "H2D BVSS");
  }
  b->device = device;
  return CPG_OK;
}

DevBvss dev_view(const cpg_bvss* b) {
  DevBvss d{};
  d.n_rows = b->hb.n_rows;
  d.n_intervals = b->hb.n_intervals;
  d.n_vss = b->hb.n_vss;
  d.ptr = static_cast<const int32_t*>(b->d_ptr.p);
  d.v2r = static_cast<const int32_t*>(b->d_v2r.p);
  d.cnt = static_cast<const uint8_t*>(b->d_cnt.p);
  d.rows = static_cast<const int32_t*>(b->d_rows.p);
  d.masks = static_cast<const unsigned int*>(b->d_masks.p);
  return d;
}

BvssDispatch dispatch(const cpg_bvss_opts& o) {
  BvssDispatch d{};
  d.mode = o.tiles;
  d.min_bits = o.min_bits > 0 ? o.min_bits : 2;
  d.min_slices = o.min_slices > 0 ? o.min_slices : 32;
  d.half_slices = o.half_slices > 0 ? o.half_slices : 64;
  return d;
}

// Transposed deviation relation: row v -> tails u of edges u -> v, v != succ[u].
Status adev_csr(int32_t n, const int32_t* rp, const int32_t* ci, const int32_t* succ,
                std::vector<int32_t>& trp, std::vector<int32_t>& tci, std::string& err) {
  if (n < 0 || !rp || rp[0] != 0) {
    err = "BVSS: invalid CSR";
    return CPG_ERR_INVALID;
  }
  for (int32_t u = 0; u < n; ++u) {
    if (rp[u] > rp[u + 1]) {
      err = "BVSS: row_ptr must be nondecreasing";
      return CPG_ERR_INVALID;
    }
    if (succ[u] < -1 || succ[u] >= n) {
      err = "BVSS: succs outside [-1, n)";
      return CPG_ERR_INVALID;
    }
  }
  for (int32_t e = 0; e < rp[n]; ++e)
    if (ci[e] < 0 || ci[e] >= n) {
      err = "BVSS: column outside [0, n)";
      return CPG_ERR_INVALID;
    }
  trp.assign(static_cast<size_t>(n) + 1, 0);
  for (int32_t u = 0; u < n; ++u)
    for (int32_t e = rp[u]; e < rp[u + 1]; ++e)
      if (ci[e] != succ[u]) trp[ci[e] + 1]++;
  for (int32_t v = 0; v < n; ++v) trp[v + 1] += trp[v];
  tci.resize(static_cast<size_t>(trp[n]));
  std::vector<int32_t> fill(trp.begin(), trp.end() - 1);
  for (int32_t u = 0; u < n; ++u)
    for (int32_t e = rp[u]; e < rp[u + 1]; ++e)
      if (ci[e] != succ[u]) tci[fill[ci[e]]++] = u;
  return CPG_OK;
}

}  // namespace

extern "C" {

void cpg_bvss_opts_init(cpg_bvss_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
}

cpg_status cpg_bvss_build(cpg_bvss** out, int32_t n, const int32_t* row_ptr,
                          const int32_t* col_idx, const int32_t* succs) {
  if (!out) return CPG_ERR_INVALID;
  *out = nullptr;
  cpg_bvss* b = new cpg_bvss();
  Status st;
  if (succs) {
    std::vector<int32_t> trp, tci;
    st = adev_csr(n, row_ptr, col_idx, succs, trp, tci, b->err);
    if (st == CPG_OK) st = pack_bvss(n, trp.data(), tci.data(), b->hb, b->err);
    b->adev = true;
  } else {
    st = pack_bvss(n, row_ptr, col_idx, b->hb, b->err);
  }
  if (st != CPG_OK) {
    delete b;
    return static_cast<cpg_status>(st);
  }
  *out = b;
  return CPG_OK;
}

cpg_status cpg_bvss_build_compact(cpg_bvss** out, int32_t n, const int32_t* deviation_offsets) {
  if (!out) return CPG_ERR_INVALID;
  *out = nullptr;
  cpg_bvss* b = new cpg_bvss();
  Status st = pack_bvss_compact(n, deviation_offsets, b->hb, b->err);
  if (st != CPG_OK) {
    delete b;
    return static_cast<cpg_status>(st);
  }
  b->adev = true;
  *out = b;
  return CPG_OK;
}

void cpg_bvss_destroy(cpg_bvss* b) {
  if (!b) return;
  if (b->device >= 0) {
    cudaSetDevice(b->device);
    Buf* all[] = {&b->d_ptr, &b->d_v2r, &b->d_cnt, &b->d_rows, &b->d_masks,
                  &b->d_scratch, &b->d_ctr, &b->d_io, &b->d_out};
    for (Buf* x : all)
      if (x->p) cudaFree(x->p);
  }
  delete b;
}

const char* cpg_bvss_last_error(const cpg_bvss* b) { return b ? b->err.c_str() : "null BVSS"; }

cpg_status cpg_bvss_get_info(const cpg_bvss* b, cpg_bvss_info* info) {
  if (!b || !info) return CPG_ERR_INVALID;
  std::memset(info, 0, sizeof(*info));
  info->sigma = 8;
  info->slices_per_thread = 4;
  info->slice_capacity = 128;
  info->n_intervals = b->hb.n_intervals;
  info->n_vss = b->hb.n_vss;
  info->n_rows = b->hb.n_rows;
  info->unpadded_slices = static_cast<int64_t>(b->hb.unpadded_slices);
  info->total_set_bits = static_cast<int64_t>(b->hb.total_set_bits);
  info->compression_ratio =
      b->hb.unpadded_slices ? static_cast<double>(b->hb.total_set_bits) /
                                  (8.0 * static_cast<double>(b->hb.unpadded_slices))
                            : 0.0;
  return CPG_OK;
}

cpg_status cpg_bvss_get_arrays(const cpg_bvss* b, int32_t* real_ptrs, int32_t* virtual_to_real,
                               uint8_t* slice_counts, int32_t* row_ids, uint32_t* masks) {
  if (!b) return CPG_ERR_INVALID;
  const HostBvss& h = b->hb;
  if (real_ptrs) std::copy(h.ptr.begin(), h.ptr.end(), real_ptrs);
  if (virtual_to_real) std::copy(h.v2r.begin(), h.v2r.end(), virtual_to_real);
  if (slice_counts) std::copy(h.cnt.begin(), h.cnt.end(), slice_counts);
  if (row_ids) std::copy(h.rows.begin(), h.rows.end(), row_ids);
  if (masks) std::copy(h.masks.begin(), h.masks.end(), masks);
  return CPG_OK;
}

cpg_status cpg_bvss_decode_row(const cpg_bvss* b, int32_t row, int32_t* out, int32_t cap,
                               int32_t* n_out) {
  if (!b || !n_out || (cap > 0 && !out)) return CPG_ERR_INVALID;
  const std::vector<int32_t> cols = bvss_decode_row(b->hb, row);
  *n_out = static_cast<int32_t>(cols.size());
  if (static_cast<int32_t>(cols.size()) > cap) return CPG_ERR_CAPACITY;
  std::copy(cols.begin(), cols.end(), out);
  return CPG_OK;
}

int32_t cpg_bvss_verify(const cpg_bvss* b, int32_t n, const int32_t* row_ptr,
                        const int32_t* col_idx, const int32_t* succs) {
  if (!b || n < 0 || !row_ptr) return -1;
  std::vector<int32_t> trp, tci;
  const int32_t* rp = row_ptr;
  const int32_t* ci = col_idx;
  if (succs) {
    std::string err;
    if (adev_csr(n, row_ptr, col_idx, succs, trp, tci, err) != CPG_OK) return -1;
    rp = trp.data();
    ci = tci.data();
  } else {
    if (row_ptr[0] != 0) return -1;
    for (int32_t e = 0; e < row_ptr[n]; ++e)
      if (col_idx[e] < 0 || col_idx[e] >= n) return -1;
  }
  if (b->hb.n_rows != n || b->hb.n_intervals != (n + 7) / 8) return 0;
  // decode every row at once: rows -> columns from the packed arrays
  std::vector<std::vector<int32_t>> got(static_cast<size_t>(n));
  const HostBvss& h = b->hb;
  for (int32_t vss = 0; vss < h.n_vss; ++vss)
    for (int32_t slot = 0; slot < 128; ++slot) {
      const int32_t r = h.rows[static_cast<size_t>(vss) * 128 + slot];
      if (r < 0) continue;
      if (r >= n) return 0;
      const uint32_t m = (h.masks[static_cast<size_t>(vss) * 32 + slot / 4] >> (8 * (slot % 4))) & 0xffu;
      for (int32_t bit = 0; bit < 8; ++bit)
        if (m & (1u << bit)) got[r].push_back(h.v2r[vss] * 8 + bit);
    }
  std::vector<int32_t> want;
  for (int32_t r = 0; r < n; ++r) {
    want.assign(ci + rp[r], ci + rp[r + 1]);
    std::sort(want.begin(), want.end());
    want.erase(std::unique(want.begin(), want.end()), want.end());
    std::sort(got[r].begin(), got[r].end());
    if (got[r] != want) return 0;
  }
  return 1;
}

cpg_status cpg_bvss_levels(cpg_bvss* b, const cpg_bvss_opts* opts, const int32_t* sinks,
                           int32_t n_sinks, int32_t* levels, cpg_bvss_run_stats* stats) {
  if (!b || !levels || n_sinks < 0 || (n_sinks > 0 && !sinks)) return CPG_ERR_INVALID;
  if (b->adev) return bfail(b, CPG_ERR_INVALID, "levels need a fan-out BVSS");
  cpg_bvss_opts o;
  cpg_bvss_opts_init(&o);
  if (opts) o = *opts;
  Status st = upload(b, o.device);
  if (st != CPG_OK) return static_cast<cpg_status>(st);
  const HostBvss& h = b->hb;
  std::vector<int32_t> own;
  if (!sinks) {
    for (int32_t r = 0; r < h.n_rows; ++r)
      if (h.row_bits[r] == 0) own.push_back(r);
    sinks = own.data();
    n_sinks = static_cast<int32_t>(own.size());
  }
  const size_t sw = bvss_levels_scratch_words(h.n_rows, h.n_intervals, h.n_vss);
  BCK(grow(b->d_scratch, sw * 4), "alloc BVSS scratch");
  BCK(grow(b->d_io, static_cast<size_t>(n_sinks) * 4), "alloc BVSS sinks");
  BCK(grow(b->d_out, static_cast<size_t>(h.n_rows) * 4), "alloc BVSS levels");
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0), "event");
  BCK(cudaEventCreate(&e1), "event");
  cudaError_t e = cudaSuccess;
  if (n_sinks) e = cudaMemcpyAsync(b->d_io.p, sinks, static_cast<size_t>(n_sinks) * 4,
                                   cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaEventRecord(e0, s);
  if (e == cudaSuccess)
    e = static_cast<cudaError_t>(launch_bvss_levels(
        dev_view(b), static_cast<const int32_t*>(b->d_io.p), n_sinks,
        static_cast<int32_t*>(b->d_out.p), static_cast<unsigned int*>(b->d_scratch.p),
        static_cast<BvssCounters*>(b->d_ctr.p), dispatch(o),
        o.spin_limit ? o.spin_limit : kBvssSpinLimit, o.device, s));
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  BvssCounters c{};
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&c, b->d_ctr.p, sizeof(c), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && h.n_rows)
    e = cudaMemcpyAsync(levels, b->d_out.p, static_cast<size_t>(h.n_rows) * 4,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BCK(e, "BVSS levels");
  if (c.err == kDevTimeout) return bfail(b, CPG_ERR_TIMEOUT, "BVSS levels: grid barrier wait ran out");
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->levels = c.level;
    stats->tiles_tensor = static_cast<int64_t>(c.tiles_tensor);
    stats->tiles_scalar = static_cast<int64_t>(c.tiles_scalar);
    stats->mma_issued = static_cast<int64_t>(c.mma_issued);
    stats->device_ms = ms;
  }
  return CPG_OK;
}

cpg_status cpg_bvss_discover_pairs(cpg_bvss* b, const cpg_bvss_opts* opts,
                                   const int32_t* sources, int32_t n_sources, int32_t* pairs,
                                   int64_t max_pairs, int64_t* n_pairs,
                                   cpg_bvss_run_stats* stats) {
  if (!b || !n_pairs || n_sources < 0 || (n_sources > 0 && !sources) || max_pairs < 0 ||
      (max_pairs > 0 && !pairs))
    return CPG_ERR_INVALID;
  cpg_bvss_opts o;
  cpg_bvss_opts_init(&o);
  if (opts) o = *opts;
  Status st = upload(b, o.device);
  if (st != CPG_OK) return static_cast<cpg_status>(st);
  const HostBvss& h = b->hb;
  const size_t sw = bvss_pairs_scratch_words(h.n_intervals, h.n_vss);
  BCK(grow(b->d_scratch, sw * 4), "alloc BVSS scratch");
  BCK(grow(b->d_io, static_cast<size_t>(n_sources) * 4), "alloc BVSS sources");
  BCK(grow(b->d_out, static_cast<size_t>(std::max<int64_t>(max_pairs, 1)) * 8), "alloc BVSS pairs");
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0), "event");
  BCK(cudaEventCreate(&e1), "event");
  cudaError_t e = cudaSuccess;
  if (n_sources) e = cudaMemcpyAsync(b->d_io.p, sources, static_cast<size_t>(n_sources) * 4,
                                     cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaEventRecord(e0, s);
  if (e == cudaSuccess)
    e = static_cast<cudaError_t>(launch_bvss_pairs(
        dev_view(b), static_cast<const int32_t*>(b->d_io.p), n_sources,
        static_cast<int32_t*>(b->d_out.p), max_pairs, static_cast<unsigned int*>(b->d_scratch.p),
        static_cast<BvssCounters*>(b->d_ctr.p), dispatch(o), s));
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  BvssCounters c{};
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&c, b->d_ctr.p, sizeof(c), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  const int64_t total = static_cast<int64_t>(c.pairs);
  const int64_t got = std::min(total, max_pairs);
  if (e == cudaSuccess && got > 0)
    e = cudaMemcpy(pairs, b->d_out.p, static_cast<size_t>(got) * 8, cudaMemcpyDeviceToHost);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BCK(e, "BVSS pairs");
  *n_pairs = total;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->tiles_tensor = static_cast<int64_t>(c.tiles_tensor);
    stats->tiles_scalar = static_cast<int64_t>(c.tiles_scalar);
    stats->mma_issued = static_cast<int64_t>(c.mma_issued);
    stats->device_ms = ms;
  }
  // (u, v) order, as the reference returns them
  std::vector<std::pair<int32_t, int32_t>> pv(static_cast<size_t>(got));
  for (int64_t i = 0; i < got; ++i) pv[i] = {pairs[2 * i], pairs[2 * i + 1]};
  std::sort(pv.begin(), pv.end());
  for (int64_t i = 0; i < got; ++i) {
    pairs[2 * i] = pv[i].first;
    pairs[2 * i + 1] = pv[i].second;
  }
  if (total > max_pairs) return bfail(b, CPG_ERR_CAPACITY, "BVSS pairs: more pairs than max_pairs");
  return CPG_OK;
}

}  // extern "C"
