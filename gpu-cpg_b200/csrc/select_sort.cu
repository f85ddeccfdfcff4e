// Top-K selection and sorting of path costs for sm_100a (HBM-bound integer
// work, no tensor cores): a three-pass radix select (11/11/10-bit digits) of
// the k-th smallest non-zero cost, a compaction of the k winners and an LSD
// radix sort (4 x 8-bit digits) of their (orderable cost, path index) pairs.
//
// Replaces the reference's final comparator merge sort of the whole short
// pile and its zero-cost filter (gpucpg/gpucpg.cu:21323-21360): only the k
// survivors are sorted, and zero-cost paths are excluded before selection.
#include <mutex>

#include "device_common.cuh"

namespace cpg {

namespace {

constexpr int kSelThreads = 256;
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;

struct SelectState {
  unsigned int prefix;        // decided high bits of the k-th key
  unsigned int pad;
  unsigned long long k_rem;   // rank still wanted inside the current prefix
};

__device__ __forceinline__ float load_strided(const float* a, unsigned long long i,
                                              unsigned stride) {
  return __ldcg(a + i * stride);
}

__global__ void select_init_kernel(SelectState* st, unsigned long long k) {
  st->prefix = 0;
  st->k_rem = k;
}

// One radix pass: histogram of digit (key >> shift) & (bins-1) among keys whose
// bits above shift+bits equal the decided prefix.
__global__ void select_hist_kernel(const float* a, unsigned long long na,
                                   unsigned sa, const float* b,
                                   unsigned long long nb, unsigned sb,
                                   int skip_zero, const SelectState* st,
                                   int shift, int bits, unsigned int* hist) {
  extern __shared__ unsigned int sh[];
  const int bins = 1 << bits;
  for (int i = threadIdx.x; i < bins; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const unsigned int prefix = st->prefix;
  const int hi = shift + bits;
  const unsigned int hmask = hi >= 32 ? 0u : ~((1u << hi) - 1u);
  const unsigned long long n = na + nb;
  const unsigned long long stride =
      static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  for (unsigned long long i =
           static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
       i < n; i += stride) {
    const float x = i < na ? load_strided(a, i, sa) : load_strided(b, i - na, sb);
    if (skip_zero && x == 0.0f) continue;
    const unsigned int k = float_key(x);
    if ((k & hmask) != (prefix & hmask)) continue;
    atomicAdd(&sh[(k >> shift) & (bins - 1)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bins; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Single block: find the bin holding the k_rem-th key, narrow the prefix.
__global__ void select_pick_kernel(SelectState* st, int shift, int bits,
                                   unsigned int* hist) {
  __shared__ unsigned long long part[1024];
  const int bins = 1 << bits;
  const int per = (bins + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per;
  unsigned long long s = 0;
  for (int i = b0; i < b0 + per && i < bins; ++i) s += hist[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long k = st->k_rem, acc = 0;
    int t = 0;
    for (; t < static_cast<int>(blockDim.x); ++t) {
      if (acc + part[t] >= k) break;
      acc += part[t];
    }
    if (t == static_cast<int>(blockDim.x)) t = blockDim.x - 1;  // k > total: clamp
    int bin = t * per;
    for (; bin < bins - 1; ++bin) {
      if (acc + hist[bin] >= k) break;
      acc += hist[bin];
    }
    st->prefix |= static_cast<unsigned int>(bin) << shift;
    st->k_rem = k - acc;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bins; i += blockDim.x) hist[i] = 0;
}

__global__ void count_le_kernel(const float* a, unsigned long long n,
                                unsigned stride_f, const unsigned int* t_key,
                                unsigned long long* out) {
  const unsigned int t = *t_key;
  unsigned long long le = 0, nz = 0;
  const unsigned long long stride =
      static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  for (unsigned long long i =
           static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
       i < n; i += stride) {
    const float x = load_strided(a, i, stride_f);
    if (x == 0.0f) continue;
    ++nz;
    le += float_key(x) <= t;
  }
  for (int o = 16; o > 0; o >>= 1) {
    le += __shfl_xor_sync(0xffffffffu, le, o);
    nz += __shfl_xor_sync(0xffffffffu, nz, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (le) atomicAdd(out, le);
    if (nz) atomicAdd(out + 1, nz);
  }
}

// Keys strictly below the k-th key all win; of the keys equal to it, the
// first need_eq to arrive win.
__global__ void compact_kernel(const float* cost, unsigned long long n,
                               const SelectState* st, unsigned long long k,
                               unsigned int* keys, unsigned int* vals,
                               unsigned long long* cnt) {
  const unsigned int kth = st->prefix;
  const unsigned long long need_eq = st->k_rem;
  const unsigned long long n_lt = k - need_eq;
  const unsigned long long stride =
      static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  const unsigned long long n_pad = (n + 31) & ~31ull;
  for (unsigned long long i =
           static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
       i < n_pad; i += stride) {
    bool lt = false, eq = false;
    unsigned int key = 0;
    if (i < n) {
      const float x = __ldcg(cost + i);
      if (x != 0.0f) {
        key = float_key(x);
        lt = key < kth;
        eq = key == kth;
      }
    }
    const unsigned long long a = warp_append(&cnt[0], lt);
    if (lt && a < n_lt) {
      keys[a] = key;
      vals[a] = static_cast<unsigned int>(i);
    }
    const unsigned long long b = warp_append(&cnt[1], eq);
    if (eq && b < need_eq) {
      keys[n_lt + b] = key;
      vals[n_lt + b] = static_cast<unsigned int>(i);
    }
  }
}

__global__ void sort_hist_kernel(const unsigned int* keys, unsigned long long n,
                                 int shift, unsigned int* hist, int nblocks) {
  __shared__ unsigned int sh[256];
  sh[threadIdx.x] = 0;
  __syncthreads();
  const unsigned long long base = static_cast<unsigned long long>(blockIdx.x) * kSortTile;
  for (int t = 0; t < kSortItems; ++t) {
    const unsigned long long i = base + t * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&sh[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * nblocks + blockIdx.x] = sh[threadIdx.x];
}

// Exclusive scan of 256*nblocks digit-major counts in one block.
__global__ void sort_scan_kernel(unsigned int* hist, int total) {
  __shared__ unsigned int warp_sums[32];
  __shared__ unsigned int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = 0; base < total; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const unsigned int x = i < total ? hist[i] : 0u;
    unsigned int incl = x;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      unsigned int ws = lane < static_cast<int>(blockDim.x >> 5) ? warp_sums[lane] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, ws, o);
        if (lane >= o) ws += y;
      }
      warp_sums[lane] = ws;
    }
    __syncthreads();
    const unsigned int before = (wid ? warp_sums[wid - 1] : 0u) + carry;
    if (i < total) hist[i] = before + incl - x;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + incl;
    __syncthreads();
  }
}

// Stable scatter: elements are ranked in tile order (round-major, then thread).
__global__ void sort_scatter_kernel(const unsigned int* keys_in,
                                    const unsigned int* vals_in,
                                    unsigned int* keys_out,
                                    unsigned int* vals_out,
                                    unsigned long long n, int shift,
                                    const unsigned int* hist, int nblocks) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ unsigned int running[256];
  __shared__ unsigned int wcount[kWarps][256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  running[threadIdx.x] = hist[threadIdx.x * nblocks + blockIdx.x];
  for (int w = 0; w < kWarps; ++w) wcount[w][threadIdx.x] = 0;
  __syncthreads();
  const unsigned long long base = static_cast<unsigned long long>(blockIdx.x) * kSortTile;
  for (int t = 0; t < kSortItems; ++t) {
    const unsigned long long i = base + t * kSortThreads + threadIdx.x;
    const bool valid = i < n;
    unsigned int key = 0, val = 0, d = 256u;
    if (valid) {
      key = keys_in[i];
      val = vals_in[i];
      d = (key >> shift) & 255u;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned int lrank = __popc(peers & lanemask_lt());
    if (valid && lrank == 0) wcount[wid][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      unsigned int pos = running[d] + lrank;
      for (int w = 0; w < wid; ++w) pos += wcount[w][d];
      keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads();
    {
      unsigned int s = 0;
      for (int w = 0; w < kWarps; ++w) {
        s += wcount[w][threadIdx.x];
        wcount[w][threadIdx.x] = 0;
      }
      running[threadIdx.x] += s;
    }
    __syncthreads();
  }
}

__global__ void rank_kernel(const unsigned int* vals, unsigned long long n,
                            int32_t* rank_of) {
  const unsigned long long i =
      static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) rank_of[vals[i]] = static_cast<int32_t>(i);
}

__global__ void emit_kernel(PathStore ps, const unsigned int* vals,
                            unsigned long long n, const int32_t* rank_of,
                            float* out_cost, cpg_path_node* out_nodes) {
  const unsigned long long i =
      static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned int idx = vals[i];
  const float c = ps.cost[idx];
  out_cost[i] = c;
  if (out_nodes) {
    cpg_path_node nd;
    nd.level = ps.level[idx];
    nd.from = ps.from[idx];
    nd.to = ps.to[idx];
    const int par = ps.parent[idx];
    nd.parent = par >= 0 ? rank_of[par] : -1;
    nd.num_children = 0;
    nd.slack = c;
    out_nodes[i] = nd;
  }
}

int grid_for(unsigned long long n, int threads, int cap_blocks) {
  unsigned long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > static_cast<unsigned long long>(cap_blocks)) b = cap_blocks;
  return static_cast<int>(b);
}

}  // namespace

size_t select_state_bytes() { return sizeof(SelectState); }

// k-th smallest (1-based) among the union of a (stride sa floats) and b
// (stride sb floats).  state receives {prefix = key, k_rem = rank among equal}.
int launch_select_kth(const float* a, unsigned long long na, unsigned sa,
                      const float* b, unsigned long long nb, unsigned sb,
                      unsigned long long k, int skip_zero, void* state,
                      unsigned int* hist, void* stream, int* launches) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  SelectState* st = static_cast<SelectState*>(state);
  select_init_kernel<<<1, 1, 0, s>>>(st, k);
  const int shifts[3] = {21, 10, 0};
  const int bits[3] = {11, 11, 10};
  const int grid = grid_for(na + nb, kSelThreads, 148 * 8);
  for (int pass = 0; pass < 3; ++pass) {
    select_hist_kernel<<<grid, kSelThreads, (1 << bits[pass]) * sizeof(unsigned int), s>>>(
        a, na, sa, b, nb, sb, skip_zero, st, shifts[pass], bits[pass], hist);
    select_pick_kernel<<<1, 1024, 0, s>>>(st, shifts[pass], bits[pass], hist);
  }
  if (launches) *launches += 7;
  return cudaGetLastError();
}

int launch_count_le(const float* a, unsigned long long n, unsigned stride_f,
                    const unsigned int* t_key, unsigned long long* out,
                    void* stream) {
  if (n == 0) return cudaSuccess;
  count_le_kernel<<<grid_for(n, 256, 148 * 8), 256, 0,
                    static_cast<cudaStream_t>(stream)>>>(a, n, stride_f, t_key, out);
  return cudaGetLastError();
}

// Sorted top-k emission.  state holds the k-th key from launch_select_kth run
// over the accepted costs with k.  keys/vals need 2*k entries each; hist needs
// 256*ceil(k/2048) words; rank_of needs n_paths entries; cnt 2 words.
int launch_emit_topk(const PathStore& ps, unsigned long long n_paths,
                     const void* state, unsigned long long k,
                     unsigned int* keys, unsigned int* vals, unsigned int* hist,
                     unsigned long long* cnt, int32_t* rank_of, float* out_cost,
                     cpg_path_node* out_nodes, void* stream, int* launches) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (k == 0) return cudaSuccess;
  const SelectState* st = static_cast<const SelectState*>(state);
  cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), s);
  // every slot is overwritten by the compaction; zero-filling keeps a path
  // index in range even if the selection and the compaction ever disagreed
  cudaMemsetAsync(vals, 0, k * sizeof(unsigned int), s);
  compact_kernel<<<grid_for(n_paths, 256, 148 * 16), 256, 0, s>>>(
      ps.cost, n_paths, st, k, keys, vals, cnt);
  const int nblocks = static_cast<int>((k + kSortTile - 1) / kSortTile);
  unsigned int* kin = keys;
  unsigned int* vin = vals;
  unsigned int* kout = keys + k;
  unsigned int* vout = vals + k;
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = pass * 8;
    sort_hist_kernel<<<nblocks, kSortThreads, 0, s>>>(kin, k, shift, hist, nblocks);
    sort_scan_kernel<<<1, 1024, 0, s>>>(hist, 256 * nblocks);
    sort_scatter_kernel<<<nblocks, kSortThreads, 0, s>>>(kin, vin, kout, vout, k,
                                                         shift, hist, nblocks);
    unsigned int* t = kin;
    kin = kout;
    kout = t;
    t = vin;
    vin = vout;
    vout = t;
  }
  cudaMemsetAsync(rank_of, 0xff, n_paths * sizeof(int32_t), s);
  rank_kernel<<<grid_for(k, 256, 1 << 30), 256, 0, s>>>(vin, k, rank_of);
  emit_kernel<<<grid_for(k, 256, 1 << 30), 256, 0, s>>>(ps, vin, k, rank_of,
                                                        out_cost, out_nodes);
  if (launches) *launches += 1 + 12 + 2;
  return cudaGetLastError();
}

}  // namespace cpg

namespace cpg {

namespace {

__global__ void keys_to_costs_kernel(const unsigned int* keys, unsigned long long n,
                                     float* out) {
  for (unsigned long long i = static_cast<unsigned long long>(blockIdx.x) * blockDim.x +
                              threadIdx.x;
       i < n; i += static_cast<unsigned long long>(gridDim.x) * blockDim.x)
    out[i] = key_float(keys[i]);
}

}  // namespace

size_t topk_sort_hist_words(unsigned long long k) {
  return 256 * ((k + kSortTile - 1) / kSortTile);
}

// The k smallest non-zero values of costs[0..n), ascending, into out.  Two
// stages separated by a host read of the non-zero count: count, then select
// + compact + sort + gather.  s.hist must hold 2048 zero words (the select
// leaves them zero again); s.keys/s.vals 2*k words each.
int launch_topk_costs(const float* costs, unsigned long long n, unsigned long long k,
                      const TopkScratch& s, float* out, unsigned long long* n_out,
                      void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  *n_out = 0;
  if (n == 0 || k == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(s.counts, 0, 2 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  const unsigned int all = 0xffffffffu;
  e = cudaMemcpyAsync(s.tkey, &all, 4, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  count_le_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(costs, n, 1, s.tkey, s.counts);
  unsigned long long host_counts[2] = {0, 0};
  e = cudaMemcpyAsync(host_counts, s.counts, sizeof(host_counts), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  const unsigned long long kk = host_counts[1] < k ? host_counts[1] : k;
  *n_out = kk;
  if (kk == 0) return cudaSuccess;
  int launches = 0;
  e = static_cast<cudaError_t>(launch_select_kth(costs, n, 1, nullptr, 0, 1, kk, 1, s.state,
                                                 s.hist, st, &launches));
  if (e != cudaSuccess) return e;
  cudaMemsetAsync(s.cnt, 0, 2 * sizeof(unsigned long long), st);
  cudaMemsetAsync(s.vals, 0, kk * sizeof(unsigned int), st);
  compact_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(
      costs, n, static_cast<const SelectState*>(s.state), kk, s.keys, s.vals, s.cnt);
  const int nblocks = static_cast<int>((kk + kSortTile - 1) / kSortTile);
  unsigned int* kin = s.keys;
  unsigned int* vin = s.vals;
  unsigned int* kout = s.keys + kk;
  unsigned int* vout = s.vals + kk;
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = pass * 8;
    sort_hist_kernel<<<nblocks, kSortThreads, 0, st>>>(kin, kk, shift, s.sort_hist, nblocks);
    sort_scan_kernel<<<1, 1024, 0, st>>>(s.sort_hist, 256 * nblocks);
    sort_scatter_kernel<<<nblocks, kSortThreads, 0, st>>>(kin, vin, kout, vout, kk, shift,
                                                          s.sort_hist, nblocks);
    unsigned int* t = kin;
    kin = kout;
    kout = t;
    t = vin;
    vin = vout;
    vout = t;
  }
  keys_to_costs_kernel<<<grid_for(kk, 256, 148 * 8), 256, 0, st>>>(kin, kk, out);
  return cudaGetLastError();
}

}  // namespace cpg

// ---------------------------------------------------------------- no-alloc
// cpg_select_topk_noalloc: the same top-K as cpg_select_topk, for callers
// that must not allocate device memory.  Its scratch is this file-scope
// array, reserved when the library is loaded (4.3 MiB on every GPU that
// loads it, held until the process exits).  In host code the name
// g_topk_scratch is only a host-side stand-in: the kernels get the device
// address that cudaGetSymbolAddress returns, looked up once per device with
// that device current.
namespace cpg {
namespace {

constexpr unsigned long long kNoAllocMaxK = CPG_SELECT_TOPK_NOALLOC_MAX_K;
// hist 2048 + state 4 + counts 4 + cnt 4 + tkey 4, keys/vals 2*K each,
// sort histogram 256 * ceil(K / 2048)
constexpr size_t kNoAllocWords =
    2048 + 16 + 4 * kNoAllocMaxK + 256 * ((kNoAllocMaxK + kSortTile - 1) / kSortTile);

__device__ __align__(256) unsigned int g_topk_scratch[kNoAllocWords];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

}  // namespace
}  // namespace cpg

extern "C" cpg_status cpg_select_topk_noalloc(const float* d_costs, int64_t n,
                                              int64_t k, float* d_out,
                                              int64_t* n_out, void* stream) {
  using namespace cpg;
  if (n < 0 || k < 0 || !n_out || (n > 0 && !d_costs) || (k > 0 && !d_out))
    return CPG_ERR_INVALID;
  *n_out = 0;
  if (n > (int64_t{1} << 32) - 1) return CPG_ERR_INVALID;
  if (static_cast<unsigned long long>(k) > kNoAllocMaxK) return CPG_ERR_CAPACITY;
  if (n == 0 || k == 0) return CPG_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return CPG_ERR_CUDA;
  }
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      // one-time set-up on this device (the current one): the device address
      // of the static scratch
      void* ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_topk_scratch) != cudaSuccess || !ptr) {
        cudaGetLastError();
        return CPG_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = ptr;
    }
    base = g_noalloc_ptr[dev];
  }
  const unsigned long long kk = static_cast<unsigned long long>(k < n ? k : n);
  unsigned int* w = static_cast<unsigned int*>(base);
  TopkScratch sc;
  sc.hist = w;
  sc.state = w + 2048;
  sc.counts = reinterpret_cast<unsigned long long*>(w + 2048 + 4);
  sc.cnt = reinterpret_cast<unsigned long long*>(w + 2048 + 8);
  sc.tkey = w + 2048 + 12;
  sc.keys = w + 2048 + 16;
  sc.vals = sc.keys + 2 * kNoAllocMaxK;
  sc.sort_hist = sc.vals + 2 * kNoAllocMaxK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: the select histogram must
  // start at zero
  cudaError_t e = cudaMemsetAsync(sc.hist, 0, 2048 * sizeof(unsigned int), s);
  unsigned long long got = 0;
  if (e == cudaSuccess)
    e = static_cast<cudaError_t>(
        launch_topk_costs(d_costs, static_cast<unsigned long long>(n), kk, sc, d_out, &got, s));
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return CPG_ERR_CUDA;
  *n_out = static_cast<int64_t>(got);
  return CPG_OK;
}
