// BVSS kernels for sm_100a: pull BFS levels from the sinks and deviation pair
// discovery, both counting frontier hits with b1 AND-popc MMA tiles where the
// density test passes (bvss.cuh).
//
// Levels restate run_tc_bvss_pull_bfs_levels / tc_bvss_pull_bfs_step
// (gpucpg/tc_sfxt_bvss.cuh:245-408, 497-577): a row joins level L+1 the first
// time one of its columns is in the level-L frontier.  The reference steps
// the levels from the host (four fills, one launch and one read-back per
// level); here one persistent cooperative launch walks every level with a
// bounded grid barrier and rotates three frontier bitmaps, three
// queued-interval bitmaps and three VSS queues, so nothing is cleared on the
// host between levels.
//
// Pairs restate build_frontier_from_sources, build_active_vss_queue_from_
// frontier and tc_transposed_adev_discover_pairs_counted (gpucpg/
// tc_pfxt_bvss.cuh:289-326, 452-540): each active VSS reserves one output
// range per warp from the tile's popcounts.
#include <algorithm>

#include "bvss.cuh"
#include "device_common.cuh"

namespace cpg {

namespace {

constexpr int kBvssThreads = 512;

struct LevelsArgs {
  DevBvss b;
  const int32_t* sinks;
  int32_t n_sinks;
  int32_t* levels;
  unsigned int* fr[3];      // frontier bitmaps
  unsigned int* qd[3];      // queued-interval bitmaps
  unsigned int* vis;        // visited bitmap
  int32_t* q[3];            // VSS queues
  int32_t fw, iw;           // words per vertex / interval bitmap
  BvssCounters* ctr;
  BvssDispatch d;
  unsigned int spin_limit;
};

// Queue every VSS of interval iv once per level.
__device__ __forceinline__ void queue_interval(const LevelsArgs& a, int slot, int iv) {
  const unsigned bit = 1u << (iv & 31);
  if (atomicOr(a.qd[slot] + (iv >> 5), bit) & bit) return;
  const int beg = a.b.ptr[iv], cnt = a.b.ptr[iv + 1] - beg;
  if (cnt == 0) return;
  const int base = atomicAdd(&a.ctr->qn[slot], cnt);
  for (int j = 0; j < cnt; ++j) a.q[slot][base + j] = beg + j;
}

__global__ void __launch_bounds__(kBvssThreads) bvss_levels_kernel(LevelsArgs a) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nth = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  const int gwarp = tid >> 5;
  const int nwarps = nth >> 5;
  // phase 0: clear the bitmaps and the levels
  for (int i = tid; i < a.fw; i += nth) {
    a.fr[0][i] = a.fr[1][i] = a.fr[2][i] = 0u;
    a.vis[i] = 0u;
  }
  for (int i = tid; i < a.iw; i += nth) a.qd[0][i] = a.qd[1][i] = a.qd[2][i] = 0u;
  for (int v = tid; v < a.b.n_rows; v += nth) a.levels[v] = -1;
  if (!grid_sync(&a.ctr->bar, &a.ctr->err, a.spin_limit)) return;
  // phase 1: the sinks are level 0
  for (int i = tid; i < a.n_sinks; i += nth) {
    const int t = a.sinks[i];
    if (t < 0 || t >= a.b.n_rows) continue;
    const unsigned bit = 1u << (t & 31);
    if (atomicOr(a.vis + (t >> 5), bit) & bit) continue;  // listed twice
    a.levels[t] = 0;
    atomicOr(a.fr[0] + (t >> 5), bit);
    queue_interval(a, 0, t >> 3);
  }
  if (!grid_sync(&a.ctr->bar, &a.ctr->err, a.spin_limit)) return;

  unsigned long long n_tensor = 0, n_scalar = 0, n_mma = 0;
  int lvl = 0;
  for (;; ++lvl) {
    const int cur = lvl % 3, nxt = (lvl + 1) % 3, old = (lvl + 2) % 3;
    const int qsize = __ldcg(&a.ctr->qn[cur]);
    if (qsize == 0) break;
    // buffers pulled at lvl - 1 are written again at lvl + 1
    for (int i = tid; i < a.fw; i += nth) a.fr[old][i] = 0u;
    for (int i = tid; i < a.iw; i += nth) a.qd[old][i] = 0u;
    if (tid == 0) a.ctr->qn[old] = 0;
    for (int qi = gwarp; qi < qsize; qi += nwarps) {
      const int vss = __ldcg(a.q[cur] + qi);
      const int iv = a.b.v2r[vss];
      const unsigned fb = frontier_byte(a.fr[cur], iv);
      if (fb == 0) continue;
      const unsigned mask = a.b.masks[static_cast<size_t>(vss) * 32 + lane];
      const int4 rw = reinterpret_cast<const int4*>(a.b.rows)[static_cast<size_t>(vss) * 32 + lane];
      const int slices = a.b.cnt[vss];
      const bool tensor = bvss_use_tensor(a.d.mode, fb, slices, a.d.min_bits, a.d.min_slices);
      unsigned c[4];
      const int mmas = bvss_counts(mask, fb, tensor, slices > a.d.half_slices, c);
      n_tensor += tensor;
      n_scalar += !tensor;
      n_mma += mmas;
      const int row[4] = {rw.x, rw.y, rw.z, rw.w};
#pragma unroll
      for (int ch = 0; ch < 4; ++ch) {
        const int r = row[ch];
        if (c[ch] == 0 || r < 0) continue;
        const unsigned bit = 1u << (r & 31);
        if (atomicOr(a.vis + (r >> 5), bit) & bit) continue;
        a.levels[r] = lvl + 1;
        atomicOr(a.fr[nxt] + (r >> 5), bit);
        queue_interval(a, nxt, r >> 3);
      }
    }
    if (!grid_sync(&a.ctr->bar, &a.ctr->err, a.spin_limit)) return;
  }
  if (lane == 0) {
    atomicAdd(&a.ctr->tiles_tensor, n_tensor);
    atomicAdd(&a.ctr->tiles_scalar, n_scalar);
    atomicAdd(&a.ctr->mma_issued, n_mma);
  }
  if (tid == 0) a.ctr->level = lvl;  // levels holding at least one row
}

// ------------------------------------------------------------ pair discovery

__global__ void frontier_from_sources_kernel(const int32_t* sources, int32_t n_sources,
                                             int32_t n, unsigned int* words) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_sources) return;
  const int s = sources[i];
  if (s < 0 || s >= n) return;
  atomicOr(words + (s >> 5), 1u << (s & 31));
}

__global__ void active_vss_kernel(const unsigned int* words, const int32_t* ptr,
                                  int32_t n_intervals, int32_t* queue, BvssCounters* ctr) {
  const int iv = blockIdx.x * blockDim.x + threadIdx.x;
  if (iv >= n_intervals) return;
  if (((words[iv >> 2] >> ((iv & 3) * 8)) & 0xffu) == 0) return;
  const int beg = ptr[iv], cnt = ptr[iv + 1] - beg;
  if (cnt == 0) return;
  const int base = atomicAdd(&ctr->qn[0], cnt);
  for (int j = 0; j < cnt; ++j) queue[base + j] = beg + j;
}

__global__ void __launch_bounds__(256)
discover_pairs_kernel(DevBvss b, int32_t n_cols, const unsigned int* words, const int32_t* queue,
                      BvssCounters* ctr, int32_t* pairs, long long max_pairs, BvssDispatch d) {
  const int lane = threadIdx.x & 31;
  const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int qsize = ctr->qn[0];
  unsigned long long n_tensor = 0, n_scalar = 0, n_mma = 0;
  for (int qi = gwarp; qi < qsize; qi += nwarps) {
    const int vss = queue[qi];
    const int iv = b.v2r[vss];
    const unsigned fb = (words[iv >> 2] >> ((iv & 3) * 8)) & 0xffu;
    const unsigned mask = b.masks[static_cast<size_t>(vss) * 32 + lane];
    const int4 rw = reinterpret_cast<const int4*>(b.rows)[static_cast<size_t>(vss) * 32 + lane];
    const int slices = b.cnt[vss];
    const bool tensor = bvss_use_tensor(d.mode, fb, slices, d.min_bits, d.min_slices);
    unsigned c[4];
    n_mma += bvss_counts(mask, fb, tensor, slices > d.half_slices, c);
    n_tensor += tensor;
    n_scalar += !tensor;
    const int row[4] = {rw.x, rw.y, rw.z, rw.w};
    int mine = 0;
#pragma unroll
    for (int ch = 0; ch < 4; ++ch)
      if (row[ch] < 0 || row[ch] >= b.n_rows) c[ch] = 0;
      else mine += static_cast<int>(c[ch]);
    // one reservation per VSS: inclusive scan of the lane counts
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long base = 0;
    if (lane == 0 && total > 0) base = atomicAdd(&ctr->pairs, static_cast<unsigned long long>(total));
    base = __shfl_sync(0xffffffffu, base, 0);
    unsigned long long pos = base + static_cast<unsigned>(incl - mine);
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      if (c[ch] == 0) continue;
      unsigned hits = (mask >> (8 * ch)) & fb & 0xffu;
      while (hits) {
        const int bit = __ffs(hits) - 1;
        hits &= hits - 1;
        const int src = iv * 8 + bit;
        if (src >= n_cols) continue;
        if (pos < static_cast<unsigned long long>(max_pairs)) {
          pairs[2 * pos] = src;
          pairs[2 * pos + 1] = row[ch];
        }
        ++pos;
      }
    }
  }
  if (lane == 0) {
    atomicAdd(&ctr->tiles_tensor, n_tensor);
    atomicAdd(&ctr->tiles_scalar, n_scalar);
    atomicAdd(&ctr->mma_issued, n_mma);
  }
}

}  // namespace

size_t bvss_levels_scratch_words(int32_t n, int32_t n_intervals, int32_t n_vss) {
  const size_t fw = (static_cast<size_t>(n) + 31) / 32;
  const size_t iw = (static_cast<size_t>(n_intervals) + 31) / 32;
  return 4 * fw + 3 * iw + 3 * static_cast<size_t>(n_vss) + 4;
}

int launch_bvss_levels(const DevBvss& b, const int32_t* sinks, int32_t n_sinks,
                       int32_t* levels, unsigned int* scratch, BvssCounters* ctr,
                       BvssDispatch d, unsigned int spin_limit, int device, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  LevelsArgs a{};
  a.b = b;
  a.sinks = sinks;
  a.n_sinks = n_sinks;
  a.levels = levels;
  a.fw = (b.n_rows + 31) / 32;
  a.iw = (b.n_intervals + 31) / 32;
  unsigned int* w = scratch;
  for (int i = 0; i < 3; ++i) a.fr[i] = w + static_cast<size_t>(i) * a.fw;
  w += 3 * static_cast<size_t>(a.fw);
  a.vis = w;
  w += a.fw;
  for (int i = 0; i < 3; ++i) a.qd[i] = w + static_cast<size_t>(i) * a.iw;
  w += 3 * static_cast<size_t>(a.iw);
  for (int i = 0; i < 3; ++i)
    a.q[i] = reinterpret_cast<int32_t*>(w) + static_cast<size_t>(i) * b.n_vss;
  a.ctr = ctr;
  a.d = d;
  a.spin_limit = spin_limit;
  cudaError_t e = cudaMemsetAsync(ctr, 0, sizeof(BvssCounters), st);
  if (e != cudaSuccess) return e;
  int sms = 0, per_sm = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bvss_levels_kernel, kBvssThreads, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  void* args[] = {&a};
  e = cudaLaunchCooperativeKernel(reinterpret_cast<void*>(bvss_levels_kernel),
                                  dim3(sms * per_sm), dim3(kBvssThreads), args, 0, st);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

size_t bvss_pairs_scratch_words(int32_t n_intervals, int32_t n_vss) {
  return (static_cast<size_t>(n_intervals) * 8 + 31) / 32 + static_cast<size_t>(n_vss) + 4;
}

int launch_bvss_pairs(const DevBvss& b, const int32_t* sources, int32_t n_sources,
                      int32_t* pairs, long long max_pairs, unsigned int* scratch,
                      BvssCounters* ctr, BvssDispatch d, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // columns of an A_dev BVSS are vertices: intervals * 8 bounds them
  const int32_t n_cols = b.n_intervals * 8;
  const size_t fw = (static_cast<size_t>(n_cols) + 31) / 32;
  unsigned int* words = scratch;
  int32_t* queue = reinterpret_cast<int32_t*>(scratch + fw);
  cudaError_t e = cudaMemsetAsync(words, 0, fw * 4, st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(ctr, 0, sizeof(BvssCounters), st);
  if (e != cudaSuccess) return e;
  if (n_sources > 0)
    frontier_from_sources_kernel<<<(n_sources + 255) / 256, 256, 0, st>>>(sources, n_sources,
                                                                          n_cols, words);
  if (b.n_intervals > 0)
    active_vss_kernel<<<(b.n_intervals + 255) / 256, 256, 0, st>>>(words, b.ptr, b.n_intervals,
                                                                   queue, ctr);
  const int blocks = std::max(1, std::min(4096, (b.n_vss * 32 + 255) / 256));
  discover_pairs_kernel<<<blocks, 256, 0, st>>>(b, n_cols, words, queue, ctr, pairs, max_pairs, d);
  return cudaGetLastError();
}

}  // namespace cpg
