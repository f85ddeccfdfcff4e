// Device-side graph construction from an uploaded fan-out CSR: the 8-byte
// (head, delay) edge words, the fan-in CSR (counting sort by head: in-degree
// histogram, scan, scatter) and the source list (in-degree 0).  Replaces the
// host loops of the reference's read_input (gpucpg/gpucpg.cu:500-541), so a
// caller that hands over a CSR pays one H2D copy, not an O(M) host pass.
#include "device_common.cuh"

namespace cpg {

namespace {

constexpr int kScanTile = 2048;

// The (head, delay) edge words and the in-degree histogram in one pass over
// the heads.  Also validates the heads: one outside [0, n) sets *bad and is
// skipped, so the host learns of it after the build without an O(M) host
// pass.
__global__ void interleave_indegree_kernel(const int32_t* adj, const float* w, int64_t m,
                                           int32_t n, DevEdge* out, int32_t* indeg,
                                           int32_t* bad) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < m;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    DevEdge d;
    d.head = adj[e];
    d.w = w[e];
    out[e] = d;
    if (static_cast<unsigned>(d.head) >= static_cast<unsigned>(n)) {
      *bad = 1;
      continue;
    }
    atomicAdd(&indeg[d.head], 1);
  }
}

// exclusive scan of x[0..n) into y[0..n], y[n] = total; three-kernel
// reduce-then-scan over kScanTile-element tiles
__global__ void tile_sum_kernel(const int32_t* x, int64_t n, int32_t* sums) {
  __shared__ int32_t ws[32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
  int32_t s = 0;
  for (int t = threadIdx.x; t < kScanTile; t += blockDim.x)
    if (base + t < n) s += x[base + t];
  s = __reduce_add_sync(0xffffffffu, s);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t tot = 0;
    for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) tot += ws[i];
    sums[blockIdx.x] = tot;
  }
}

// exclusive scan of the tile sums in place (one CTA of 1024), sums[n] = total
__global__ void __launch_bounds__(1024) scan_sums_kernel(int32_t* sums, int n) {
  __shared__ int32_t wsum[32];
  __shared__ int32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int b0 = 0; b0 < n; b0 += blockDim.x) {
    const int i = b0 + threadIdx.x;
    const int32_t v = i < n ? sums[i] : 0;
    int32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const int32_t a = wsum[lane];
      int32_t y = a;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t z = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) y += z;
      }
      wsum[lane] = y - a;
    }
    __syncthreads();
    const int32_t c0 = carry;
    if (i < n) sums[i] = c0 + wsum[wid] + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = c0 + wsum[wid] + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[n] = carry;
}

__global__ void tile_scan_kernel(const int32_t* x, int64_t n, const int32_t* sums,
                                 int32_t* y) {
  __shared__ int32_t buf[kScanTile];
  __shared__ int32_t wsum[32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
  constexpr int per = kScanTile / 256;  // blockDim.x == 256
  int32_t vals[per];
  int32_t run = 0;
  for (int i = 0; i < per; ++i) {
    const int64_t g = base + threadIdx.x * per + i;
    vals[i] = g < n ? x[g] : 0;
    run += vals[i];
  }
  // exclusive scan of the per-thread totals
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int32_t incl = run;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t acc = 0;
    for (int i = 0; i < 8; ++i) {
      const int32_t v = wsum[i];
      wsum[i] = acc;
      acc += v;
    }
  }
  __syncthreads();
  int32_t pre = sums[blockIdx.x] + wsum[wid] + incl - run;
  for (int i = 0; i < per; ++i) {
    const int64_t g = base + threadIdx.x * per + i;
    if (g < n) y[g] = pre;
    pre += vals[i];
  }
  (void)buf;
}

__global__ void set_last_kernel(int32_t* y, int64_t n, const int32_t* sums, int ntiles) {
  y[n] = sums[ntiles];
}

// warp per tail vertex: each fan-out edge (u, h) lands in h's fan-in row
__global__ void fanin_scatter_kernel(const int32_t* adjp, const int32_t* adj, int32_t n,
                                     int32_t* fill, int32_t* iadj) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int u = gw; u < n; u += nw) {
    for (int e = adjp[u] + lane; e < adjp[u + 1]; e += 32) {
      const int h = adj[e];
      if (static_cast<unsigned>(h) >= static_cast<unsigned>(n)) continue;  // reported
      iadj[atomicAdd(&fill[h], 1)] = u;
    }
  }
}

__global__ void sources_kernel(const int32_t* indeg, int32_t n, int32_t* srcs,
                               int32_t* count) {
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int v = base + threadIdx.x;
    const bool src = v < n && indeg[v] == 0;
    const int slot = warp_append(count, src);
    if (src) srcs[slot] = v;
  }
}

// Blocks for n threads' worth of work: one element per thread (short blocks,
// so a build running beside another stream's kernels gives SMs back soon),
// capped far above what the loops need.
int grid_of(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (int64_t{1} << 20)) b = int64_t{1} << 20;
  return static_cast<int>(b);
}

}  // namespace

size_t build_scratch_words(int32_t n) {
  // indeg/fill (n) + tile sums
  return static_cast<size_t>(n) + (static_cast<size_t>(n) + kScanTile) / kScanTile + 2;
}

// adj/w: uploaded fan-out heads and delays; outputs edges, iadjp (n+1), iadj
// (m), srcs (n), n_srcs[0] (source count) and n_srcs[1] (1 if a head lies
// outside [0, n)).  scratch: build_scratch_words(n) ints.
int launch_build_graph(const int32_t* adjp, const int32_t* adj, const float* w,
                       int32_t n, int64_t m, DevEdge* edges, int32_t* iadjp,
                       int32_t* iadj, int32_t* srcs, int32_t* n_srcs,
                       int32_t* scratch, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int32_t* indeg = scratch;
  int32_t* sums = scratch + n;
  const int ntiles = static_cast<int>((static_cast<int64_t>(n) + kScanTile - 1) / kScanTile);
  cudaMemsetAsync(indeg, 0, static_cast<size_t>(n) * 4, s);
  cudaMemsetAsync(n_srcs, 0, 8, s);  // source count, bad-head flag
  if (m > 0)
    interleave_indegree_kernel<<<grid_of(m, 256), 256, 0, s>>>(adj, w, m, n, edges, indeg,
                                                               n_srcs + 1);
  if (n > 0) {
    tile_sum_kernel<<<ntiles, 256, 0, s>>>(indeg, n, sums);
    scan_sums_kernel<<<1, 1024, 0, s>>>(sums, ntiles);
    tile_scan_kernel<<<ntiles, 256, 0, s>>>(indeg, n, sums, iadjp);
    set_last_kernel<<<1, 1, 0, s>>>(iadjp, n, sums, ntiles);
    sources_kernel<<<grid_of(n, 256), 256, 0, s>>>(indeg, n, srcs, n_srcs);
    // reuse indeg as the scatter cursor
    cudaMemcpyAsync(indeg, iadjp, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToDevice, s);
    if (m > 0)
      fanin_scatter_kernel<<<grid_of(static_cast<int64_t>(n) * 32, 256), 256, 0, s>>>(
          adjp, adj, n, indeg, iadj);
  } else {
    cudaMemsetAsync(iadjp, 0, 4, s);
  }
  return cudaGetLastError();
}

}  // namespace cpg
