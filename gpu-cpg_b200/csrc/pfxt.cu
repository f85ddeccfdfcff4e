// Prefix tree (PFXT) enumeration for sm_100a.
//
// The reference's G-PathGen (gpucpg/gpucpg.cu:19134-20850, kernels
// expand_short_pile 3234-3306) expands every "short" path by walking its whole
// suffix chain and emitting one child per deviation edge, then sorts the short
// pile.  Here the same path set is enumerated through the deviation heaps the
// SFXT kernel built: a path is "parent + one deviation", and a deviation's
// path-graph neighbours are the next deviations in heap order, so every
// accepted path writes at most five candidate children instead of one per
// deviation edge on its chain.  The closure below accepts every candidate
// whose cost is <= lim; the host raises lim (the reference's "split") until at
// least K non-zero paths cost <= split.
//
// Child cost: new_slack = slack + dist_neighbor + wgt - dist_v with
// dist = (float)fixed/SCALE_UP, evaluated left to right exactly as
// expand_short_pile writes it (gpucpg.cu:3271-3276).  This file is compiled
// with --use_fast_math like the reference, so the REFERENCE division mode
// produces the reference's device quotients; IEEE mode uses __fdiv_rn.
#include <climits>

#include "pfxt_device.cuh"

namespace cpg {

namespace {

constexpr int kClosureThreads = 256;

// Route one candidate (all lanes call): cost <= lim goes to the next
// frontier, the rest to the pending pile.
__device__ __forceinline__ void route(const ClosureParams& p, Item* out,
                                      unsigned long long* out_cnt, bool exists,
                                      const Item& it) {
  const bool take = exists && it.cost <= p.lim;
  const bool defer = exists && !take;
  const unsigned long long a = warp_append(out_cnt, take);
  if (take) {
    if (a < p.front_cap) out[a] = it;
    else atomicCAS(&p.ctr->err, kDevOk, kDevCapacity);
  }
  const unsigned long long b = warp_append(&p.ctr->pend_out, defer);
  if (defer) {
    if (b < p.pend_cap) p.pend[b] = it;
    else atomicCAS(&p.ctr->err, kDevOk, kDevCapacity);
  }
}

__global__ void __launch_bounds__(kClosureThreads)
closure_kernel(ClosureParams p) {
  const unsigned long long tid =
      static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned long long nthreads =
      static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  int r = 0;
  for (;;) {
    volatile unsigned long long* fc = p.ctr->frontier;
    const unsigned long long n_cur = fc[r % 3];
    if (n_cur == 0) break;
    if (n_cur > p.front_cap) {  // an overflow was recorded last round
      atomicCAS(&p.ctr->err, kDevOk, kDevCapacity);
      break;
    }
    const Item* in = p.front[r & 1];
    Item* out = p.front[(r + 1) & 1];
    unsigned long long* out_cnt = &p.ctr->frontier[(r + 1) % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctr->frontier[(r + 2) % 3] = 0;
    const unsigned long long n_pad = (n_cur + 31) & ~31ull;
    for (unsigned long long i = tid; i < n_pad; i += nthreads) {
      const bool valid = i < n_cur;
      Item it;
      it.cost = 0.f;
      it.parent = -1;
      it.node = -1;
      it.j = 0;
      if (valid) {
        const int4 raw = __ldcg(reinterpret_cast<const int4*>(in + i));
        it.cost = __int_as_float(raw.x);
        it.parent = raw.y;
        it.node = raw.z;
        it.j = raw.w;
      }
      // accept: materialise the path
      const unsigned long long q = warp_append(&p.ctr->paths, valid);
      bool stored = false;
      int to = -1;
      HeapNode hn;
      hn.vtx = -1;
      hn.left = -1;
      hn.right = -1;
      hn.row = 0;
      hn.head = -1;
      hn.w = 0.f;
      hn.dist_head = 0;
      hn.dist_v = 0;
      if (valid) {
        int from = -1, level = 0;
        if (it.node <= -2) {
          to = -(it.node + 2);
        } else {
          hn = load_node(p.g.hnodes, it.node);
          from = hn.vtx;
          to = dev_head(p.g, hn, it.j);
          level = __ldcg(p.ps.level + it.parent) + 1;
        }
        if (q < p.ps.cap) {
          p.ps.cost[q] = it.cost;
          p.ps.parent[q] = it.parent;
          p.ps.from[q] = from;
          p.ps.to[q] = to;
          p.ps.level[q] = level;
          stored = true;
        } else {
          atomicCAS(&p.ctr->err, kDevOk, kDevCapacity);
        }
      }
      // A path costing exactly the final split is reported but not expanded:
      // its descendants cost at least as much, so with tied costs (integer
      // delays) they could only add to the tie group at the split.
      const bool expand = stored && !(it.cost == p.tie);
      const bool sib = expand && it.node >= 0;
      const float pcost = sib ? __ldcg(p.ps.cost + it.parent) : 0.f;
      // siblings: heap children of this deviation among the parent's options
      {
        Item c;
        c.parent = it.parent;
        bool ex;
        // first child: chain-heap left (j == 0) or list child 2j+1
        c.node = it.j == 0 ? hn.left : it.node;
        c.j = it.j == 0 ? 0 : 2 * it.j + 1;
        ex = sib && (it.j == 0 ? cand_top(p.g, c.node, pcost, c.cost)
                               : cand_row(p.g, hn, c.j, pcost, c.cost));
        route(p, out, out_cnt, ex, c);
        c.node = it.j == 0 ? hn.right : it.node;
        c.j = it.j == 0 ? 0 : 2 * it.j + 2;
        ex = sib && (it.j == 0 ? cand_top(p.g, c.node, pcost, c.cost)
                               : cand_row(p.g, hn, c.j, pcost, c.cost));
        route(p, out, out_cnt, ex, c);
        c.node = it.node;
        c.j = 1;
        ex = sib && it.j == 0 && cand_row(p.g, hn, c.j, pcost, c.cost);
        route(p, out, out_cnt, ex, c);
        c.j = 2;
        ex = sib && it.j == 0 && cand_row(p.g, hn, c.j, pcost, c.cost);
        route(p, out, out_cnt, ex, c);
      }
      // cross: the cheapest deviation on the new path's own suffix chain
      {
        Item c;
        c.parent = static_cast<int>(q);
        c.node = expand ? __ldg(p.g.ht_root + to) : -1;
        c.j = 0;
        const bool ex = expand && cand_top(p.g, c.node, it.cost, c.cost);
        route(p, out, out_cnt, ex, c);
      }
    }
    if (!grid_sync(&p.ctr->bar, &p.ctr->err, p.spin_limit)) return;
    ++r;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) p.ctr->rounds += r;
}

__global__ void seed_roots_kernel(const int32_t* srcs, int32_t n_srcs,
                                  const int32_t* dist, Item* pend,
                                  PfxtCounters* ctr) {
  const int base = blockIdx.x * blockDim.x;
  const int i = base + threadIdx.x;
  bool ok = false;
  Item it;
  if (i < n_srcs) {
    const int s = srcs[i];
    const int d = dist[s];
    if (d != INT_MAX) {
      ok = true;
      // root seeding is host code in the reference: (float)dist/SCALE_UP with
      // IEEE division (gpucpg.cu:18502-18520)
      it.cost = __fdiv_rn(static_cast<float>(d), 10000.0f);
      it.parent = -1;
      it.node = -2 - s;
      it.j = 0;
    }
  }
  const unsigned long long slot = warp_append(&ctr->pend_out, ok);
  if (ok) pend[slot] = it;
}

__global__ void promote_kernel(const Item* in, unsigned long long n, float lim,
                               Item* front, unsigned long long front_cap,
                               Item* pend_out, unsigned long long pend_cap,
                               PfxtCounters* ctr) {
  const unsigned long long stride =
      static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  const unsigned long long n_pad = (n + 31) & ~31ull;
  for (unsigned long long i =
           static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
       i < n_pad; i += stride) {
    const bool valid = i < n;
    Item it;
    it.cost = 0.f;
    if (valid) it = in[i];
    const bool take = valid && it.cost <= lim;
    const bool keep = valid && !take;
    const unsigned long long a = warp_append(&ctr->frontier[0], take);
    if (take) {
      if (a < front_cap) front[a] = it;
      else atomicCAS(&ctr->err, kDevOk, kDevCapacity);
    }
    const unsigned long long b = warp_append(&ctr->pend_out, keep);
    if (keep) {
      if (b < pend_cap) pend_out[b] = it;
      else atomicCAS(&ctr->err, kDevOk, kDevCapacity);
    }
  }
}

}  // namespace

int launch_closure(const ClosureParams& p, int device, void* stream,
                   int* grid_out) {
  int sms = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, closure_kernel,
                                                    kClosureThreads, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  const int grid = sms * per_sm;
  if (grid_out) *grid_out = grid;
  ClosureParams pp = p;
  void* args[] = {&pp};
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(closure_kernel),
                                     dim3(grid), dim3(kClosureThreads), args, 0,
                                     static_cast<cudaStream_t>(stream));
}

int launch_seed_roots(const int32_t* srcs, int32_t n_srcs, const int32_t* dist,
                      Item* pend, PfxtCounters* ctr, void* stream) {
  if (n_srcs <= 0) return cudaSuccess;
  const int threads = 256;
  const int blocks = (n_srcs + threads - 1) / threads;
  seed_roots_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(
      srcs, n_srcs, dist, pend, ctr);
  return cudaGetLastError();
}

int launch_promote(const Item* pend_in, unsigned long long n_in, float lim,
                   Item* front, unsigned long long front_cap, Item* pend_out,
                   unsigned long long pend_cap, PfxtCounters* ctr,
                   void* stream) {
  if (n_in == 0) return cudaSuccess;
  const int threads = 256;
  unsigned long long blocks = (n_in + threads - 1) / threads;
  if (blocks > 148ull * 16) blocks = 148ull * 16;
  promote_kernel<<<static_cast<unsigned>(blocks), threads, 0,
                   static_cast<cudaStream_t>(stream)>>>(
      pend_in, n_in, lim, front, front_cap, pend_out, pend_cap, ctr);
  return cudaGetLastError();
}

}  // namespace cpg
