// Suffix tree (SFXT) for sm_100a: reverse levelisation, fixed-point relax,
// successors, sorted deviation lists and persistent chain heaps, all in one
// persistent cooperative kernel that walks the levels with a bounded grid
// barrier between them (no host round trip per level).
//
// Reference behaviour reproduced (gpucpg/gpucpg.cu):
//   levelize   bfs_td_step_privatized 2215-2283, loop 17642-17677: Kahn over
//              the fan-in CSR, deps = out-degree, sinks are level 0
//   relax      relax_bu_step 1167-1188: dist[v] = min dist[n] + (int)(w*10000)
//   successor  update_successors_bu 2606-2628: largest n among the arg-mins
// The deviation lists restate the reference's static deviation CSR
// (tc_pfxt_candidates.cuh:713-750: every fan-out edge except the successor
// edge, with its cost delta), sorted by delta.
//
// This file is compiled with --use_fast_math like the reference library.
#include <climits>

#include "bvss.cuh"
#include "device_common.cuh"

namespace cpg {

namespace {

__device__ __forceinline__ bool heap_less(int va, float ka, int vb, float kb) {
  return ka < kb || (ka == kb && va < vb);
}

// Cost increase of deviation (v, head) in delay units.  Exact integer and
// delay parts are summed in double so ties between deviations stay ties.
__device__ __forceinline__ float deviation_key(int dist_head, int dist_v,
                                               float w) {
  const double d = (static_cast<double>(dist_head) - static_cast<double>(dist_v)) +
                   static_cast<double>(w) * 10000.0;
  return static_cast<float>(d * 1e-4);
}

__device__ __forceinline__ int fixed_delay(float w) {
  // relax_bu_step: const int wgt = owgts[e]*SCALE_UP;
  const int wgt = w * kScaleUp;
  return wgt;
}

// One warp builds vertex v at level lvl: fixed-point distance, successor,
// its deviation list (unsorted here; sort_rows_kernel orders it), its chain
// heap, and the Kahn step for its fan-in neighbours.
constexpr int kRegChunks = kSmemRow / 32;  // rows up to this many 32-edge chunks
                                          // stay in registers

// (key, position) word ordering a deviation row: ascending exact key, ties
// in edge order.
__device__ __forceinline__ unsigned long long sort_word(float key, int idx) {
  return (static_cast<unsigned long long>(float_key(key)) << 32) |
         static_cast<unsigned>(idx);
}

// The cheapest deviation of a row too long to sort in registers, tracked per
// lane while the row is built: the least (key, edge position) word and its
// record.  best_reduce gives every lane the row's first entry once sorted.
struct BestDev {
  unsigned long long word;
  DevSidetrack rec;
};

__device__ __forceinline__ BestDev best_none() {
  BestDev b;
  b.word = ~0ull;
  b.rec.head = -1;
  b.rec.w = 0.f;
  b.rec.dist_head = 0;
  b.rec.key = 0.f;
  return b;
}

__device__ __forceinline__ void best_take(BestDev& b, bool valid, const DevSidetrack& rec,
                                          int pos) {
  const unsigned long long x = sort_word(rec.key, pos);
  if (valid && x < b.word) {
    b.word = x;
    b.rec = rec;
  }
}

__device__ __forceinline__ DevSidetrack best_reduce(const BestDev& b) {
  unsigned long long m = b.word;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, m, o);
    m = y < m ? y : m;
  }
  const unsigned own = __ballot_sync(0xffffffffu, b.word == m);
  const int src = __ffs(own) - 1;
  DevSidetrack r;
  r.head = __shfl_sync(0xffffffffu, b.rec.head, src);
  r.w = __shfl_sync(0xffffffffu, b.rec.w, src);
  r.dist_head = __shfl_sync(0xffffffffu, b.rec.dist_head, src);
  r.key = __shfl_sync(0xffffffffu, b.rec.key, src);
  return r;
}

// Bitonic sort of one word per lane across the warp, ascending by lane.
__device__ __forceinline__ unsigned long long warp_sort32(unsigned long long x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, j);
      const bool up = (lane & k) == 0;
      const bool lower = (lane & j) == 0;
      x = (lower == up) ? (x < y ? x : y) : (x > y ? x : y);
    }
  }
  return x;
}

// Bitonic sort of 32 C words held C per lane (element c 32 + lane in x[c]),
// ascending: exchanges with j >= 32 stay inside a lane, the others are
// shuffles.
template <int C>
__device__ __forceinline__ void warp_sort_regs(unsigned long long (&x)[C]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 2; k <= 32 * C; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const int jc = j >> 5;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const int d = c ^ jc;
          if (d > c) {
            const bool up = ((c * 32) & k) == 0;
            const unsigned long long a = x[c], b = x[d];
            if ((a > b) == up) {
              x[c] = b;
              x[d] = a;
            }
          }
        }
      } else {
        const bool lower = (lane & j) == 0;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const unsigned long long y = __shfl_xor_sync(0xffffffffu, x[c], j);
          const bool up = ((c * 32 + lane) & k) == 0;
          x[c] = (lower == up) ? (x[c] < y ? x[c] : y) : (x[c] > y ? x[c] : y);
        }
      }
    }
  }
}

// A row the build left unsorted, for sort_rows_kernel.
__device__ __forceinline__ void list_long_row(const SfxtParams& p, int v) {
  p.long_rows[atomicAdd(&p.ctr->n_long, 1)] = v;
}

// C sort words a lane: the row's (key, position) words sorted in registers,
// then every lane reads the records of its C output slots before any is
// written.
template <int C>
__device__ __forceinline__ void sort_row_words(DevSidetrack* row, int cnt) {
  const int lane = threadIdx.x & 31;
  unsigned long long x[C];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int t = c * 32 + lane;
    x[c] = t < cnt ? sort_word(__ldcg(&row[t].key), t) : ~0ull;
  }
  warp_sort_regs<C>(x);
  DevSidetrack o[C];
#pragma unroll
  for (int c = 0; c < C; ++c)
    if (c * 32 + lane < cnt) o[c] = row[static_cast<int>(x[c] & 0xffffffffu)];
  __syncwarp();
#pragma unroll
  for (int c = 0; c < C; ++c)
    if (c * 32 + lane < cnt) row[c * 32 + lane] = o[c];
  __syncwarp();
}

// Sorts a deviation row of at most 128 entries by (key, position) in
// registers: one word a lane up to 32 entries, four up to 128.  All lanes
// call.
__device__ __forceinline__ void sort_row_regs(DevSidetrack* row, int cnt) {
  const int lane = threadIdx.x & 31;
  if (cnt <= 32) {
    DevSidetrack r;
    unsigned long long x = ~0ull;
    if (lane < cnt) {
      r = row[lane];
      x = sort_word(r.key, lane);
    }
    x = warp_sort32(x);
    // lane i now holds the i-th smallest; fetch that record from its lane
    const int src = static_cast<int>(x & 0xffffffffu);
    DevSidetrack o;
    o.head = __shfl_sync(0xffffffffu, r.head, src & 31);
    o.w = __shfl_sync(0xffffffffu, r.w, src & 31);
    o.dist_head = __shfl_sync(0xffffffffu, r.dist_head, src & 31);
    o.key = __shfl_sync(0xffffffffu, r.key, src & 31);
    if (lane < cnt) row[lane] = o;
    return;
  }
  sort_row_words<4>(row, cnt);
}

// A row of at most 32 edges (one per lane) is sorted in registers and
// written once, in order (write_row64 does the same up to 64 edges); longer
// rows are written in edge order and sorted by sort_rows_kernel.  Returns the
// number of deviations written; lane 0's top is the first of them.
__device__ __forceinline__ int write_short_row(const SfxtParams& p, int rb, bool valid,
                                               const DevSidetrack& rec, DevSidetrack& top) {
  const int lane = threadIdx.x & 31;
  const unsigned bal = __ballot_sync(0xffffffffu, valid);
  const unsigned long long x = warp_sort32(valid ? sort_word(rec.key, lane) : ~0ull);
  const int src = static_cast<int>(x & 31u);
  DevSidetrack o;
  o.head = __shfl_sync(0xffffffffu, rec.head, src);
  o.w = __shfl_sync(0xffffffffu, rec.w, src);
  o.dist_head = __shfl_sync(0xffffffffu, rec.dist_head, src);
  o.key = __shfl_sync(0xffffffffu, rec.key, src);
  const int cnt = __popc(bal);
  if (lane < cnt) p.dev[rb + lane] = o;
  top = o;
  return cnt;
}

// Rows of 33..64 edges: two words per lane (element i = 32 * chunk + lane),
// one 64-element bitonic network (partners across chunks swap in
// registers), then each sorted slot fetches its record from the lane and
// chunk it came from.
__device__ __forceinline__ int write_row64(const SfxtParams& p, int rb, bool v0,
                                           const DevSidetrack& r0, bool v1,
                                           const DevSidetrack& r1, DevSidetrack& top) {
  const int lane = threadIdx.x & 31;
  const unsigned b0 = __ballot_sync(0xffffffffu, v0);
  const unsigned b1 = __ballot_sync(0xffffffffu, v1);
  unsigned long long x[2] = {v0 ? sort_word(r0.key, lane) : ~0ull,
                             v1 ? sort_word(r1.key, 32 + lane) : ~0ull};
#pragma unroll
  for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j == 32) {  // only at k == 64: ascending across the chunks
        const unsigned long long lo = x[0] < x[1] ? x[0] : x[1];
        const unsigned long long hi = x[0] < x[1] ? x[1] : x[0];
        x[0] = lo;
        x[1] = hi;
      } else {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int i = 32 * c + lane;
          const unsigned long long y = __shfl_xor_sync(0xffffffffu, x[c], j);
          const bool up = (i & k) == 0;
          const bool lower = (i & j) == 0;
          x[c] = (lower == up) ? (x[c] < y ? x[c] : y) : (x[c] > y ? x[c] : y);
        }
      }
    }
  }
  const int cnt = __popc(b0) + __popc(b1);
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const int src = static_cast<int>(x[c] & 63u);
    const int sl = src & 31;
    const bool hi = src >= 32;
    DevSidetrack o;
    const int h0 = __shfl_sync(0xffffffffu, r0.head, sl), h1 = __shfl_sync(0xffffffffu, r1.head, sl);
    const float w0 = __shfl_sync(0xffffffffu, r0.w, sl), w1 = __shfl_sync(0xffffffffu, r1.w, sl);
    const int d0 = __shfl_sync(0xffffffffu, r0.dist_head, sl), d1 = __shfl_sync(0xffffffffu, r1.dist_head, sl);
    const float k0 = __shfl_sync(0xffffffffu, r0.key, sl), k1 = __shfl_sync(0xffffffffu, r1.key, sl);
    o.head = hi ? h1 : h0;
    o.w = hi ? w1 : w0;
    o.dist_head = hi ? d1 : d0;
    o.key = hi ? k1 : k0;
    const int i = 32 * c + lane;
    if (i < cnt) p.dev[rb + i] = o;
    if (c == 0) top = o;
  }
  return cnt;
}

__device__ __forceinline__ int cand_dist(int dh, float w) {
  return static_cast<int>(static_cast<unsigned>(dh) + static_cast<unsigned>(fixed_delay(w)));
}

// Successor tie-break on relabelled graphs (p.orig_id set): among the heads
// that tie for the least distance, the one with the largest caller id, as
// update_successors_bu picks it (gpucpg.cu:2606-2628).  The word orders by
// caller id and carries the head's own id; 0 is "none".  Ties are rare, so
// the callers read caller ids only when more than one head ties.
__device__ __forceinline__ unsigned long long succ_word(const SfxtParams& p, int head) {
  return (static_cast<unsigned long long>(static_cast<unsigned>(__ldg(p.orig_id + head)) + 1u)
          << 32) |
         static_cast<unsigned>(head);
}

template <int G>
__device__ __forceinline__ unsigned long long group_max_u64(unsigned long long x) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o, G);
    x = y > x ? y : x;
  }
  return x;
}

// kLevel (dataflow build): the level is not known in advance; it is one
// more than the heads' highest level (0 for a sink), read with their
// distances, and written to level_of[v].  Returns the level.
template <bool kLevel = false>
__device__ int build_vertex(const SfxtParams& p, int v, int lvl, bool do_kahn) {
  const int lane = threadIdx.x & 31;
  const int rb = p.adjp[v];
  const int re = p.adjp[v + 1];
  if (kLevel) lvl = re == rb ? 0 : 1;  // the exact value follows; only 0 matters below
  int best = INT_MAX;
  int s = -1;
  int cnt = 0;
  DevSidetrack top;  // the cheapest deviation (lane 0's copy is used)
  top.head = -1;
  if (re - rb <= kRegChunks * 32) {
    // the whole row in registers: every edge word, then every head distance,
    // is requested before any is used, so a long row costs about two memory
    // round trips instead of one per 32-edge chunk
    DevEdge ed[kRegChunks];
    int dh[kRegChunks];
#pragma unroll
    for (int c = 0; c < kRegChunks; ++c) {
      const int e = rb + c * 32 + lane;
      ed[c].head = -1;
      ed[c].w = 0.f;
      if (e < re) ed[c] = p.edges[e];
    }
#pragma unroll
    for (int c = 0; c < kRegChunks; ++c) dh[c] = ed[c].head >= 0 ? __ldcg(p.dist + ed[c].head) : INT_MAX;
    if (kLevel) {
      int lmax = -1;
#pragma unroll
      for (int c = 0; c < kRegChunks; ++c)
        if (ed[c].head >= 0) lmax = max(lmax, __ldcg(p.level_of + ed[c].head));
      lvl = warp_max_i(lmax) + 1;
    }
    if (lvl == 0) {
      best = 0;  // sinks (out-degree 0) start at distance 0 (gpucpg.cu:17034-17038)
    } else {
#pragma unroll
      for (int c = 0; c < kRegChunks; ++c)
        if (ed[c].head >= 0) best = min(best, cand_dist(dh[c], ed[c].w));
      best = warp_min_i(best);
      int nt = 0;  // this lane's tied heads
#pragma unroll
      for (int c = 0; c < kRegChunks; ++c)
        if (ed[c].head >= 0 && cand_dist(dh[c], ed[c].w) == best) {
          s = max(s, ed[c].head);
          ++nt;
        }
      if (p.orig_id && __reduce_add_sync(0xffffffffu, nt) > 1) {
        unsigned long long k = 0;
#pragma unroll
        for (int c = 0; c < kRegChunks; ++c)
          if (ed[c].head >= 0 && cand_dist(dh[c], ed[c].w) == best) {
            const unsigned long long x = succ_word(p, ed[c].head);
            k = x > k ? x : k;
          }
        s = static_cast<int>(group_max_u64<32>(k) & 0xffffffffu);
      } else {
        s = warp_max_i(s);
      }
    }
    // deviations: fan-out edges whose head is not the successor and has a
    // finite distance, compacted in edge order into v's own fan-out slots
    // (a row of at most 64 edges already sorted)
    if (re - rb <= 32) {
      const bool valid = ed[0].head >= 0 && ed[0].head != s && dh[0] != INT_MAX;
      DevSidetrack rec;
      rec.head = ed[0].head;
      rec.w = ed[0].w;
      rec.dist_head = dh[0];
      rec.key = deviation_key(dh[0], best, ed[0].w);
      cnt = write_short_row(p, rb, valid, rec, top);
    } else if (re - rb <= 64) {
      DevSidetrack r[2];
      bool v[2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        v[c] = ed[c].head >= 0 && ed[c].head != s && dh[c] != INT_MAX;
        r[c].head = ed[c].head;
        r[c].w = ed[c].w;
        r[c].dist_head = dh[c];
        r[c].key = deviation_key(dh[c], best, ed[c].w);
      }
      cnt = write_row64(p, rb, v[0], r[0], v[1], r[1], top);
    } else {
      BestDev bd = best_none();
#pragma unroll
      for (int c = 0; c < kRegChunks; ++c) {
        if (rb + c * 32 >= re) break;
        const bool valid = ed[c].head >= 0 && ed[c].head != s && dh[c] != INT_MAX;
        const unsigned bal = __ballot_sync(0xffffffffu, valid);
        if (valid) {
          DevSidetrack rec;
          rec.head = ed[c].head;
          rec.w = ed[c].w;
          rec.dist_head = dh[c];
          rec.key = deviation_key(dh[c], best, ed[c].w);
          p.dev[rb + cnt + __popc(bal & lanemask_lt())] = rec;
          best_take(bd, true, rec, c * 32 + lane);
        }
        cnt += __popc(bal);
      }
      top = best_reduce(bd);
    }
  } else {
    // long rows (a super-source, say): chunk by chunk
    if (kLevel) {
      int lmax = -1;
      for (int e = rb + lane; e < re; e += 32) lmax = max(lmax, __ldcg(p.level_of + p.edges[e].head));
      lvl = warp_max_i(lmax) + 1;
    }
    if (lvl == 0) {
      best = 0;
    } else {
      for (int e = rb + lane; e < re; e += 32) {
        const DevEdge ed = p.edges[e];
        best = min(best, cand_dist(__ldcg(p.dist + ed.head), ed.w));
      }
      best = warp_min_i(best);
      int nt = 0;
      for (int e = rb + lane; e < re; e += 32) {
        const DevEdge ed = p.edges[e];
        if (cand_dist(__ldcg(p.dist + ed.head), ed.w) == best) {
          s = max(s, ed.head);
          ++nt;
        }
      }
      if (p.orig_id && __reduce_add_sync(0xffffffffu, nt) > 1) {
        unsigned long long k = 0;
        for (int e = rb + lane; e < re; e += 32) {
          const DevEdge ed = p.edges[e];
          if (cand_dist(__ldcg(p.dist + ed.head), ed.w) == best) {
            const unsigned long long x = succ_word(p, ed.head);
            k = x > k ? x : k;
          }
        }
        s = static_cast<int>(group_max_u64<32>(k) & 0xffffffffu);
      } else {
        s = warp_max_i(s);
      }
    }
    BestDev bd = best_none();
    for (int base = rb; base < re; base += 32) {
      const int e = base + lane;
      bool valid = false;
      DevSidetrack rec;
      if (e < re) {
        const DevEdge ed = p.edges[e];
        const int dh = __ldcg(p.dist + ed.head);
        valid = ed.head != s && dh != INT_MAX;
        rec.head = ed.head;
        rec.w = ed.w;
        rec.dist_head = dh;
        rec.key = deviation_key(dh, best, ed.w);
      }
      const unsigned bal = __ballot_sync(0xffffffffu, valid);
      if (valid) p.dev[rb + cnt + __popc(bal & lanemask_lt())] = rec;
      best_take(bd, valid, rec, e - rb);
      cnt += __popc(bal);
    }
    top = best_reduce(bd);
  }

  if (lane == 0) {
    p.dist[v] = best;
    p.succ[v] = s;
    p.dev_cnt[v] = cnt;
    if (re - rb > 64 && cnt > 1 && cnt <= kSmemRow) list_long_row(p, v);
    // the chain-heap insert, one level later, takes v's cheapest deviation
    if (cnt > 0) p.best[v] = top;
    if (kLevel) p.level_of[v] = lvl;
  }

  if (do_kahn) {
    // every fan-in neighbour loses one pending fan-out; the last one to
    // reach zero joins the next level.  Up to four chunks of fan-in are
    // loaded and decremented before any result is used.
    const int ib = p.iadjp[v];
    const int ie = p.iadjp[v + 1];
    for (int base = ib; base < ie; base += 4 * 32) {
      int u[4];
      bool ready[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int e = base + c * 32 + lane;
        u[c] = e < ie ? p.iadj[e] : -1;
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) ready[c] = u[c] >= 0 && atomicSub(&p.deps[u[c]], 1) == 1;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int slot = warp_append(&p.ctr->tail, ready[c]);
        if (ready[c]) {
          p.order[slot] = u[c];
          p.level_of[u[c]] = lvl + 1;
        }
      }
    }
  }
  return lvl;
}

// Level-synchronous builds of short rows: a warp builds four vertices at
// once, one per 8-lane group (rows of at most 8 edges), or two, one per
// 16-lane group (at most 16), so a level of low-degree vertices costs a
// fraction of the warp passes.

template <int G>
__device__ __forceinline__ int group_min_i(int x) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) x = min(x, __shfl_xor_sync(0xffffffffu, x, o, G));
  return x;
}

template <int G>
__device__ __forceinline__ int group_max_i(int x) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o, G));
  return x;
}

// Position of the k-th (from 0) set bit of m; k < popc(m).
__device__ __forceinline__ int kth_set_bit(unsigned m, int k) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    const int c = __popc(m & ((1u << w) - 1u));
    if (k >= c) {
      k -= c;
      m >>= w;
      pos += w;
    }
  }
  return pos;
}

// Builds vertex v (< 0: none) of each G-lane group, whose row has at most G
// edges, at level lvl: the same distance, successor, sorted deviation row and
// Kahn step as build_vertex.  Every lane of the warp calls.
template <int G>
__device__ void build_group(const SfxtParams& p, int v, int lvl, bool do_kahn) {
  const int lane = threadIdx.x & 31;
  const int l = lane & (G - 1), g = lane / G;
  const bool has_v = v >= 0;
  // The build's loads and the Kahn step's are independent, so each round
  // trip carries both: the row and fan-in ranges, then the row's edge and
  // the first fan-in tail, then the head's distance and that tail's
  // decrement.
  int rb = 0, re = 0, ib = 0, ie = 0;
  if (has_v) {
    rb = p.adjp[v];
    re = p.adjp[v + 1];
    if (do_kahn) {
      ib = p.iadjp[v];
      ie = p.iadjp[v + 1];
    }
  }
  const bool has = has_v && rb + l < re;
  DevEdge ed;
  ed.head = -1;
  ed.w = 0.f;
  if (has) ed = p.edges[rb + l];
  const int u0 = ib + l < ie ? p.iadj[ib + l] : -1;
  const int dh = has ? __ldcg(p.dist + ed.head) : INT_MAX;
  const bool ready0 = u0 >= 0 && atomicSub(&p.deps[u0], 1) == 1;
  int best = group_min_i<G>(has ? cand_dist(dh, ed.w) : INT_MAX);
  if (lvl == 0) best = 0;  // sinks start at distance 0
  const bool tie = has && lvl > 0 && cand_dist(dh, ed.w) == best;
  int s = group_max_i<G>(tie ? ed.head : -1);
  if (p.orig_id) {
    const int gt = __popc((__ballot_sync(0xffffffffu, tie) >> (g * G)) & ((1u << G) - 1u));
    if (__any_sync(0xffffffffu, gt > 1)) {
      const unsigned long long k = group_max_u64<G>(tie && gt > 1 ? succ_word(p, ed.head) : 0ull);
      if (gt > 1) s = static_cast<int>(k & 0xffffffffu);
    }
  }
  // deviations: every edge but the successor's, sorted by (key, position)
  const bool valid = has && ed.head != s && dh != INT_MAX;
  DevSidetrack rec;
  rec.head = ed.head;
  rec.w = ed.w;
  rec.dist_head = dh;
  rec.key = deviation_key(dh, best, ed.w);
  unsigned long long x = valid ? sort_word(rec.key, l) : ~0ull;
#pragma unroll
  for (int k = 2; k <= G; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, j, G);
      const bool up = (l & k) == 0;
      const bool lower = (l & j) == 0;
      x = (lower == up) ? (x < y ? x : y) : (x > y ? x : y);
    }
  }
  const unsigned bal = __ballot_sync(0xffffffffu, valid);
  const int cnt = __popc((bal >> (g * G)) & ((1u << G) - 1u));
  const int src = g * G + static_cast<int>(x & static_cast<unsigned long long>(G - 1));
  DevSidetrack o;
  o.head = __shfl_sync(0xffffffffu, rec.head, src);
  o.w = __shfl_sync(0xffffffffu, rec.w, src);
  o.dist_head = __shfl_sync(0xffffffffu, rec.dist_head, src);
  o.key = __shfl_sync(0xffffffffu, rec.key, src);
  if (has_v && l < cnt) p.dev[rb + l] = o;
  if (has_v && l == 0) {
    p.dist[v] = best;
    p.succ[v] = s;
    p.dev_cnt[v] = cnt;
    if (cnt > 0) p.best[v] = o;  // the row's first entry
  }
  if (do_kahn) {
    // every fan-in neighbour loses one pending fan-out; the last one to
    // reach zero joins the next level (the first G went above)
    const int passes = warp_max_i((ie - ib + G - 1) / G);
    for (int r = 0; r < passes; ++r) {
      const int e = ib + r * G + l;
      const int u = r == 0 ? u0 : (e < ie ? p.iadj[e] : -1);
      const bool ready = r == 0 ? ready0 : u >= 0 && atomicSub(&p.deps[u], 1) == 1;
      const int slot = warp_append(&p.ctr->tail, ready);
      if (ready) {
        p.order[slot] = u;
        p.level_of[u] = lvl + 1;
      }
    }
  }
}

// Whether an incremental build rebuilds v (at level lvl).
__device__ __forceinline__ bool rebuilt(const SfxtParams& p, int v, int lvl) {
  return !p.vgraph || lvl >= __ldg(p.graph_from + __ldg(p.vgraph + v));
}

// Chain heap of v: the heap of succ[v] with v's cheapest deviation inserted
// at position size+1 of a complete binary heap, copying the root-to-position
// path and carrying the larger element down.  One thread per vertex; runs one
// level after v was relaxed, when succ[v]'s heap is complete.
// kPublish: other threads poll ht_size[v] >= 0 for completion (the dataflow
// build), so the root is made visible before the size.
template <bool kPublish>
__device__ __forceinline__ void heap_store(const SfxtParams& p, int v, int root, int size) {
  p.ht_root[v] = root;
  if (kPublish) {
    st_release(p.ht_size + v, size);  // the heap's nodes and root before its size
  } else {
    p.ht_size[v] = size;
  }
}

// Heap nodes for one insert: from the global cursor, or (chunk != nullptr)
// from the calling thread's private chunk of the pool, refilled 64 nodes at
// a time, so concurrent inserts neither contend for the cursor nor share
// cache lines.  Returns ~0 when the pool is exhausted.
constexpr unsigned kHeapChunk = 64;

__device__ __forceinline__ unsigned long long heap_alloc(const SfxtParams& p, unsigned need,
                                                         unsigned long long* chunk) {
  if (!chunk) {
    const unsigned long long a = atomicAdd(&p.ctr->hnode_used, static_cast<unsigned long long>(need));
    return a + need > p.hnode_cap ? ~0ull : a;
  }
  if (chunk[0] + need > chunk[1]) {
    const unsigned grab = need > kHeapChunk ? need : kHeapChunk;
    const unsigned long long a = atomicAdd(&p.ctr->hnode_used, static_cast<unsigned long long>(grab));
    if (a + grab > p.hnode_cap) return ~0ull;
    chunk[0] = a;
    chunk[1] = a + grab;
  }
  const unsigned long long a = chunk[0];
  chunk[0] += need;
  return a;
}

// The element a chain-heap node carries: everything but the child links.
struct HeapElem {
  int32_t vtx, row, head;
  float w;
  int32_t dist_head, dist_v;
  float key;  // deviation_key of the record: the heap order, with vtx
};

__device__ __forceinline__ HeapNode load_heap_node(const HeapNode* h, int i) {
  const int4 a = __ldcg(reinterpret_cast<const int4*>(h + i));
  const int4 b = __ldcg(reinterpret_cast<const int4*>(h + i) + 1);
  HeapNode n;
  n.vtx = a.x;
  n.left = a.y;
  n.right = a.z;
  n.row = a.w;
  n.head = b.x;
  n.w = __int_as_float(b.y);
  n.dist_head = b.z;
  n.dist_v = b.w;
  return n;
}

__device__ __forceinline__ HeapElem elem_of(const HeapNode& n) {
  HeapElem e;
  e.vtx = n.vtx;
  e.row = n.row;
  e.head = n.head;
  e.w = n.w;
  e.dist_head = n.dist_head;
  e.dist_v = n.dist_v;
  e.key = deviation_key(n.dist_head, n.dist_v, n.w);
  return e;
}

__device__ __forceinline__ void store_heap_node(HeapNode* at, const HeapElem& e, int left,
                                                int right) {
  int4* q = reinterpret_cast<int4*>(at);
  q[0] = make_int4(e.vtx, left, right, e.row);
  q[1] = make_int4(e.head, __float_as_int(e.w), e.dist_head, e.dist_v);
}

// What an insert of v needs: its successor's heap and its element.
struct InsertPlan {
  int base_root, base_size;
  bool empty;   // v has no deviation: its heap is its successor's
  HeapElem ce;
};

__device__ __forceinline__ InsertPlan plan_insert(const SfxtParams& p, int v) {
  InsertPlan q;
  const int s = __ldcg(p.succ + v);
  const int cnt = __ldcg(p.dev_cnt + v);
  q.base_root = s >= 0 ? __ldcg(p.ht_root + s) : -1;
  q.base_size = s >= 0 ? __ldcg(p.ht_size + s) : 0;
  q.empty = cnt == 0;
  if (!q.empty) {
    // v's element: its cheapest deviation, as the build left it
    const int4 b = __ldcg(reinterpret_cast<const int4*>(p.best + v));
    q.ce.vtx = v;
    q.ce.row = __ldg(p.adjp + v);
    q.ce.head = b.x;
    q.ce.w = __int_as_float(b.y);
    q.ce.dist_head = b.z;
    q.ce.key = __int_as_float(b.w);
    q.ce.dist_v = __ldcg(p.dist + v);
  }
  return q;
}

// Nodes an insert into a heap of base_size elements copies.
__device__ __forceinline__ unsigned insert_nodes(int base_size) {
  return static_cast<unsigned>(31 - __clz(static_cast<unsigned>(base_size) + 1u)) + 1u;
}

// The insert itself, into nodes a .. a + depth already taken from the pool.
template <bool kPublish>
__device__ __forceinline__ void heap_insert_at(const SfxtParams& p, int v, const InsertPlan& q,
                                               unsigned long long a) {
  HeapElem ce = q.ce;
  const unsigned pos = static_cast<unsigned>(q.base_size) + 1u;
  const int depth = 31 - __clz(pos);
  int cur = q.base_root;
  for (int d = depth - 1; d >= 0; --d) {
    const HeapNode old = load_heap_node(p.hnodes, cur);
    const HeapElem oe = elem_of(old);
    const int bit = (pos >> d) & 1u;
    const int next = static_cast<int>(a) + (depth - d);
    const bool carry_down = heap_less(ce.vtx, ce.key, oe.vtx, oe.key);
    store_heap_node(p.hnodes + a + (depth - 1 - d), carry_down ? ce : oe,
                    bit ? old.left : next, bit ? next : old.right);
    if (carry_down) ce = oe;
    cur = bit ? old.right : old.left;
  }
  store_heap_node(p.hnodes + a + depth, ce, -1, -1);
  heap_store<kPublish>(p, v, static_cast<int>(a), static_cast<int>(pos));
}

template <bool kPublish = false>
__device__ void heap_insert(const SfxtParams& p, int v, unsigned long long* chunk = nullptr) {
  const InsertPlan q = plan_insert(p, v);
  if (q.empty) {
    heap_store<kPublish>(p, v, q.base_root, q.base_size);
    return;
  }
  const unsigned long long a = heap_alloc(p, insert_nodes(q.base_size), chunk);
  if (a == ~0ull) {
    atomicCAS(&p.ctr->err, kDevOk, kDevCapacity);
    heap_store<kPublish>(p, v, -1, 0);
    return;
  }
  heap_insert_at<kPublish>(p, v, q, a);
}

// Level-synchronous inserts, one vertex per lane (v < 0: none): the warp
// takes all its lanes' nodes with one atomic on the pool cursor.  Every lane
// of the warp calls.  kPublish: other threads poll the new heaps' sizes.
template <bool kPublish = false>
__device__ void heap_insert_lanes(const SfxtParams& p, int v) {
  const int lane = threadIdx.x & 31;
  InsertPlan q;
  q.empty = true;
  q.base_root = -1;
  q.base_size = 0;
  if (v >= 0) q = plan_insert(p, v);
  const unsigned need = v >= 0 && !q.empty ? insert_nodes(q.base_size) : 0u;
  unsigned incl = need;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const unsigned tot = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long base = 0;
  if (lane == 31 && tot) base = atomicAdd(&p.ctr->hnode_used, static_cast<unsigned long long>(tot));
  base = __shfl_sync(0xffffffffu, base, 31);
  if (v < 0) return;
  if (q.empty) {
    heap_store<kPublish>(p, v, q.base_root, q.base_size);
    return;
  }
  if (base + tot > p.hnode_cap) {
    atomicCAS(&p.ctr->err, kDevOk, kDevCapacity);
    heap_store<kPublish>(p, v, -1, 0);
    return;
  }
  heap_insert_at<kPublish>(p, v, q, base + (incl - need));
}

// The chain-heap phase of a dataflow build (p.heap_phase): after every
// vertex is built, each lane inserts the heaps of the queue slots it owns,
// in queue order (a vertex's successor is queued before it).  A heap waits
// only for its successor's, so the waits follow successor chains (about 80
// hops on the 1M-pin graph) instead of the 200 levels, and no build waits on
// a heap.  The 32 lanes of a warp take 32 consecutive slots; a lane's
// successor may be one of them, so the warp inserts, round after round, the
// lanes whose successor's heap is complete, with one pool reservation per
// round.  Returns false if a wait ran out.
__device__ bool heap_phase(const SfxtParams& p) {
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x >> 5);
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int base = gw * 32; base < p.n; base += nw * 32) {
    const int g = base + lane;
    const int v = g < p.n ? __ldcg(p.queue + g) : -1;
    const int s = v >= 0 ? __ldcg(p.succ + v) : -1;
    bool pending = v >= 0;
    unsigned int it = 0;
    while (__any_sync(0xffffffffu, pending)) {
      bool ready = false;
      if (pending)
        ready = s < 0 || ld_acquire(p.ht_size + s) >= 0;  // and the heap's nodes after it
      if (!__any_sync(0xffffffffu, ready)) {
        ++it;
        const bool bail = __any_sync(0xffffffffu, it > p.spin_limit ||
                                     ((it & 31) == 0 &&
                                      *reinterpret_cast<volatile int*>(&p.ctr->err) != kDevOk));
        if (bail) {
          if (lane == 0) atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
          return false;
        }
        __nanosleep(32);
        continue;
      }
      heap_insert_lanes<true>(p, ready ? v : -1);
      pending = pending && !ready;
    }
  }
  return true;
}

// BVSS form of the Kahn step.  A vertex that joins level L sets its bit in
// the level-parity frontier bitmap fbits[L & 1] and, first in its interval of
// 8, appends the interval to act_list.  Pulling level L, one warp per active
// interval counts for every slice (row u, mask of u's heads in the interval)
// how many heads just finished, popc(mask & frontier byte) -- on the tensor
// cores where the density test passes -- and takes that many off deps[u],
// which starts at u's number of distinct heads.  The warp then clears the
// interval's byte and bit so the bitmaps are clean for level L + 2.
__device__ __forceinline__ void bvss_mark(const SfxtParams& p, int parity, int u) {
  const size_t fw = (static_cast<size_t>(p.n) + 31) / 32;
  const size_t iw = ((static_cast<size_t>(p.n) + 7) / 8 + 31) / 32;
  atomicOr(p.fbits + parity * fw + (u >> 5), 1u << (u & 31));
  const int iv = u >> 3;
  const unsigned bit = 1u << (iv & 31);
  if (!(atomicOr(p.iact + parity * iw + (iv >> 5), bit) & bit))
    p.act_list[atomicAdd(&p.ctr->act_n, 1)] = iv;
}

__device__ void bvss_pull_interval(const SfxtParams& p, int iv, int lvl,
                                   unsigned long long& n_tensor, unsigned long long& n_scalar) {
  const int lane = threadIdx.x & 31;
  const size_t fw = (static_cast<size_t>(p.n) + 31) / 32;
  const size_t iw = ((static_cast<size_t>(p.n) + 7) / 8 + 31) / 32;
  unsigned int* fr = p.fbits + (lvl & 1) * fw;
  const unsigned fb = frontier_byte(fr, iv);
  for (int vss = p.bv_ptr[iv]; vss < p.bv_ptr[iv + 1]; ++vss) {
    const unsigned mask = p.bv_masks[static_cast<size_t>(vss) * 32 + lane];
    const int4 rw = reinterpret_cast<const int4*>(p.bv_rows)[static_cast<size_t>(vss) * 32 + lane];
    const int slices = p.bv_cnt[vss];
    const bool tensor = bvss_use_tensor(p.mma_mode, fb, slices, p.mma_min_bits, p.mma_min_slices);
    unsigned c[4];
    bvss_counts(mask, fb, tensor, slices > 64, c);
    n_tensor += tensor;
    n_scalar += !tensor;
    const int row[4] = {rw.x, rw.y, rw.z, rw.w};
    bool ready[4];
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      const int cnt = static_cast<int>(c[ch]);
      ready[ch] = cnt > 0 && row[ch] >= 0 && atomicSub(&p.deps[row[ch]], cnt) == cnt;
    }
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      const int slot = warp_append(&p.ctr->tail, ready[ch]);
      if (ready[ch]) {
        p.order[slot] = row[ch];
        p.level_of[row[ch]] = lvl + 1;
        bvss_mark(p, (lvl + 1) & 1, row[ch]);
      }
    }
  }
  if (lane == 0) {
    atomicAnd(fr + (iv >> 2), ~(0xffu << ((iv & 3) * 8)));
    atomicAnd(p.iact + (lvl & 1) * iw + (iv >> 5), ~(1u << (iv & 31)));
  }
}

// kBvss: the Kahn step pulls over the BVSS form (full builds only); a
// separate instantiation keeps the CSR build's registers unchanged.
template <bool kBvss>
__global__ void __launch_bounds__(kSfxtThreads)
sfxt_persistent_kernel(SfxtParams p) {
  const int warp_in_block = threadIdx.x >> 5;
  const int gwarp = blockIdx.x * (blockDim.x >> 5) + warp_in_block;
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  const bool full = p.start_level == 0;

  int beg, end, lvl;
  if (blockIdx.x == 0 && threadIdx.x == 0)
    p.ctr->sort_beg = full ? 0 : p.lvlp[p.start_level];
  if (full) {
    // phase 0: reset per-vertex state, seed level 0 with the sinks
    for (int base = blockIdx.x * blockDim.x; base < p.n;
         base += gridDim.x * blockDim.x) {
      const int v = base + threadIdx.x;
      bool sink = false;
      if (v < p.n) {
        const int od = p.adjp[v + 1] - p.adjp[v];
        p.deps[v] = kBvss ? p.bv_deps[v] : od;
        p.dist[v] = INT_MAX;
        p.succ[v] = -1;
        p.dev_cnt[v] = 0;
        p.ht_root[v] = -1;
        p.ht_size[v] = 0;
        p.level_of[v] = od == 0 ? 0 : -1;
        sink = od == 0;
      }
      const int slot = warp_append(&p.ctr->tail, sink);
      if (sink) {
        p.order[slot] = v;
        if (kBvss) bvss_mark(p, 0, v);
      }
    }
    if (!grid_sync(&p.ctr->bar, &p.ctr->err, p.spin_limit, &p.ctr->tail,
                   &p.ctr->level_end, 2))
      return;
    beg = 0;
    end = *reinterpret_cast<volatile int*>(&p.ctr->level_end);
    lvl = 0;
  } else {
    lvl = p.start_level;
    beg = p.lvlp[lvl];
    end = p.lvlp[lvl + 1];
  }

  const int first = lvl;   // first level rebuilt by this launch
  int pbeg = beg;          // previous level's range, whose heaps are pending
  int pend = beg;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nth = gridDim.x * blockDim.x;
  const bool pull = kBvss && full;
  int abeg = 0;            // act_list range of the level being pulled
  int aend = pull ? *reinterpret_cast<volatile int*>(&p.ctr->act_end) : 0;
  unsigned long long n_tensor = 0, n_scalar = 0;
  while (beg < end) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      p.lvlp[lvl] = beg;
      p.lvlp[lvl + 1] = end;
      // heap nodes in use before the previous level's inserts (which start
      // in this pass)
      if (lvl > first && !p.append_pool)
        p.pool_mark[lvl - 1] = *reinterpret_cast<volatile unsigned long long*>(&p.ctr->hnode_used);
    }
    {
      // a warp takes c consecutive vertices of the level (4..32, so that all
      // warps share a wide level): short rows four at a time by 8-lane
      // groups, the others one at a time by the whole warp
      const int lane = threadIdx.x & 31;
      const int per = (end - beg + nwarps - 1) / nwarps;
      const int c = per <= 4 ? 4 : per >= 32 ? 32 : (per + 3) & ~3;
      for (int i0 = beg + c * gwarp; i0 < end; i0 += c * nwarps) {
        const int i = i0 + lane;
        int v = -1, len = 0;
        if (lane < c && i < end) {
          v = __ldcg(p.order + i);
          if (!(full || rebuilt(p, v, lvl))) v = -1;
          else len = p.adjp[v + 1] - p.adjp[v];
        }
        const unsigned m8 = __ballot_sync(0xffffffffu, v >= 0 && len <= 8);
        const unsigned m16 = __ballot_sync(0xffffffffu, v >= 0 && len > 8 && len <= 16);
        const unsigned lg = __ballot_sync(0xffffffffu, v >= 0 && len > 16);
        const int n8 = __popc(m8), n16 = __popc(m16);
        for (int t = 0; t < n8; t += 4) {
          const int k = t + (lane >> 3);
          const int from = k < n8 ? kth_set_bit(m8, k) : 0;
          const int vg = __shfl_sync(0xffffffffu, v, from);
          build_group<8>(p, k < n8 ? vg : -1, lvl, full && !kBvss);
        }
        for (int t = 0; t < n16; t += 2) {
          const int k = t + (lane >> 4);
          const int from = k < n16 ? kth_set_bit(m16, k) : 0;
          const int vg = __shfl_sync(0xffffffffu, v, from);
          build_group<16>(p, k < n16 ? vg : -1, lvl, full && !kBvss);
        }
        for (unsigned b = lg; b; b &= b - 1) {
          const int vb = __shfl_sync(0xffffffffu, v, __ffs(b) - 1);
          build_vertex(p, vb, lvl, full && !kBvss);
        }
      }
    }
    if (kBvss && pull)
      for (int i = abeg + gwarp; i < aend; i += nwarps)
        bvss_pull_interval(p, __ldcg(p.act_list + i), lvl, n_tensor, n_scalar);
    for (int i0 = pbeg + (tid & ~31); i0 < pend; i0 += nth) {
      const int i = i0 + (threadIdx.x & 31);
      int v = i < pend ? __ldcg(p.order + i) : -1;
      if (v >= 0 && !(full || rebuilt(p, v, lvl - 1))) v = -1;
      heap_insert_lanes(p, v);
    }
    // the tail keeps growing as soon as the next level starts appending, so
    // the level bound is the snapshot the last arriving block took
    if (!grid_sync(&p.ctr->bar, &p.ctr->err, p.spin_limit, &p.ctr->tail,
                   &p.ctr->level_end, 2))
      return;
    ++lvl;
    pbeg = beg;
    pend = end;
    beg = end;
    abeg = aend;
    if (pull) aend = *reinterpret_cast<volatile int*>(&p.ctr->act_end);
    if (full) {
      end = *reinterpret_cast<volatile int*>(&p.ctr->level_end);
    } else {
      end = lvl < p.known_levels ? p.lvlp[lvl + 1] : beg;
    }
  }
  // heaps of the last level
  if (blockIdx.x == 0 && threadIdx.x == 0 && lvl > first && !p.append_pool)
    p.pool_mark[lvl - 1] = *reinterpret_cast<volatile unsigned long long*>(&p.ctr->hnode_used);
  for (int i0 = pbeg + (tid & ~31); i0 < pend; i0 += nth) {
    const int i = i0 + (threadIdx.x & 31);
    int v = i < pend ? __ldcg(p.order + i) : -1;
    if (v >= 0 && !(full || rebuilt(p, v, lvl - 1))) v = -1;
    heap_insert_lanes(p, v);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    p.ctr->levels = lvl;
    p.lvlp[lvl] = beg;
    p.ctr->sort_end = beg;
  }
  if (kBvss && (threadIdx.x & 31) == 0 && (n_tensor | n_scalar)) {
    atomicAdd(&p.ctr->vss_tensor, n_tensor);
    atomicAdd(&p.ctr->vss_scalar, n_scalar);
  }
}

// ------------------------------------------------------------ dataflow build
// Full CSR build without a barrier per level.  Kahn's algorithm runs as a
// work queue: a vertex is appended to queue[] when its last head finishes,
// and warp w builds the vertices in slots w, w + W, w + 2W, ... as they fill
// (a warp waits only for its next slot).  Every warp takes its slots in
// pushed order, so the earliest unfinished slot never waits on a later one
// and the walk always progresses.  A head raises its tails' levels
// (atomicMax) before taking its count off them, so a vertex's level is final
// when it is queued.  The chain-heap insert follows the decrements, off the
// build's critical path; it waits for the successor's heap (ht_size >= 0),
// which lies on a lower level.  Afterwards the vertices are counting-sorted
// by level into order[] / lvlp[] for the level-synchronous incremental
// rebuilds.  Every wait is bounded by spin_limit polls (kDevTimeout).

__device__ __forceinline__ int wait_slot(const SfxtParams& p, int s, bool acquire) {
  int v = -1;
  if ((threadIdx.x & 31) == 0) {
    unsigned int it = 0;
    const volatile int* q = p.queue + s;
    while ((v = *q) < 0) {
      if (++it > p.spin_limit ||
          ((it & 31) == 0 && *reinterpret_cast<volatile int*>(&p.ctr->err) != kDevOk)) {
        atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
        break;
      }
      __nanosleep(32);
    }
    if (acquire) __threadfence();  // late push: the heads' dist / level writes
  }
  return __shfl_sync(0xffffffffu, v, 0);
}

__device__ __forceinline__ bool wait_heap(const SfxtParams& p, int s) {
  if (s < 0) return true;
  unsigned int it = 0;
  while (ld_acquire(p.ht_size + s) < 0) {
    if (++it > p.spin_limit ||
        ((it & 31) == 0 && *reinterpret_cast<volatile int*>(&p.ctr->err) != kDevOk)) {
      atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
      return false;
    }
    __nanosleep(32);
  }
  return true;
}

// Early-push build of v: v's tails were decremented when v was taken, so a
// head may still be building; each head's (dist, level) word dl[] is polled
// until it is published (not ~0).  Same results as build_vertex.  Returns
// v's level, or -1 if a wait ran out (warp-uniform).
__device__ __forceinline__ unsigned long long ld_dl(const SfxtParams& p, int h) {
  return *reinterpret_cast<const volatile unsigned long long*>(p.dl + h);
}

__device__ int build_vertex_polled(const SfxtParams& p, int v, int rb, int re, DevEdge ed0,
                                   unsigned long long dl0) {
  const int lane = threadIdx.x & 31;
  int best = INT_MAX;
  int s = -1;
  int cnt = 0;
  int lmax = -1;
  DevSidetrack top;  // the cheapest deviation (lane 0's copy is used)
  top.head = -1;
  constexpr unsigned long long kNone = ~0ull;
  if (re - rb <= kRegChunks * 32) {
    DevEdge ed[kRegChunks];
    int dh[kRegChunks];
    ed[0] = ed0;  // loaded before the push (dl0: its head's word, or ~0)
#pragma unroll
    for (int c = 1; c < kRegChunks; ++c) {
      const int e = rb + c * 32 + lane;
      ed[c].head = -1;
      ed[c].w = 0.f;
      if (e < re) ed[c] = p.edges[e];
    }
    unsigned pending = 0;
#pragma unroll
    for (int c = 0; c < kRegChunks; ++c) {
      dh[c] = INT_MAX;
      if (ed[c].head >= 0) {
        // a published word never changes: one read before the push stands
        const unsigned long long x = c == 0 && dl0 != kNone ? dl0 : ld_dl(p, ed[c].head);
        if (x == kNone) {
          pending |= 1u << c;
        } else {
          dh[c] = static_cast<int>(x & 0xffffffffu);
          lmax = max(lmax, static_cast<int>(x >> 32));
        }
      }
    }
    unsigned int it = 0;
    while (__any_sync(0xffffffffu, pending != 0)) {
      // the lanes may read err differently: decide for the whole warp
      ++it;
      const bool bail = __any_sync(0xffffffffu, it > p.spin_limit ||
                                   ((it & 31) == 0 &&
                                    *reinterpret_cast<volatile int*>(&p.ctr->err) != kDevOk));
      if (bail) {
        if (lane == 0) atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
        return -1;
      }
      __nanosleep(32);
#pragma unroll
      for (int c = 0; c < kRegChunks; ++c) {
        if (pending & (1u << c)) {
          const unsigned long long x = ld_dl(p, ed[c].head);
          if (x != kNone) {
            dh[c] = static_cast<int>(x & 0xffffffffu);
            lmax = max(lmax, static_cast<int>(x >> 32));
            pending &= ~(1u << c);
          }
        }
      }
    }
    const int lvl = warp_max_i(lmax) + 1;
    if (lvl == 0) {
      best = 0;  // a sink
    } else {
#pragma unroll
      for (int c = 0; c < kRegChunks; ++c)
        if (ed[c].head >= 0) best = min(best, cand_dist(dh[c], ed[c].w));
      best = warp_min_i(best);
      int nt = 0;  // this lane's tied heads
#pragma unroll
      for (int c = 0; c < kRegChunks; ++c)
        if (ed[c].head >= 0 && cand_dist(dh[c], ed[c].w) == best) {
          s = max(s, ed[c].head);
          ++nt;
        }
      if (p.orig_id && __reduce_add_sync(0xffffffffu, nt) > 1) {
        unsigned long long k = 0;
#pragma unroll
        for (int c = 0; c < kRegChunks; ++c)
          if (ed[c].head >= 0 && cand_dist(dh[c], ed[c].w) == best) {
            const unsigned long long x = succ_word(p, ed[c].head);
            k = x > k ? x : k;
          }
        s = static_cast<int>(group_max_u64<32>(k) & 0xffffffffu);
      } else {
        s = warp_max_i(s);
      }
    }
    if (re - rb <= 32) {
      const bool valid = ed[0].head >= 0 && ed[0].head != s && dh[0] != INT_MAX;
      DevSidetrack rec;
      rec.head = ed[0].head;
      rec.w = ed[0].w;
      rec.dist_head = dh[0];
      rec.key = deviation_key(dh[0], best, ed[0].w);
      cnt = write_short_row(p, rb, valid, rec, top);
    } else if (re - rb <= 64) {
      DevSidetrack r[2];
      bool v[2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        v[c] = ed[c].head >= 0 && ed[c].head != s && dh[c] != INT_MAX;
        r[c].head = ed[c].head;
        r[c].w = ed[c].w;
        r[c].dist_head = dh[c];
        r[c].key = deviation_key(dh[c], best, ed[c].w);
      }
      cnt = write_row64(p, rb, v[0], r[0], v[1], r[1], top);
    } else {
      BestDev bd = best_none();
#pragma unroll
      for (int c = 0; c < kRegChunks; ++c) {
        if (rb + c * 32 >= re) break;
        const bool valid = ed[c].head >= 0 && ed[c].head != s && dh[c] != INT_MAX;
        const unsigned bal = __ballot_sync(0xffffffffu, valid);
        if (valid) {
          DevSidetrack rec;
          rec.head = ed[c].head;
          rec.w = ed[c].w;
          rec.dist_head = dh[c];
          rec.key = deviation_key(dh[c], best, ed[c].w);
          p.dev[rb + cnt + __popc(bal & lanemask_lt())] = rec;
          best_take(bd, true, rec, c * 32 + lane);
        }
        cnt += __popc(bal);
      }
      top = best_reduce(bd);
    }
    lmax = lvl;
  } else {
    // Long rows (a super-source's, say), eight chunks of 32 edges per pass
    // with every load of a pass issued before any is used.  Pass 1 waits for
    // each head's published word and takes, per lane, the least candidate
    // distance and the largest head reaching it; pass 2 writes the row.
    constexpr int kC = 8;
    int lbest = INT_MAX, ls = -1, lnt = 0;
    bool ok = true;
    for (int base = rb; base < re && ok; base += kC * 32) {
      DevEdge ed[kC];
      unsigned long long x[kC];
#pragma unroll
      for (int c = 0; c < kC; ++c) {
        const int e = base + c * 32 + lane;
        ed[c].head = -1;
        ed[c].w = 0.f;
        if (e < re) ed[c] = p.edges[e];
      }
#pragma unroll
      for (int c = 0; c < kC; ++c) x[c] = ed[c].head >= 0 ? ld_dl(p, ed[c].head) : 0ull;
#pragma unroll
      for (int c = 0; c < kC; ++c) {
        if (ed[c].head < 0) continue;
        unsigned int it = 0;
        while (x[c] == kNone && ok) {
          if (++it > p.spin_limit ||
              ((it & 31) == 0 && *reinterpret_cast<volatile int*>(&p.ctr->err) != kDevOk)) {
            atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
            ok = false;
            break;
          }
          __nanosleep(32);
          x[c] = ld_dl(p, ed[c].head);
        }
        if (!ok) break;
        lmax = max(lmax, static_cast<int>(x[c] >> 32));
        const int cd = cand_dist(static_cast<int>(x[c] & 0xffffffffu), ed[c].w);
        if (cd < lbest) {
          lbest = cd;
          ls = ed[c].head;
          lnt = 1;
        } else if (cd == lbest) {
          ls = max(ls, ed[c].head);
          ++lnt;
        }
      }
    }
    if (!__all_sync(0xffffffffu, ok)) return -1;
    const int lvl = warp_max_i(lmax) + 1;
    best = warp_min_i(lbest);
    s = warp_max_i(lbest == best ? ls : -1);
    // the heads' distances come from their published words
    auto dist_of = [&](int h) { return static_cast<int>(ld_dl(p, h) & 0xffffffffu); };
    if (p.orig_id && __reduce_add_sync(0xffffffffu, lbest == best ? lnt : 0) > 1) {
      unsigned long long k = 0;
      for (int e = rb + lane; e < re; e += 32) {
        const DevEdge ed = p.edges[e];
        if (cand_dist(dist_of(ed.head), ed.w) == best) {
          const unsigned long long y = succ_word(p, ed.head);
          k = y > k ? y : k;
        }
      }
      s = static_cast<int>(group_max_u64<32>(k) & 0xffffffffu);
    }
    BestDev bd = best_none();
    for (int base = rb; base < re; base += kC * 32) {
      DevEdge ed[kC];
      int dh[kC];
#pragma unroll
      for (int c = 0; c < kC; ++c) {
        const int e = base + c * 32 + lane;
        ed[c].head = -1;
        ed[c].w = 0.f;
        if (e < re) ed[c] = p.edges[e];
      }
#pragma unroll
      for (int c = 0; c < kC; ++c) dh[c] = ed[c].head >= 0 ? dist_of(ed[c].head) : INT_MAX;
#pragma unroll
      for (int c = 0; c < kC; ++c) {
        const int e = base + c * 32 + lane;
        const bool valid = ed[c].head >= 0 && ed[c].head != s && dh[c] != INT_MAX;
        DevSidetrack rec;
        rec.head = ed[c].head;
        rec.w = ed[c].w;
        rec.dist_head = dh[c];
        rec.key = deviation_key(dh[c], best, ed[c].w);
        const unsigned bal = __ballot_sync(0xffffffffu, valid);
        if (valid) p.dev[rb + cnt + __popc(bal & lanemask_lt())] = rec;
        best_take(bd, valid, rec, e - rb);
        cnt += __popc(bal);
      }
    }
    top = best_reduce(bd);
    lmax = lvl;
  }
  if (lane == 0) {
    p.dist[v] = best;
    p.succ[v] = s;
    p.dev_cnt[v] = cnt;
    if (re - rb > 64 && cnt > 1 && cnt <= kSmemRow) list_long_row(p, v);
    if (cnt > 0) p.best[v] = top;
    p.level_of[v] = lmax;
    // the word carries everything a tail's build reads of v, so it needs
    // no fence before it
    *reinterpret_cast<volatile unsigned long long*>(p.dl + v) =
        (static_cast<unsigned long long>(static_cast<unsigned>(lmax)) << 32) |
        static_cast<unsigned>(best);
  }
  return lmax;
}

// A lane-granular wait for queue slot s (the heap workers).
__device__ __forceinline__ int wait_slot_lane(const SfxtParams& p, int s) {
  unsigned int it = 0;
  const volatile int* q = p.queue + s;
  int v;
  while ((v = *q) < 0) {
    if (++it > p.spin_limit ||
        ((it & 31) == 0 && *reinterpret_cast<volatile int*>(&p.ctr->err) != kDevOk)) {
      atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
      return -1;
    }
    __nanosleep(32);
  }
  __threadfence();
  return v;
}

// Wait until a vertex's build is published (its flag in order[] is set).
__device__ __forceinline__ bool wait_built(const SfxtParams& p, int v) {
  unsigned int it = 0;
  const volatile int* f = p.order + v;
  while (*f == 0) {
    if (++it > p.spin_limit ||
        ((it & 31) == 0 && *reinterpret_cast<volatile int*>(&p.ctr->err) != kDevOk)) {
      atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
      return false;
    }
    __nanosleep(32);
  }
  __threadfence();
  return true;
}

// The dataflow work queue can be split in kSfxtQueues queues (vertex v goes
// to queue v % kSfxtQueues, whose segment of queue[] holds exactly those
// vertices), so appends spread over several counters.  One queue is kept:
// eight measured slower on the 1M-pin workload (kernel 2.60 ms against
// 2.41 ms), the single cursor not being the bottleneck.
constexpr int kSfxtQueues = 1;

__device__ __forceinline__ int queue_seg(const SfxtParams& p) {
  return (p.n + kSfxtQueues - 1) / kSfxtQueues;
}
__device__ __forceinline__ int queue_count(const SfxtParams& p, int q) {
  return p.n > q ? (p.n - 1 - q) / kSfxtQueues + 1 : 0;
}

// Append the lanes' u (where on) to their queues: one atomic per distinct
// queue among the warp's lanes.  All lanes call.
__device__ __forceinline__ void queue_push(const SfxtParams& p, bool on, int u) {
  const int lane = threadIdx.x & 31;
  const unsigned key = on ? static_cast<unsigned>(u) % kSfxtQueues : 0xffffffffu;
  const unsigned m = __match_any_sync(0xffffffffu, key);
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (on && lane == leader) base = atomicAdd(&p.ctr->qtail[key][0], __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (on) {
    const int slot = static_cast<int>(key) * queue_seg(p) + base + __popc(m & lanemask_lt());
    *reinterpret_cast<volatile int*>(p.queue + slot) = u;
  }
}

// Kahn step of the dataflow build: take one pending fan-out off each tail;
// tails reaching zero are queued.  kRelease: v's build precedes the push and
// is published by it (late push); an early push publishes nothing.
// Up to eight chunks of 32 tails per pass: their loads, then their
// decrements, then one queue reservation for all the tails that became
// ready, so a hub (the super-sink's 2,000 fan-in edges, say) costs a few
// round trips per 256 tails instead of several per 32.
// `before_counts` runs once, between the first pass's tail loads and its
// decrements, so loads it issues travel with the decrements.
struct NoHook {
  __device__ __forceinline__ void operator()() const {}
};

template <bool kRelease, class Hook = NoHook>
__device__ __forceinline__ void dataflow_push(const SfxtParams& p, int v, int ib, int ie,
                                              Hook before_counts = Hook()) {
  static_assert(kSfxtQueues == 1, "one reservation per pass assumes one queue");
  constexpr int kC = 8;
  const int lane = threadIdx.x & 31;
  for (int base = ib; base < ie; base += kC * 32) {
    const int nc = min(kC, (ie - base + 31) / 32);  // warp-uniform
    int u[kC];
#pragma unroll
    for (int c = 0; c < kC; ++c) {
      const int e = base + c * 32 + lane;
      u[c] = c < nc && e < ie ? p.iadj[e] : -1;
    }
    if (base == ib) before_counts();
    if (kRelease) __threadfence();  // release: v's dist and level before the counts
    unsigned ready = 0;  // bit c: this lane's tail of chunk c reached zero
#pragma unroll
    for (int c = 0; c < kC; ++c)
      if (u[c] >= 0 && atomicSub(&p.deps[u[c]], 1) == 1) ready |= 1u << c;
    if (kRelease) __threadfence();
    // slots: chunk by chunk, lane order within a chunk
    int total = 0, mine[kC];
#pragma unroll
    for (int c = 0; c < kC; ++c) {
      const unsigned bal = __ballot_sync(0xffffffffu, (ready >> c) & 1u);
      mine[c] = total + __popc(bal & lanemask_lt());
      total += __popc(bal);
    }
    if (total == 0) continue;
    int slot0 = 0;
    if (lane == 0) slot0 = atomicAdd(&p.ctr->qtail[0][0], total);
    slot0 = __shfl_sync(0xffffffffu, slot0, 0);
#pragma unroll
    for (int c = 0; c < kC; ++c)
      if ((ready >> c) & 1u) *reinterpret_cast<volatile int*>(p.queue + slot0 + mine[c]) = u[c];
  }
}

// One taken queue slot of the dataflow build: v's Kahn push and build (in
// either order), then its chain-heap insert unless the heap phase (kHp) or
// the heap workers do it.  False when a wait ran out (warp-uniform).
template <bool kHp>
__device__ __forceinline__ bool dataflow_slot(const SfxtParams& p, int v, int heap_warps,
                                              unsigned long long* chunk, int& max_lvl) {
  const int lane = threadIdx.x & 31;
  if (p.early_push) {
    // the tails learn of v before it is built; they wait on its word.
    // Graphs big enough for the heap phase keep a backlog of queued vertices
    // through most of the wave, so the warps' round trips count: the build's
    // row offsets are loaded with the push's, in one round trip, and the
    // row's first 32 edge words with the push's tails.  Smaller graphs leave
    // warps waiting on pushes: the push goes first, carrying no loads of the
    // build.  (The push is never deferred past the build: that puts every
    // build on the level-to-level path.)
    const int ib = p.iadjp[v], ie = p.iadjp[v + 1];
    int rb = 0, re = 0;
    DevEdge ed0;
    ed0.head = -1;
    ed0.w = 0.f;
    unsigned long long dl0 = ~0ull;
    if (kHp) {
      rb = p.adjp[v];
      re = p.adjp[v + 1];
      if (rb + lane < re) ed0 = p.edges[rb + lane];
      // the first heads' words are read with the push's decrements (with a
      // backlog the heads are almost always built by then)
      dataflow_push<false>(p, v, ib, ie, [&] {
        if (ed0.head >= 0) dl0 = ld_dl(p, ed0.head);
      });
    } else {
      dataflow_push<false>(p, v, ib, ie);
      rb = p.adjp[v];
      re = p.adjp[v + 1];
      if (rb + lane < re) ed0 = p.edges[rb + lane];
    }
    const int lvl = build_vertex_polled(p, v, rb, re, ed0, dl0);
    if (lvl < 0) return false;
    max_lvl = max(max_lvl, lvl);
    if (!kHp && lane == 0 && wait_heap(p, __ldcg(p.succ + v)))
      heap_insert<true>(p, v, chunk);
    __syncwarp();
    return true;
  }
  const int lvl = build_vertex<true>(p, v, 0, false);
  max_lvl = max(max_lvl, lvl);
  __syncwarp();
  if (heap_warps > 0 && lane == 0) {  // publish the build for the heap workers
    __threadfence();
    *reinterpret_cast<volatile int*>(p.order + v) = 1;
  }
  dataflow_push<true>(p, v, p.iadjp[v], p.iadjp[v + 1]);
  if (heap_warps == 0 && !kHp && lane == 0 && wait_heap(p, __ldcg(p.succ + v)))
    heap_insert<true>(p, v, chunk);
  __syncwarp();
  return true;
}

// A build warp's loop over the work queue (warp wib of its CTA).
// Claimed slots (claim_sets S > 0): a free warp claims the next slot of its
// claim set (slots q, q + S, ...), so a slot that fills while some warp is
// still building waits for nobody: any idle warp of the set takes it.  The S
// counters spread the claims (one atomic per vertex).  Static slots (S = 0):
// build warp bw serves queue bw % kSfxtQueues, taking every nwq-th slot.
template <bool kHp>
__device__ __forceinline__ void dataflow_build_warp(const SfxtParams& p, int wib, int build_warps,
                                                    int heap_warps, unsigned long long* chunk,
                                                    int& max_lvl) {
  const int lane = threadIdx.x & 31;
  const int nbw = gridDim.x * build_warps;
  const int bw = blockIdx.x * build_warps + wib;
  const int S = p.claim_sets;
  const int q = S > 0 ? bw % S : bw % kSfxtQueues;
  const int cnt = S > 0 ? (p.n > q ? (p.n - 1 - q) / S + 1 : 0) : queue_count(p, q);
  const int nwq = (nbw - q + kSfxtQueues - 1) / kSfxtQueues;
  const int seg0 = q * queue_seg(p);
  for (int k = bw / kSfxtQueues;; k += nwq) {
    int slot;
    if (S > 0) {
      int t = 0;
      if (lane == 0) t = atomicAdd(&p.ctr->claim[q][0], 1);
      t = __shfl_sync(0xffffffffu, t, 0);
      if (t >= cnt) break;
      slot = t * S + q;
    } else {
      if (k >= cnt) break;
      slot = seg0 + k;
    }
    const int v = wait_slot(p, slot, !p.early_push);
    if (v < 0 || !dataflow_slot<kHp>(p, v, heap_warps, chunk, max_lvl)) break;
  }
}

__global__ void __launch_bounds__(kSfxtThreads)
sfxt_dataflow_kernel(SfxtParams p) {
  __shared__ int s_hist[kSfxtThreads];
  const int lane = threadIdx.x & 31;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nth = gridDim.x * blockDim.x;
  // phase 0: reset, clear the queue and the level histogram
  for (int v = tid; v < p.n; v += nth) {
    p.deps[v] = p.adjp[v + 1] - p.adjp[v];
    p.dist[v] = INT_MAX;
    p.succ[v] = -1;
    p.dev_cnt[v] = 0;
    p.ht_root[v] = -1;
    p.ht_size[v] = -1;  // heap not built yet
    p.level_of[v] = 0;
    p.order[v] = 0;  // build-published flags until the final level sort
    p.dl[v] = ~0ull;  // (dist, level) not published yet
  }
  for (int i = tid; i < kSfxtQueues * queue_seg(p); i += nth) p.queue[i] = -1;
  for (int i = tid; i < p.n + 2; i += nth) p.lvlp[i] = 0;
  if (!grid_sync(&p.ctr->bar, &p.ctr->err, p.spin_limit)) return;
  // the sinks start the queue
  for (int base = blockIdx.x * blockDim.x; base < p.n; base += nth) {
    const int v = base + threadIdx.x;
    const bool sink = v < p.n && p.adjp[v + 1] == p.adjp[v];
    queue_push(p, sink, v);
  }
  // the last kHeapWarps warps of each CTA insert chain heaps, one vertex per
  // lane, in queue order; the others build.  A build never waits on a heap.
  int max_lvl = -1;
  const int wib = threadIdx.x >> 5;
  // each warp's private share of the heap pool (used by its lane 0)
  __shared__ unsigned long long s_chunk[kSfxtThreads / 32][2];
  unsigned long long* chunk = s_chunk[wib];
  if (lane == 0) chunk[0] = chunk[1] = 0;
  __syncwarp();
  const int heap_warps = p.heap_warps;  // 0: the build warp inserts the heap itself
  const int build_warps = kSfxtThreads / 32 - heap_warps;
  // The heap phase pays once the build warps have over ~128 vertices each
  // (measured: it loses 0.25-0.45 ms from 200,000 to 400,000 vertices,
  // where its chain of successor heaps is not hidden, and wins 0.2-0.35 ms
  // at 1,000,000)
  const bool hp = p.heap_phase == 2 ||
                  (p.heap_phase == 1 && p.n >= 128 * static_cast<int>(gridDim.x) * build_warps);
  if (wib < build_warps) {
    // one copy of the loop per regime, each compiled for its own order
    if (hp)
      dataflow_build_warp<true>(p, wib, build_warps, heap_warps, chunk, max_lvl);
    else
      dataflow_build_warp<false>(p, wib, build_warps, heap_warps, chunk, max_lvl);
  } else {
    const int nhl = gridDim.x * heap_warps * 32;
    const int seg = queue_seg(p);
    for (int g = (blockIdx.x * heap_warps + (wib - build_warps)) * 32 + lane;
         g < kSfxtQueues * seg; g += nhl) {
      const int q = g % kSfxtQueues, k = g / kSfxtQueues;
      if (k >= queue_count(p, q)) continue;
      const int v = wait_slot_lane(p, q * seg + k);
      if (v < 0 || !wait_built(p, v) || !wait_heap(p, __ldcg(p.succ + v))) break;
      heap_insert<true>(p, v);
    }
  }
  if (lane == 0) atomicMax(&p.ctr->levels, max_lvl + 1);
  if (!grid_sync(&p.ctr->bar, &p.ctr->err, p.spin_limit)) return;
  // Every vertex is built.  What is left: the chain heaps (the heap phase)
  // and the counting sort by level into order[] / lvlp[].  The sort's level
  // histogram comes first; block 0 scans it while the others start on the
  // heaps, and every block scatters its own vertices once its heaps are in,
  // so the sort costs no grid barrier of its own.
  const int L = *reinterpret_cast<volatile int*>(&p.ctr->levels);
  const bool small_l = L <= kSfxtThreads;
  __shared__ int s_base[kSfxtThreads];
  if (small_l) {
    for (int i = threadIdx.x; i < L; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    for (int v = tid; v < p.n; v += nth) atomicAdd(&s_hist[p.level_of[v]], 1);
    __syncthreads();
    for (int i = threadIdx.x; i < L; i += blockDim.x)
      if (s_hist[i]) atomicAdd(p.lvlp + i + 1, s_hist[i]);
  } else {
    for (int v = tid; v < p.n; v += nth) atomicAdd(p.lvlp + p.level_of[v] + 1, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(&p.ctr->sort_blocks, 1);
  }
  bool ok = true;
  if (blockIdx.x == 0) {
    // inclusive scan of lvlp[1..L] once every block's histogram is in
    __shared__ int carry, s_ok;
    if (threadIdx.x == 0) {
      carry = 0;
      unsigned int it = 0;
      bool w = true;
      while (*reinterpret_cast<volatile int*>(&p.ctr->sort_blocks) < static_cast<int>(gridDim.x)) {
        if (++it > p.spin_limit) {
          atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
          w = false;
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
      s_ok = w;
    }
    __syncthreads();
    ok = s_ok != 0;
    for (int base = 1; ok && base <= L; base += blockDim.x) {
      const int i = base + threadIdx.x;
      s_base[threadIdx.x] = i <= L ? __ldcg(p.lvlp + i) : 0;
      __syncthreads();
      for (int o = 1; o < blockDim.x; o <<= 1) {
        const int y = threadIdx.x >= o ? s_base[threadIdx.x - o] : 0;
        __syncthreads();
        s_base[threadIdx.x] += y;
        __syncthreads();
      }
      if (i <= L) p.lvlp[i] = s_base[threadIdx.x] + carry;
      __syncthreads();
      if (threadIdx.x == blockDim.x - 1) carry += s_base[threadIdx.x];
      __syncthreads();
    }
    if (threadIdx.x == 0 && ok) {
      p.ctr->sort_beg = 0;
      p.ctr->sort_end = p.n;
      __threadfence();
      *reinterpret_cast<volatile int*>(&p.ctr->sort_ready) = 1;
    }
  }
  if (hp) ok = heap_phase(p) && ok;
  // scatter this block's vertices by level: one reservation per (block,
  // level) on the level's cursor (deps[], all zero once every vertex was
  // queued), then a shared-memory cursor per level
  __shared__ int s_ready;
  if (threadIdx.x == 0) {
    unsigned int it = 0;
    bool w = true;
    while (*reinterpret_cast<volatile int*>(&p.ctr->sort_ready) == 0) {
      if (++it > p.spin_limit ||
          ((it & 31) == 0 && *reinterpret_cast<volatile int*>(&p.ctr->err) != kDevOk)) {
        atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
        w = false;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    s_ready = w;
  }
  __syncthreads();
  if (!__syncthreads_and(ok && s_ready != 0)) {
    if (threadIdx.x == 0) atomicCAS(&p.ctr->err, kDevOk, kDevTimeout);
    return;
  }
  if (small_l) {
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
      s_base[i] = s_hist[i] ? __ldcg(p.lvlp + i) + atomicAdd(p.deps + i, s_hist[i]) : 0;
      s_hist[i] = 0;
    }
    __syncthreads();
    for (int v = tid; v < p.n; v += nth) {
      const int l = p.level_of[v];
      p.order[s_base[l] + atomicAdd(&s_hist[l], 1)] = v;
    }
  } else {
    for (int v = tid; v < p.n; v += nth) {
      const int l = p.level_of[v];
      p.order[__ldcg(p.lvlp + l) + atomicAdd(p.deps + l, 1)] = v;
    }
  }
}

// ------------------------------------------------------------ row sorting
// Orders each rebuilt vertex's deviation list by (key, edge position): one
// warp per vertex, a register bitonic network of one or four words a lane for
// rows up to 32 or 128, a shared-memory one up to kSmemRow.  Longer rows go
// to sort_big_rows_kernel.
constexpr int kSortWarps = 8;

__global__ void __launch_bounds__(kSortWarps * 32)
sort_rows_kernel(const int32_t* rows, const int* n_rows, const int32_t* adjp,
                 const int32_t* dev_cnt, DevSidetrack* dev) {
  __shared__ unsigned long long skey[kSortWarps][kSmemRow];
  __shared__ DevSidetrack srec[kSortWarps][kSmemRow];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int end = *n_rows;  // the build listed the rows it left unsorted
  for (int i = blockIdx.x * kSortWarps + w; i < end; i += gridDim.x * kSortWarps) {
    const int v = rows[i];
    const int cnt = dev_cnt[v];
    DevSidetrack* row = dev + adjp[v];
    if (cnt <= 128) {
      sort_row_regs(row, cnt);
      continue;
    }
    int n2 = 256;
    for (int t = lane; t < n2; t += 32) {
      if (t < cnt) {
        const DevSidetrack r = row[t];
        srec[w][t] = r;
        skey[w][t] = sort_word(r.key, t);
      } else {
        skey[w][t] = ~0ull;
      }
    }
    __syncwarp();
    for (int k = 2; k <= n2; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int t = lane; t < n2; t += 32) {
          const int u = t ^ j;
          if (u > t) {
            const unsigned long long a = skey[w][t], b = skey[w][u];
            const bool asc = (t & k) == 0;
            if ((a > b) == asc) {
              skey[w][t] = b;
              skey[w][u] = a;
            }
          }
        }
        __syncwarp();
      }
    }
    for (int t = lane; t < cnt; t += 32)
      row[t] = srec[w][static_cast<int>(skey[w][t] & 0xffffffffu)];
    __syncwarp();
  }
}

// Rows longer than kSmemRow (a super-source, say): one block per row, a
// bitonic sort of the (key, position) words in dynamic shared memory, then a
// gather through the staging copy kept in big_tmp.
__global__ void sort_big_rows_kernel(const int32_t* rows, const int32_t* adjp,
                                     const int32_t* dev_cnt, DevSidetrack* dev,
                                     const int32_t* big_off, DevSidetrack* big_tmp,
                                     int cap, const int32_t* vgraph,
                                     const int32_t* graph_from, const int32_t* level_of) {
  extern __shared__ unsigned long long wbuf[];
  const int v = rows[blockIdx.x];
  const int cnt = dev_cnt[v];
  if (cnt <= kSmemRow) return;
  if (vgraph && level_of[v] < graph_from[vgraph[v]]) return;  // not rebuilt
  DevSidetrack* row = dev + adjp[v];
  DevSidetrack* tmp = big_tmp + big_off[blockIdx.x];
  int n2 = 1;
  while (n2 < cnt) n2 <<= 1;
  if (n2 > cap) n2 = cap;  // host guarantees cnt <= cap
  for (int t = threadIdx.x; t < n2; t += blockDim.x) {
    if (t < cnt) {
      const DevSidetrack r = row[t];
      tmp[t] = r;
      wbuf[t] = sort_word(r.key, t);
    } else {
      wbuf[t] = ~0ull;
    }
  }
  __syncthreads();
  for (int k = 2; k <= n2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < n2; t += blockDim.x) {
        const int u = t ^ j;
        if (u > t) {
          const unsigned long long a = wbuf[t], b = wbuf[u];
          const bool asc = (t & k) == 0;
          if ((a > b) == asc) {
            wbuf[t] = b;
            wbuf[u] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < cnt; t += blockDim.x)
    row[t] = tmp[static_cast<int>(wbuf[t] & 0xffffffffu)];
}

}  // namespace

int launch_sfxt(const SfxtParams& p, int device, void* stream, int* grid_out,
                int* launches, void* ev_before, void* ev_after) {
  int sms = 0, per_sm = 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  // full CSR builds run as a dataflow walk (unless asked to step the levels);
  // the BVSS pull and incremental rebuilds step level by level
  const bool bvss = p.bvss && p.start_level == 0;
  const bool dataflow = !bvss && p.start_level == 0 && !p.level_sync;
  void* kern = bvss       ? reinterpret_cast<void*>(sfxt_persistent_kernel<true>)
               : dataflow ? reinterpret_cast<void*>(sfxt_dataflow_kernel)
                          : reinterpret_cast<void*>(sfxt_persistent_kernel<false>);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSfxtThreads, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int grid = sms * per_sm;
  if (p.grid_limit > 0 && p.grid_limit < grid) grid = p.grid_limit;
  if (grid_out) *grid_out = grid;
  SfxtParams pp = p;
  void* args[] = {&pp};
  if (ev_before) {
    e = cudaEventRecord(static_cast<cudaEvent_t>(ev_before), st);
    if (e != cudaSuccess) return e;
  }
  e = cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kSfxtThreads), args, 0, st);
  if (e != cudaSuccess) return e;
  if (ev_after) {
    e = cudaEventRecord(static_cast<cudaEvent_t>(ev_after), st);
    if (e != cudaSuccess) return e;
  }
  sort_rows_kernel<<<sms * 8, kSortWarps * 32, 0, st>>>(p.long_rows, &p.ctr->n_long, p.adjp,
                                                        p.dev_cnt, p.dev);
  int n = 2;
  if (p.n_big_rows > 0) {
    const size_t smem = static_cast<size_t>(p.big_row_cap) * sizeof(unsigned long long);
    if (smem > 48 * 1024) {
      e = cudaFuncSetAttribute(sort_big_rows_kernel,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem));
      if (e != cudaSuccess) return e;
    }
    sort_big_rows_kernel<<<p.n_big_rows, 1024, smem, st>>>(
        p.big_rows, p.adjp, p.dev_cnt, p.dev, p.big_off, p.big_tmp, p.big_row_cap, p.vgraph,
        p.graph_from, p.level_of);
    ++n;
  }
  if (launches) *launches += n;
  return cudaGetLastError();
}

}  // namespace cpg

namespace cpg {
namespace {
__global__ void scatter_delays_kernel(DevEdge* edges, const int32_t* eids,
                                      const float* w, int64_t count) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < count) edges[eids[i]].w = w[i];
}
}  // namespace

int launch_scatter_delays(DevEdge* edges, const int32_t* eids, const float* w,
                          int64_t count, void* stream) {
  if (count <= 0) return cudaSuccess;
  const int threads = 256;
  const int64_t blocks = (count + threads - 1) / threads;
  scatter_delays_kernel<<<static_cast<unsigned>(blocks), threads, 0,
                          static_cast<cudaStream_t>(stream)>>>(edges, eids, w, count);
  return cudaGetLastError();
}
}  // namespace cpg

namespace cpg {
namespace {
// Counters for a build: zero, except the heap-pool cursor of an incremental
// rebuild, which restarts where the first rebuilt level's heaps began.
__global__ void init_sfxt_counters_kernel(SfxtCounters* c,
                                          const unsigned long long* pool_mark,
                                          int start_level, int append_pool) {
  static_assert(sizeof(SfxtCounters) % 4 == 0, "counters are cleared as ints");
  __shared__ unsigned long long used;
  if (threadIdx.x == 0)
    used = start_level > 0 ? (append_pool ? c->hnode_used : pool_mark[start_level]) : 0ull;
  __syncthreads();
  int* w = reinterpret_cast<int*>(c);
  for (int i = threadIdx.x; i < static_cast<int>(sizeof(SfxtCounters) / 4); i += blockDim.x)
    w[i] = 0;
  __syncthreads();
  if (threadIdx.x == 0) c->hnode_used = used;
}
}  // namespace

int launch_init_sfxt_counters(SfxtCounters* c, const unsigned long long* pool_mark,
                              int start_level, int append_pool, void* stream) {
  init_sfxt_counters_kernel<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      c, pool_mark, start_level, append_pool);
  return cudaGetLastError();
}
}  // namespace cpg
