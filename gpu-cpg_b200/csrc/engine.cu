// Persistent query engine for sm_100a: whole critical-path queries on the
// device, for one query or a batch of them, in one cooperative launch.
//
// Per query it reproduces the reference's report_paths after the suffix tree
// (gpucpg/gpucpg.cu:18502-21366) for SHORT_LONG:
//   roots       one PfxtNode per reachable source, cost (float)dist/SCALE_UP
//               (18502-18520), optionally trimmed by G-PathGen's initial split
//               (19136-19179)
//   split       raised until at least K non-zero paths cost <= split, the
//               stopping rule of the SHORT_LONG driver (19134-20850)
//   output      the K cheapest non-zero paths, ascending (21323-21360)
// The split raises, the closures between them, the top-K select and the
// segmented sort run back to back between bounded grid barriers; the host
// launches once and reads the results.
//
// Work layout: pending path-graph items of all queries share one pile (the
// query id rides in the top bits of Item::j), accepted paths share one store
// (pq[] holds their query); per-query state lives in EngineQuery.  Selection
// is a three-pass radix select per query over kSelBins-bin histograms;
// output is a stable LSD radix sort over (query, cost) words.
//
// This file is compiled with --use_fast_math like the reference (see
// pfxt_device.cuh for the child-cost expression).
#include <climits>
#include <cstddef>

#include "pfxt_device.cuh"

namespace cpg {

namespace {

constexpr int kEngThreads = 1024;  // one block per SM: fewer grid-barrier arrivals
constexpr int kEngWarps = kEngThreads / 32;

// Stage clock: block 0's thread 0 adds the globaltimer time since the last
// stamp to ctr->t_ns[stage] (stage = where the time went).
#define STAMP(stage)                                                   \
  do {                                                                 \
    if (blockIdx.x == 0 && threadIdx.x == 0) {                         \
      const unsigned long long now_ = gtime();                          \
      p.ctr->t_ns[stage] += now_ - t_last;                             \
      t_last = now_;                                                   \
    }                                                                  \
  } while (0)

__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid barriers of the engine.  The arrival counter only grows, so the
// barrier a block arrives at is told by the count it finds: arrivals
// n * G .. n * G + G - 1 (G blocks) belong to the n-th barrier of the launch,
// which is passed once the counter reads (n + 1) * G.  The last block to
// arrive has nothing to reset and the others leave on the first poll that
// sees its arrival.  eng_sync_last lets that last block run f() first and
// then publish the same target in a second word the others wait on.  Waits
// are bounded (kDevTimeout).
//
// Errors carry the stage they happened in (stage n is the work between
// barriers n - 1 and n), and barrier n fails for every block exactly when a
// stage up to n recorded one.  A block that leaves barrier n late must not
// see an error that a faster block records in stage n + 1: it would return
// while the others wait for it at barrier n + 1.
__shared__ unsigned int s_stage;  // the stage this block is in

__device__ __forceinline__ void eng_fail(const EngineParams& p, int code) {
  atomicCAS(&p.ctr->err, kDevOk, code);
  atomicCAS(reinterpret_cast<unsigned int*>(&p.ctr->err_stage), 0u, s_stage + 1u);
}

__device__ __forceinline__ void bar_wait(const EngineParams& p, const unsigned int* word,
                                         unsigned int target) {
  const volatile unsigned int* w = word;
  unsigned int it = 0;
  while (static_cast<int>(*w - target) < 0) {
    if (++it > p.spin_limit) {
      eng_fail(p, kDevTimeout);
      return;
    }
    __nanosleep(32);
  }
}

// On leaving barrier n (s_stage == n + 1): false if stages 0..n failed.
__device__ __forceinline__ bool eng_passed(const EngineParams& p) {
  const unsigned int es = *reinterpret_cast<const volatile unsigned int*>(&p.ctr->err_stage);
  return es == 0u || es > s_stage;
}

__device__ __forceinline__ bool eng_sync(const EngineParams& p) {
  __syncthreads();
  if (gridDim.x == 1) {
    // one CTA: the block barrier is the grid barrier
    if (threadIdx.x == 0) ++s_stage;
    __syncthreads();
    return eng_passed(p);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int old = atomicAdd(&p.ctr->bar.count, 1u);
    bar_wait(p, &p.ctr->bar.count, (old / gridDim.x + 1u) * gridDim.x);
    __threadfence();
    s_stage = old / gridDim.x + 1u;
  }
  __syncthreads();
  return eng_passed(p);
}

template <typename F>
__device__ __forceinline__ bool eng_sync_last(const EngineParams& p, F&& f) {
  __shared__ unsigned int s_target;
  __shared__ int s_last;
  __syncthreads();
  if (gridDim.x == 1) {
    f();
    __syncthreads();
    if (threadIdx.x == 0) ++s_stage;
    __syncthreads();
    return eng_passed(p);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int old = atomicAdd(&p.ctr->bar.count, 1u);
    s_target = (old / gridDim.x + 1u) * gridDim.x;
    s_last = old + 1u == s_target;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();  // the other blocks' writes before their arrival
    f();
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicMax(&p.ctr->bar.gen, s_target);
  } else if (threadIdx.x == 0) {
    bar_wait(p, &p.ctr->bar.gen, s_target);
    __threadfence();
  }
  if (threadIdx.x == 0) s_stage = s_target / gridDim.x;
  __syncthreads();
  return eng_passed(p);
}

#define ENG_SYNC()              \
  do {                          \
    if (!eng_sync(p)) return;   \
  } while (0)

__device__ __forceinline__ unsigned q_of(const Item& it) {
  return static_cast<unsigned>(it.j) >> kJBits;
}
__device__ __forceinline__ int j_of(const Item& it) {
  return static_cast<int>(static_cast<unsigned>(it.j) & kJMask);
}
__device__ __forceinline__ int pack_j(unsigned q, int j) {
  return static_cast<int>((q << kJBits) | static_cast<unsigned>(j));
}

__device__ __forceinline__ Item load_item(const Item* a, unsigned long long i) {
  const int4 r = __ldcg(reinterpret_cast<const int4*>(a + i));
  Item it;
  it.cost = __int_as_float(r.x);
  it.parent = r.y;
  it.node = r.z;
  it.j = r.w;
  return it;
}

__device__ __forceinline__ float float_below(float t) {
  // largest float < t
  if (t == 0.0f) return -__int_as_float(1);
  const int b = __float_as_int(t);
  return __int_as_float(t > 0.0f ? b - 1 : b + 1);
}

__device__ __forceinline__ void agg_add_u32(unsigned int* base, bool on, unsigned key) {
  const unsigned m = __match_any_sync(0xffffffffu, on ? key : 0xffffffffu);
  const int lane = threadIdx.x & 31;
  if (on && (__ffs(m) - 1) == lane) atomicAdd(base + key, static_cast<unsigned>(__popc(m)));
}

// Warp-aggregated per-query add: lanes with `on` add v to the 64-bit field at
// byte offset `off` of their query's EngineQuery; one atomic per distinct
// query in the warp.  All lanes call.
__device__ __forceinline__ void qadd(EngineQuery* qs, size_t off, bool on, unsigned q,
                                     unsigned v) {
  unsigned act = __ballot_sync(0xffffffffu, on && v != 0);
  const int lane = threadIdx.x & 31;
  while (act) {
    const int leader = __ffs(act) - 1;
    const unsigned ql = __shfl_sync(0xffffffffu, q, leader);
    const bool mine = on && v != 0 && q == ql;
    const unsigned m = __ballot_sync(0xffffffffu, mine);
    const unsigned sum = __reduce_add_sync(0xffffffffu, mine ? v : 0u);
    if (lane == leader)
      atomicAdd(reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(qs + ql) + off),
                static_cast<unsigned long long>(sum));
    act &= ~m;
  }
}
#define QOFF(field) offsetof(EngineQuery, field)

// ------------------------------------------------------------------ seeding
// One warp per query: reachable sources become root items; with the
// reference rule, roots at or below the initial split beyond the first
// (int)(0.005f*R + 1) (in source-id order) are dropped.
__device__ void seed_query(const EngineParams& p, int qi) {
  const int lane = threadIdx.x & 31;
  EngineQuery& Q = p.q[qi];
  const int b = Q.src_beg, e = Q.src_end;
  // number of reachable sources
  int r = 0;
  for (int i = b + lane; i < e; i += 32) r += __ldg(p.g.dist + p.srcs[i]) != INT_MAX;
  r = __reduce_add_sync(0xffffffffu, r);
  float split = __int_as_float(0x7f800000);
  int n_short = INT_MAX;
  if (p.root_ref && r > 0) {
    const float perc = 0.005f;
    const int idx = static_cast<int>(perc * r);
    n_short = static_cast<int>(perc * r + 1);
    // split = the idx-th smallest reachable root cost (rank by value, then id)
    float found = 0.f;
    int hit = 0;
    for (int i = b + lane; i < e; i += 32) {
      const int di = __ldg(p.g.dist + p.srcs[i]);
      if (di == INT_MAX) continue;
      const float ci = __fdiv_rn(static_cast<float>(di), 10000.0f);
      int rank = 0;
      for (int jj = b; jj < e; ++jj) {
        const int dj = __ldg(p.g.dist + p.srcs[jj]);
        if (dj == INT_MAX) continue;
        const float cj = __fdiv_rn(static_cast<float>(dj), 10000.0f);
        rank += (cj < ci) || (cj == ci && jj < i);
      }
      if (rank == idx) {
        found = ci;
        hit = 1;
      }
    }
    const unsigned hb = __ballot_sync(0xffffffffu, hit);
    split = __shfl_sync(0xffffffffu, found, __ffs(hb) - 1);
  }
  int short_seen = 0, kept_n = 0, kept_nz = 0;
  float rabs = 0.f;
  for (int base = b; base < e; base += 32) {
    const int i = base + lane;
    float c = 0.f;
    bool reach = false;
    int src = -1;
    if (i < e) {
      src = p.srcs[i];
      const int d = __ldg(p.g.dist + src);
      reach = d != INT_MAX;
      c = __fdiv_rn(static_cast<float>(d), 10000.0f);
    }
    const bool low = reach && !(c > split);
    const unsigned lb = __ballot_sync(0xffffffffu, low);
    const int before = short_seen + __popc(lb & lanemask_lt());
    const bool keep = reach && (!low || before < n_short);
    short_seen += __popc(lb);
    kept_n += __popc(__ballot_sync(0xffffffffu, keep));
    kept_nz += __popc(__ballot_sync(0xffffffffu, keep && c != 0.0f));
    if (keep) rabs = fmaxf(rabs, fabsf(c));
    const unsigned long long slot = warp_append(&p.ctr->pend_out, keep);
    if (keep) {
      if (slot < p.pend_cap) {
        Item it;
        it.cost = c;
        it.parent = -1;
        it.node = -2 - src;
        it.j = pack_j(static_cast<unsigned>(qi), 0);
        p.pend[0][slot] = it;
      } else {
        eng_fail(p, kDevCapacity);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) rabs = fmaxf(rabs, __shfl_xor_sync(0xffffffffu, rabs, o));
  if (lane == 0) {
    Q.root_abs = rabs;
    Q.done = 0;
    Q.mode = 0;
    Q.phases = 0;
    Q.paths_nz = 0;
    Q.pend_n = static_cast<unsigned long long>(kept_n);
    Q.pend_nz = static_cast<unsigned long long>(kept_nz);
    Q.pend_next_n = Q.pend_next_nz = 0;
    Q.out_lt = Q.out_eq = 0;
  }
}

// ------------------------------------------------------------------ select
// One histogram pass of the per-query radix select.  Elements: accepted
// paths (when the query's mode selects over them) and pending items.
__device__ void select_hist(const EngineParams& p, unsigned long long n_paths,
                            const Item* pend, unsigned long long n_pend, int shift,
                            int bits) {
  __shared__ unsigned int sh[kSelBins];
  const unsigned long long tid =
      static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned long long nth = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  const int hi = shift + bits;
  const unsigned hmask = hi >= 32 ? 0u : ~((1u << hi) - 1u);
  // accepted paths take part only when some query selects over them
  const unsigned long long np =
      *reinterpret_cast<const volatile int*>(&p.ctr->sel_paths) ? n_paths : 0;
  const unsigned long long tot = np + n_pend;
  const unsigned long long pad = (tot + 31) & ~31ull;
  const bool single = p.nq == 1;
  // one query: its mode and prefix hold for every element
  const int mode0 = single ? __ldcg(&p.q[0].mode) : 0;
  const unsigned prefix0 = single ? __ldcg(&p.q[0].prefix) : 0u;
  if (single) {
    for (int i = threadIdx.x; i < kSelBins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
  }
  for (unsigned long long i = tid; i < pad; i += nth) {
    bool on = false;
    unsigned key = 0, q = 0;
    if (i < tot) {
      float c;
      int mode;
      if (i < np) {
        q = single ? 0u : static_cast<unsigned>(__ldcg(p.pq + i));
        c = __ldcg(p.ps.cost + i);
        mode = single ? mode0 : __ldcg(&p.q[q].mode);
        on = (mode == 2 || mode == 3) && c != 0.0f;
      } else {
        const Item it = load_item(pend, i - np);
        q = q_of(it);
        c = it.cost;
        mode = single ? mode0 : __ldcg(&p.q[q].mode);
        on = (mode == 2 && c != 0.0f) || mode == 1;
      }
      if (on) {
        key = float_key(c);
        on = (key & hmask) == ((single ? prefix0 : __ldcg(&p.q[q].prefix)) & hmask);
      }
    }
    const unsigned bin = (key >> shift) & ((1u << bits) - 1u);
    if (single) {
      // costs cluster, so many lanes share a bin: one add per distinct bin
      agg_add_u32(sh, on, bin);
    } else {
      agg_add_u32(p.hist, on, q * kSelBins + bin);
    }
  }
  if (single) {
    __syncthreads();
    for (int i = threadIdx.x; i < (1 << bits); i += blockDim.x)
      if (sh[i]) atomicAdd(&p.hist[i], sh[i]);
  }
}

// select_pick for a single query by a whole block: each thread sums its
// share of the bins, a block scan finds the share holding the krem-th key,
// and its thread walks its few bins.  Each thread then clears its own bins.
__device__ __noinline__ void select_pick_block(EngineQuery* q0, unsigned int* h, int shift,
                                               int bits, unsigned int* chosen_n) {
  __shared__ unsigned long long s_wsum[kEngWarps];
  EngineQuery& Q = *q0;
  if (Q.mode == 0) return;  // the same for every thread
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int bins = 1 << bits;
  const int per = (bins + static_cast<int>(blockDim.x) - 1) / static_cast<int>(blockDim.x);
  const int b0 = static_cast<int>(threadIdx.x) * per;
  unsigned int mine[2] = {0u, 0u};  // per <= 2 (2048 bins, 1024 threads)
  unsigned long long sum = 0;
#pragma unroll
  for (int t = 0; t < 2; ++t)
    if (t < per && b0 + t < bins) {
      mine[t] = __ldcg(h + b0 + t);
      sum += mine[t];
    }
  // inclusive scan over the block, in thread (= bin) order
  unsigned long long incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const int nwarps = static_cast<int>(blockDim.x >> 5);
    unsigned long long w = lane < nwarps ? s_wsum[lane] : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nwarps) s_wsum[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  incl += wid > 0 ? s_wsum[wid - 1] : 0ull;
  const unsigned long long total = s_wsum[(blockDim.x >> 5) - 1];
  const unsigned long long k = Q.krem;
  const unsigned long long excl = incl - sum;
  // k beyond the total (cannot happen when the counts hold): the last thread
  const bool owner = (excl < k && k <= incl) ||
                     (k > total && threadIdx.x == blockDim.x - 1);
  __syncthreads();  // every thread has read krem before the owner updates it
  if (owner) {
    unsigned long long acc = excl;
    int bin = b0;
    if (per == 2 && acc + mine[0] < k) {  // the key is in the second bin
      acc += mine[0];
      ++bin;
    }
    Q.prefix |= static_cast<unsigned>(bin) << shift;
    Q.krem = k - acc;
    *chosen_n = bin == b0 ? mine[0] : mine[1];
  }
#pragma unroll
  for (int t = 0; t < 2; ++t)
    if (t < per && b0 + t < bins) h[b0 + t] = 0u;
}

// One warp per selecting query (warps gw, gw + nw, ...): find the bin
// holding the krem-th key.
__device__ void select_pick(const EngineParams& p, int shift, int bits, int gw, int nw) {
  const int lane = threadIdx.x & 31;
  const int bins = 1 << bits;
  const int per = bins / 32;
  for (int qi = gw; qi < p.nq; qi += nw) {
    EngineQuery& Q = p.q[qi];
    if (Q.mode == 0) continue;
    unsigned int* h = p.hist + static_cast<size_t>(qi) * kSelBins;
    unsigned long long sum = 0;
    for (int t = 0; t < per; ++t) sum += h[lane * per + t];
    unsigned long long incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const unsigned long long k = Q.krem;
    const unsigned long long excl = incl - sum;
    const bool mine = excl < k && k <= incl;
    const unsigned mb = __ballot_sync(0xffffffffu, mine);
    // k beyond the total (cannot happen when the host-side counts hold):
    // clamp to the last non-empty chunk
    const int owner = mb ? __ffs(mb) - 1 : 31;
    if (lane == owner) {
      unsigned long long acc = excl;
      int bin = lane * per;
      for (int t = 0; t < per - 1; ++t, ++bin) {
        if (acc + h[bin] >= k) break;
        acc += h[bin];
      }
      Q.prefix |= static_cast<unsigned>(bin) << shift;
      Q.krem = k - acc;
    }
    __syncwarp();
    for (int t = lane; t < bins; t += 32) h[t] = 0;
  }
}

// D. The split and acceptance limit of every selecting query (threads t0,
// t0 + nt, ...), and the cursors the promotion starts from.
__device__ void set_limits(const EngineParams& p, unsigned t0, unsigned nt, bool reset) {
  for (unsigned qi = t0; qi < static_cast<unsigned>(p.nq); qi += nt) {
    EngineQuery& Q = p.q[qi];
    if (Q.mode == 0) continue;
    const float t = key_float(Q.prefix);
    Q.t = t;
    if (Q.mode == 2) {
      const float a = fmaxf(fmaxf(fabsf(t), Q.root_abs), 1.0f);
      Q.lim = t + a * 0x1p-16f;
      Q.tie = t;
    } else {
      // accept strictly below the split when anything pending is cheaper
      // than it (ksel - krem items are), so a tie group at the split waits;
      // a coarse split is a bin's upper edge and takes the whole bin
      Q.lim = (Q.ksel > Q.krem && !Q.coarse) ? float_below(t) : t;
      Q.tie = __int_as_float(0x7fc00000);  // NaN: expand every path
    }
  }
  if (reset) {
    p.ctr->frontier[0] = 0;
    p.ctr->frontier[1] = 0;
    p.ctr->frontier[2] = 0;
    p.ctr->pend_out = 0;
  }
}

// The per-query radix select, then (with_limits) the split and limits.
// With at most one query per warp of a block, the last block to finish a
// histogram pass picks the bins itself before releasing the barrier, so a
// pass costs one grid barrier instead of two (and the limits none).
__device__ bool run_select(const EngineParams& p, unsigned long long n_paths,
                           const Item* pend, unsigned long long n_pend, bool with_limits) {
  const bool fused = p.nq <= kEngWarps;
  for (int pass = 0; pass < p.sel_passes; ++pass) {
    const int shift = p.sel_shift[pass], bits = p.sel_bits[pass];
    const bool last = pass == p.sel_passes - 1;
    select_hist(p, n_paths, pend, n_pend, shift, bits);
    if (fused) {
      __shared__ unsigned int s_chosen_n;
      if (!eng_sync_last(p, [&]() {
            bool done = last;
            if (p.nq == 1) {
              select_pick_block(p.q, p.hist, shift, bits, &s_chosen_n);
              __syncthreads();
              // A growth phase needs only about j items promoted, not the
              // j-th exactly: when the bin holding it is small against j,
              // split at the bin's upper edge and skip the last pass.
              EngineQuery& Q = p.q[0];
              if (with_limits && pass == p.sel_passes - 2 && Q.mode == 1 &&
                  static_cast<unsigned long long>(s_chosen_n) <=
                      (Q.ksel / 8 > 256 ? Q.ksel / 8 : 256ull)) {
                __syncthreads();  // every thread has read the query's mode
                if (threadIdx.x == 0) {
                  Q.prefix |= (1u << shift) - 1u;
                  Q.coarse = 1;
                  p.ctr->sel_stop = 1;
                }
                done = true;
              }
            } else {
              select_pick(p, shift, bits, static_cast<int>(threadIdx.x >> 5),
                          static_cast<int>(blockDim.x >> 5));
            }
            if (done && with_limits) {
              __syncthreads();
              set_limits(p, threadIdx.x, blockDim.x, threadIdx.x == 0);
            }
          }))
        return false;
      if (*reinterpret_cast<volatile int*>(&p.ctr->sel_stop)) break;
    } else {
      if (!eng_sync(p)) return false;
      select_pick(p, shift, bits, static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5),
                  static_cast<int>((gridDim.x * blockDim.x) >> 5));
      if (!eng_sync(p)) return false;
      if (last && with_limits) {
        set_limits(p, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x,
                   blockIdx.x == 0 && threadIdx.x == 0);
        if (!eng_sync(p)) return false;
      }
    }
  }
  return true;
}

// Block-wide appends to two piles (all threads of the block call): this
// thread's slot in pile A (if a) and in pile B (if b), with one reservation
// per block and pile instead of one per warp, since every block appends to
// the same two counters.
__device__ __forceinline__ void block_append2(unsigned long long* ca, bool a,
                                              unsigned long long* cb, bool b,
                                              unsigned long long& sa, unsigned long long& sb) {
  __shared__ unsigned int s_w[kEngWarps];        // per warp: count A << 16 | count B
  __shared__ unsigned long long s_base[2];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned ma = __ballot_sync(0xffffffffu, a), mb = __ballot_sync(0xffffffffu, b);
  if (lane == 0) s_w[wid] = (static_cast<unsigned>(__popc(ma)) << 16) | __popc(mb);
  __syncthreads();
  if (wid == 0) {
    const unsigned x = lane < kEngWarps ? s_w[lane] : 0u;
    unsigned incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < kEngWarps) s_w[lane] = incl - x;
    if (lane == 31) {
      const unsigned ta = incl >> 16, tb = incl & 0xffffu;
      s_base[0] = ta ? atomicAdd(ca, static_cast<unsigned long long>(ta)) : 0ull;
      s_base[1] = tb ? atomicAdd(cb, static_cast<unsigned long long>(tb)) : 0ull;
    }
  }
  __syncthreads();
  const unsigned pre = s_w[wid];
  sa = s_base[0] + (pre >> 16) + __popc(ma & lanemask_lt());
  sb = s_base[1] + (pre & 0xffffu) + __popc(mb & lanemask_lt());
  __syncthreads();  // s_w and s_base are reused by the next call
}

// ------------------------------------------------------------------ closure
// One reservation per warp for n items per lane (all lanes call): returns
// this lane's first slot.
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long* ctr, unsigned n) {
  const int lane = threadIdx.x & 31;
  unsigned incl = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const unsigned tot = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long base = 0;
  if (lane == 31 && tot) base = atomicAdd(ctr, static_cast<unsigned long long>(tot));
  base = __shfl_sync(0xffffffffu, base, 31);
  return base + (incl - n);
}

// Rounds over the frontier until it is empty.  Returns false on error.
__device__ bool run_closure(const EngineParams& p, Item* pend_out) {
  const unsigned long long tid =
      static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned long long nth = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  const bool single = p.nq == 1;
  const float lim0 = single ? __ldcg(&p.q[0].lim) : 0.f;
  const float tie0 = single ? __ldcg(&p.q[0].tie) : 0.f;
  unsigned acc_nz = 0, acc_pn = 0, acc_pnz = 0;
  int r = 0;
  for (;;) {
    volatile unsigned long long* fc = p.ctr->frontier;
    const unsigned long long n_cur = fc[r % 3];
    if (n_cur == 0) break;
    if (n_cur > p.front_cap) {
      eng_fail(p, kDevCapacity);
      return false;
    }
    const Item* in = p.front[r & 1];
    Item* out = p.front[(r + 1) & 1];
    unsigned long long* out_cnt = &p.ctr->frontier[(r + 1) % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctr->frontier[(r + 2) % 3] = 0;
    const unsigned long long n_pad = (n_cur + 31) & ~31ull;
    for (unsigned long long i = tid; i < n_pad; i += nth) {
      const bool valid = i < n_cur;
      Item it;
      it.cost = 0.f;
      it.parent = -1;
      it.node = -1;
      it.j = 0;
      if (valid) it = load_item(in, i);
      const unsigned q = q_of(it);
      const int jj = j_of(it);
      const unsigned long long qp = warp_append(&p.ctr->paths, valid);
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
      float lim = 0.f, tie = 0.f;
      if (valid) {
        lim = single ? lim0 : __ldcg(&p.q[q].lim);
        tie = single ? tie0 : __ldcg(&p.q[q].tie);
        int from = -1, level = 0;
        if (it.node <= -2) {
          to = -(it.node + 2);
        } else {
          hn = load_node(p.g.hnodes, it.node);
          from = hn.vtx;
          to = dev_head(p.g, hn, jj);
          level = __ldcg(p.ps.level + it.parent) + 1;
        }
        if (qp < p.ps.cap) {
          p.ps.cost[qp] = it.cost;
          p.ps.parent[qp] = it.parent;
          p.ps.from[qp] = from;
          p.ps.to[qp] = to;
          p.ps.level[qp] = level;
          p.pq[qp] = static_cast<int>(q);
          stored = true;
        } else {
          eng_fail(p, kDevCapacity);
        }
      }
      if (single) acc_nz += stored && it.cost != 0.0f;
      else qadd(p.q, QOFF(paths_nz), stored && it.cost != 0.0f, q, 1u);
      // a path costing exactly the final split is reported, not expanded
      const bool expand = stored && !(it.cost == tie);
      const bool sib = expand && it.node >= 0;
      const float pcost = sib ? __ldcg(p.ps.cost + it.parent) : 0.f;
      // the (up to) five children: heap left / right (or row 2j+1 / 2j+2),
      // row entries 1 and 2 of a heap node's row, and the cross child
      const int cross = expand ? __ldg(p.g.ht_root + to) : -1;
      float cc[5];
      unsigned exm = 0;
      // (the item's own node carries its row start, and every node the
      // record of its element, so no child costs more than one more load)
      if (sib && (jj == 0 ? cand_top(p.g, hn.left, pcost, cc[0])
                          : cand_row(p.g, hn, 2 * jj + 1, pcost, cc[0]))) exm |= 1u;
      if (sib && (jj == 0 ? cand_top(p.g, hn.right, pcost, cc[1])
                          : cand_row(p.g, hn, 2 * jj + 2, pcost, cc[1]))) exm |= 2u;
      if (sib && jj == 0 && cand_row(p.g, hn, 1, pcost, cc[2])) exm |= 4u;
      if (sib && jj == 0 && cand_row(p.g, hn, 2, pcost, cc[3])) exm |= 8u;
      if (expand && cand_top(p.g, cross, it.cost, cc[4])) exm |= 16u;
      unsigned tm = 0, dm = 0, dnz = 0;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        if (!(exm & (1u << k))) continue;
        if (cc[k] <= lim) tm |= 1u << k;
        else {
          dm |= 1u << k;
          dnz += cc[k] != 0.0f;
        }
      }
      // one reservation per warp and counter for all five
      unsigned long long bt = warp_reserve(out_cnt, __popc(tm));
      unsigned long long bd = warp_reserve(&p.ctr->pend_out, __popc(dm));
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const unsigned bit = 1u << k;
        if (!((tm | dm) & bit)) continue;
        Item c;
        c.cost = cc[k];
        c.parent = k == 4 ? static_cast<int>(qp) : it.parent;
        const int cn = k == 4 ? cross : (k < 2 && jj == 0 ? (k == 0 ? hn.left : hn.right) : it.node);
        const int cj = k == 4 ? 0 : k == 2 ? 1 : k == 3 ? 2 : (jj == 0 ? 0 : 2 * jj + 1 + k);
        c.node = cn;
        c.j = pack_j(q, cj);
        if (tm & bit) {
          if (bt < p.front_cap) out[bt] = c;
          else eng_fail(p, kDevCapacity);
          ++bt;
        } else {
          if (bd < p.pend_cap) pend_out[bd] = c;
          else eng_fail(p, kDevCapacity);
          ++bd;
        }
      }
      const unsigned ndef = __popc(dm), ndef_nz = dnz;
      if (single) {
        acc_pn += ndef;
        acc_pnz += ndef_nz;
      } else {
        qadd(p.q, QOFF(pend_next_n), valid, q, ndef);
        qadd(p.q, QOFF(pend_next_nz), valid, q, ndef_nz);
      }
    }
    if (!eng_sync(p)) return false;
    ++r;
  }
  if (single) {
    // one query: counts kept per thread through the whole closure (nothing
    // reads them before the phase ends), added once
    qadd(p.q, QOFF(paths_nz), acc_nz != 0, 0u, acc_nz);
    qadd(p.q, QOFF(pend_next_n), acc_pn != 0, 0u, acc_pn);
    qadd(p.q, QOFF(pend_next_nz), acc_pnz != 0, 0u, acc_pnz);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) p.ctr->rounds += r;
  return true;
}

// ------------------------------------------------------------------ sort
// Stable LSD pass over n (query, cost key, path) triples, 8-bit digit taken
// from the cost key (on_q == 0) or the query id.  Each block owns one
// contiguous tile.
__device__ bool lsd_pass(const EngineParams& p, unsigned long long n, int src,
                         int shift, bool on_q) {
  __shared__ unsigned int running[256];
  __shared__ unsigned int wcount[kEngWarps][256];
  __shared__ unsigned int dbase[256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned G = gridDim.x;
  const unsigned long long tile = (n + G - 1) / G;
  const unsigned long long t0 = blockIdx.x * tile;
  const unsigned long long t1 = t0 + tile < n ? t0 + tile : n;
  const unsigned int* kin = p.keys[src];
  const unsigned int* qin = p.qids[src];
  const unsigned int* vin = p.vals[src];
  auto digit_of = [&](unsigned long long i) -> unsigned {
    return ((on_q ? __ldcg(qin + i) : __ldcg(kin + i)) >> shift) & 255u;
  };
  // 1. tile histogram
  for (int d = threadIdx.x; d < 256; d += blockDim.x) running[d] = 0;
  __syncthreads();
  for (unsigned long long i = t0 + threadIdx.x; i < t1; i += blockDim.x)
    atomicAdd(&running[digit_of(i)], 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) p.sort_hist[d * G + blockIdx.x] = running[d];
  if (!eng_sync(p)) return false;
  // 2. one warp per digit: exclusive scan across tiles
  {
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int d = gw; d < 256; d += nw) {
      unsigned int carry = 0;
      for (unsigned b0 = 0; b0 < G; b0 += 32) {
        const unsigned b = b0 + lane;
        const unsigned x = b < G ? p.sort_hist[d * G + b] : 0u;
        unsigned incl = x;
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        if (b < G) p.sort_hist[d * G + b] = carry + incl - x;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) p.digit_tot[d] = carry;
    }
  }
  if (!eng_sync(p)) return false;
  // 3. digit bases, then a stable scatter of the tile
  if (threadIdx.x == 0) {
    unsigned acc = 0;
    for (int d = 0; d < 256; ++d) {
      dbase[d] = acc;
      acc += __ldcg(p.digit_tot + d);
    }
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x)
    running[d] = dbase[d] + __ldcg(p.sort_hist + d * G + blockIdx.x);
  for (int x = threadIdx.x; x < kEngWarps * 256; x += blockDim.x) wcount[x >> 8][x & 255] = 0;
  __syncthreads();
  unsigned int* kout = p.keys[src ^ 1];
  unsigned int* qout = p.qids[src ^ 1];
  unsigned int* vout = p.vals[src ^ 1];
  for (unsigned long long c0 = t0; c0 < t1; c0 += blockDim.x) {
    const unsigned long long i = c0 + threadIdx.x;
    const bool valid = i < t1;
    unsigned d = 256u, kk = 0, qq = 0, vv = 0;
    if (valid) {
      kk = __ldcg(kin + i);
      qq = __ldcg(qin + i);
      vv = __ldcg(vin + i);
      d = ((on_q ? qq : kk) >> shift) & 255u;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned lrank = __popc(peers & lanemask_lt());
    if (valid && lrank == 0) wcount[wid][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      unsigned pos = running[d] + lrank;
      for (int w = 0; w < wid; ++w) pos += wcount[w][d];
      kout[pos] = kk;
      qout[pos] = qq;
      vout[pos] = vv;
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) {
      unsigned s = 0;
      for (int w = 0; w < kEngWarps; ++w) {
        s += wcount[w][d];
        wcount[w][d] = 0;
      }
      running[d] += s;
    }
    __syncthreads();
  }
  return eng_sync(p);
}

// B. The next phase of one query: its mode and the rank its select aims at.
// Returns true if the query takes part in the phase.
__device__ bool decide_query(const EngineParams& p, EngineQuery& Q) {
  Q.mode = 0;
  if (Q.done) return false;
  Q.prefix = 0;
  Q.coarse = 0;
  // Every path costing <= the last phase's limit is accepted, so once
  // K non-zero paths are, the K-th of them is the answer's K-th cost and
  // the final phase only sweeps items within the rounding margin.
  if (Q.paths_nz >= static_cast<unsigned long long>(Q.k)) {
    Q.mode = 2;                       // final: the k-th of paths+pending
    Q.krem = static_cast<unsigned long long>(Q.k);
    Q.ksel = Q.krem;
    atomicOr(&p.ctr->sel_paths, 1);
  } else if (Q.pend_n > 0) {
    Q.mode = 1;                       // grow by count
    // promote ~4x the accepted count, but never more than half the
    // pile: every path below the split is accepted with its whole
    // closure, and the upper half of the pile reaches costs whose
    // closure is exponentially large (measured: a 3/4 cap accepted 77x
    // the paths needed)
    unsigned long long j = 4 * (Q.paths_nz + 1);
    // Near K, aim at K: every promoted item is accepted with its closure
    // below the split, and the last growth phase showed how many paths
    // one promoted item brings.  Promote the missing paths over that
    // ratio (with 20% to spare), so the phase that reaches K overshoots
    // little; falling short costs one more phase, which is only worth
    // risking when the overshoot would be large (an extra phase costs
    // about as much as closing ~1e5 more paths).
    // With fewer than 2^17 paths missing the aim keeps twice the spare
    // (falling short then costs one more phase, which is cheap against an
    // overshoot: promoting 4x the accepted count there once closed 8x K).
    if (p.grow_cap_k) {
      const unsigned long long miss = static_cast<unsigned long long>(Q.k) - Q.paths_nz;
      const bool far = miss >= (1ull << 17);
      unsigned long long aim = far ? miss : ~0ull;
      if (Q.last_j > 0 && Q.paths_nz > Q.acc_prev) {
        const double ratio = static_cast<double>(Q.paths_nz - Q.acc_prev) /
                             static_cast<double>(Q.last_j);
        if (ratio > 1.0) aim = static_cast<unsigned long long>((far ? 1.2 : 2.0) * miss / ratio) + 64;
      }
      if (j > aim) j = aim;
    }
    if (j < 64) j = 64;
    const unsigned long long half = (Q.pend_n + 1) / 2;
    if (j > half) j = half;
    Q.acc_prev = Q.paths_nz;
    Q.last_j = j;
    Q.krem = j;
    Q.ksel = j;
  } else {
    Q.done = 1;                       // every path enumerated
    return false;
  }
  ++Q.phases;
  return true;
}

// The bookkeeping between two phases, done by the last block to reach the
// grid barrier after the closure (or after seeding, finish == false): the
// finished phase's counts become the pending pile's, and every query's next
// phase is decided.  ctr->active then holds the number of running queries.
__device__ void next_phase(const EngineParams& p, int phase, bool finish) {
  if (threadIdx.x == 0) {
    if (finish) p.ctr->phases = phase + 1;
    p.ctr->active = 0;
    p.ctr->sel_paths = 0;
    p.ctr->sel_stop = 0;
  }
  __syncthreads();
  for (int qi = threadIdx.x; qi < p.nq; qi += blockDim.x) {
    EngineQuery& Q = p.q[qi];
    if (finish) {
      // G. final-mode queries are answered; counts restart
      if (Q.mode == 2) Q.done = 1;
      Q.pend_n = Q.pend_next_n;
      Q.pend_nz = Q.pend_next_nz;
      Q.pend_next_n = Q.pend_next_nz = 0;
    }
    if (decide_query(p, Q)) atomicAdd(&p.ctr->active, 1);
  }
}

// ------------------------------------------------------------------ kernel
__global__ void __launch_bounds__(kEngThreads) engine_kernel(EngineParams p) {
  const unsigned long long tid =
      static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned long long nth = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  const int gw = static_cast<int>(tid >> 5);
  const int nw = static_cast<int>(nth >> 5);

  unsigned long long t_last = 0;
  if (threadIdx.x == 0) s_stage = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) t_last = gtime();
  int pin = 0, phase0 = 0;
  unsigned long long n_pend = 0, n_paths = 0;
  if (p.resume) {
    // the one-CTA launch before this one either finished the query or
    // stopped at the top of a phase; an error there ends this launch too
    if (*reinterpret_cast<volatile int*>(&p.ctr->err) != kDevOk ||
        !*reinterpret_cast<volatile int*>(&p.ctr->stopped))
      return;
    pin = __ldcg(&p.ctr->res_pin);
    phase0 = __ldcg(&p.ctr->res_phase);
    n_pend = __ldcg(&p.ctr->res_pend);
    n_paths = __ldcg(&p.ctr->res_paths);
  } else {
    // seed roots (pending pile 0)
    for (int qi = gw; qi < p.nq; qi += nw) seed_query(p, qi);
    if (!eng_sync_last(p, [&]() { next_phase(p, 0, false); }))
      return;
    STAMP(0);
    n_pend = *reinterpret_cast<volatile unsigned long long*>(&p.ctr->pend_out);
  }

  for (int phase = phase0;; ++phase) {
    const Item* pend = p.pend[pin];
    Item* pend_next = p.pend[pin ^ 1];
    // (per-query counts are kept current by seeding, promotion and closure)
    if (*reinterpret_cast<volatile int*>(&p.ctr->active) == 0) break;
    if (p.solo_stop && n_pend > p.solo_stop) {
      // the pile outgrew one CTA: leave the rest to the full launch
      if (threadIdx.x == 0) {
        p.ctr->res_pin = pin;
        p.ctr->res_phase = phase;
        p.ctr->res_pend = n_pend;
        p.ctr->res_paths = n_paths;
        p.ctr->stopped = 1;
        __threadfence();
      }
      return;
    }
    // C + D. per-query radix select, split and acceptance limit
    if (!run_select(p, n_paths, pend, n_pend, true)) return;
    STAMP(2);
    // E. promote pending items under their query's limit
    {
      const bool single = p.nq == 1;
      const int mode0 = single ? __ldcg(&p.q[0].mode) : 0;
      const int done0 = single ? __ldcg(&p.q[0].done) : 0;
      const float lim0 = single ? __ldcg(&p.q[0].lim) : 0.f;
      unsigned acc_n = 0, acc_nz = 0;
      // block-uniform trip count: the appends synchronise the block
      for (unsigned long long b0 = tid - threadIdx.x; b0 < n_pend; b0 += nth) {
        const unsigned long long i = b0 + threadIdx.x;
        bool take = false, keep = false;
        Item it;
        it.cost = 0.f;
        it.j = 0;
        if (i < n_pend) {
          it = load_item(pend, i);
          const EngineQuery& Q = p.q[q_of(it)];
          const int mode = single ? mode0 : __ldcg(&Q.mode);
          const int done = single ? done0 : __ldcg(&Q.done);
          take = mode != 0 && it.cost <= (single ? lim0 : __ldcg(&Q.lim));
          keep = !take && !done;
        }
        unsigned long long a = 0, b = 0;
        block_append2(&p.ctr->frontier[0], take, &p.ctr->pend_out, keep, a, b);
        if (take) {
          if (a < p.front_cap) p.front[0][a] = it;
          else eng_fail(p, kDevCapacity);
        }
        if (keep) {
          if (b < p.pend_cap) pend_next[b] = it;
          else eng_fail(p, kDevCapacity);
        }
        if (single) {
          acc_n += keep;
          acc_nz += keep && it.cost != 0.0f;
        } else {
          qadd(p.q, QOFF(pend_next_n), keep, q_of(it), 1u);
          qadd(p.q, QOFF(pend_next_nz), keep && it.cost != 0.0f, q_of(it), 1u);
        }
      }
      if (single) {
        qadd(p.q, QOFF(pend_next_n), acc_n != 0, 0u, acc_n);
        qadd(p.q, QOFF(pend_next_nz), acc_nz != 0, 0u, acc_nz);
      }
    }
    ENG_SYNC();
    STAMP(3);
    // F. closure
    if (!run_closure(p, pend_next)) return;
    STAMP(4);
    // G + B. counts restart, the next phase is decided
    if (!eng_sync_last(p, [&]() { next_phase(p, phase, true); }))
      return;
    STAMP(1);
    n_paths = *reinterpret_cast<volatile unsigned long long*>(&p.ctr->paths);
    n_pend = *reinterpret_cast<volatile unsigned long long*>(&p.ctr->pend_out);
    pin ^= 1;
  }

  // ---------------------------------------------------------------- output
  if (n_paths > p.ps.cap) {
    eng_fail(p, kDevCapacity);
    return;
  }
  for (unsigned long long i = tid; i < n_paths; i += nth) p.rank_of[i] = -1;
  // One query: once K non-zero paths were accepted, the final phase's split
  // T is the K-th cost of the paths and pending items then known, and every
  // item up to T was accepted with its closure.  Fewer than K accepted paths
  // cost less than T unless a closure produced a child a few ulps below its
  // parent's T; so one pass puts the paths below T in the output buffer and
  // those at T in a side buffer, the first K - (below) of those follow, and
  // no output select is needed.  (Below T counting K or more falls back to
  // the select.)  If the paths ran out before K, every one is reported.
  unsigned int out_lo = 0u, out_hi = 0xffffffffu;  // key range, for the sort
  bool fast_out = false;
  if (p.nq == 1) {
    const EngineQuery& Q = p.q[0];
    const unsigned long long k = static_cast<unsigned long long>(Q.k);
    const unsigned long long k_out = Q.paths_nz < k ? Q.paths_nz : k;
    const unsigned kT = Q.paths_nz >= k ? float_key(__ldcg(&Q.t)) : 0xffffffffu;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      p.ctr->key_min = 0xffffffffu;
      p.ctr->key_max = 0u;
    }
    ENG_SYNC();
    unsigned kmin = 0xffffffffu, kmax = 0u;
    // block-uniform trip count: the appends synchronise the block
    for (unsigned long long b0 = tid - threadIdx.x; b0 < n_paths; b0 += nth) {
      const unsigned long long i = b0 + threadIdx.x;
      bool lt = false, eq = false;
      unsigned key = 0;
      if (i < n_paths) {
        const float c = __ldcg(p.ps.cost + i);
        if (c != 0.0f) {
          key = float_key(c);
          lt = key < kT;
          eq = key == kT;
        }
      }
      unsigned long long a = 0, b = 0;
      block_append2(&p.ctr->out_below, lt, &p.ctr->out_at, eq, a, b);
      if (lt && a < k_out) {
        p.keys[0][a] = key;
        p.vals[0][a] = static_cast<unsigned>(i);
        p.qids[0][a] = 0u;
      }
      if (eq && b < k_out) p.vals[1][b] = static_cast<unsigned>(i);
      if (lt || eq) {
        kmin = min(kmin, key);
        kmax = max(kmax, key);
      }
    }
    kmin = __reduce_min_sync(0xffffffffu, kmin);
    kmax = __reduce_max_sync(0xffffffffu, kmax);
    if ((threadIdx.x & 31) == 0 && kmin <= kmax) {
      atomicMin(&p.ctr->key_min, kmin);
      atomicMax(&p.ctr->key_max, kmax);
    }
    ENG_SYNC();
    const unsigned long long below = *reinterpret_cast<volatile unsigned long long*>(&p.ctr->out_below);
    fast_out = below <= k_out;
    if (fast_out) {
      const unsigned long long need = k_out - below;
      for (unsigned long long i = tid; i < need; i += nth) {
        p.keys[0][below + i] = kT;
        p.vals[0][below + i] = __ldcg(p.vals[1] + i);
        p.qids[0][below + i] = 0u;
      }
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        EngineQuery& W = p.q[0];
        W.k_out = k_out;
        W.out_off = 0;
        W.mode = k_out > 0 ? 3 : 0;
        p.ctr->out_total = k_out;
      }
      out_lo = *reinterpret_cast<volatile unsigned int*>(&p.ctr->key_min);
      out_hi = *reinterpret_cast<volatile unsigned int*>(&p.ctr->key_max);
      ENG_SYNC();
    }
  }
  if (!fast_out) {
    // H. per-query counts are current (kept up to date by the closures)
    ENG_SYNC();
    for (unsigned long long qi = tid; qi < static_cast<unsigned long long>(p.nq); qi += nth) {
      EngineQuery& Q = p.q[qi];
      const unsigned long long k = static_cast<unsigned long long>(Q.k);
      Q.k_out = Q.paths_nz < k ? Q.paths_nz : k;
      Q.mode = Q.k_out > 0 ? 3 : 0;
      Q.prefix = 0;
      Q.krem = Q.k_out;
      Q.out_lt = Q.out_eq = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctr->sel_paths = 1;
    ENG_SYNC();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      unsigned long long acc = 0;
      for (int qi = 0; qi < p.nq; ++qi) {
        p.q[qi].out_off = acc;
        acc += p.q[qi].k_out;
      }
      p.ctr->out_total = acc;
    }
    if (!run_select(p, n_paths, nullptr, 0, false)) return;
    STAMP(5);
    const unsigned long long n_out = *reinterpret_cast<volatile unsigned long long*>(&p.ctr->out_total);
    if (n_out > p.out_cap) {
      eng_fail(p, kDevCapacity);
      return;
    }
    // J. compaction into per-query segments: keys below the k-th, then the
    // first ones equal to it
    {
      const unsigned long long pad = (n_paths + 31) & ~31ull;
      for (unsigned long long i = tid; i < pad; i += nth) {
        bool lt = false, eq = false;
        unsigned q = 0, key = 0;
        if (i < n_paths) {
          q = static_cast<unsigned>(__ldcg(p.pq + i));
          const float c = __ldcg(p.ps.cost + i);
          const EngineQuery& Q = p.q[q];
          if (c != 0.0f && __ldcg(&Q.mode) == 3) {
            key = float_key(c);
            const unsigned kth = __ldcg(&Q.prefix);
            lt = key < kth;
            eq = key == kth;
          }
        }
        const int lane = threadIdx.x & 31;
        const unsigned ml = __match_any_sync(0xffffffffu, lt ? q : 0xffffffffu);
        unsigned long long bl = 0;
        if (lt && (__ffs(ml) - 1) == lane) bl = atomicAdd(&p.q[q].out_lt, static_cast<unsigned long long>(__popc(ml)));
        bl = __shfl_sync(0xffffffffu, bl, lt ? __ffs(ml) - 1 : lane);
        const unsigned me = __match_any_sync(0xffffffffu, eq ? q : 0xffffffffu);
        unsigned long long be = 0;
        if (eq && (__ffs(me) - 1) == lane) be = atomicAdd(&p.q[q].out_eq, static_cast<unsigned long long>(__popc(me)));
        be = __shfl_sync(0xffffffffu, be, eq ? __ffs(me) - 1 : lane);
        if (lt || eq) {
          const EngineQuery& Q = p.q[q];
          const unsigned long long need_eq = __ldcg(&Q.krem);
          const unsigned long long n_lt = __ldcg(&Q.k_out) - need_eq;
          const unsigned long long off = __ldcg(&Q.out_off);
          unsigned long long slot = ~0ull;
          if (lt) {
            const unsigned long long r = bl + __popc(ml & lanemask_lt());
            if (r < n_lt) slot = off + r;
          } else {
            const unsigned long long r = be + __popc(me & lanemask_lt());
            if (r < need_eq) slot = off + n_lt + r;
          }
          if (slot != ~0ull) {
            p.keys[0][slot] = key;
            p.qids[0][slot] = q;
            p.vals[0][slot] = static_cast<unsigned>(i);
          }
        }
      }
    }
    ENG_SYNC();
  }
  STAMP(5);
  // K. stable LSD sort over (query, cost); a digit that every key shares
  // (the keys span out_lo..out_hi) needs no pass
  const unsigned long long n_sort = *reinterpret_cast<volatile unsigned long long*>(&p.ctr->out_total);
  int src = 0;
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = pass * 8;
    if (out_lo <= out_hi && (out_lo >> shift) == (out_hi >> shift)) break;
    if (!lsd_pass(p, n_sort, src, shift, false)) return;
    src ^= 1;
  }
  for (int shift = 0; (p.nq - 1) >> shift; shift += 8) {
    if (!lsd_pass(p, n_sort, src, shift, true)) return;
    src ^= 1;
  }
  STAMP(6);
  // L. ranks within each query's list, then M. emission
  for (unsigned long long i = tid; i < n_sort; i += nth) {
    const unsigned q = __ldcg(p.qids[src] + i);
    p.rank_of[__ldcg(p.vals[src] + i)] =
        static_cast<int>(i - __ldcg(&p.q[q].out_off));
  }
  ENG_SYNC();
  for (unsigned long long i = tid; i < n_sort; i += nth) {
    const unsigned idx = __ldcg(p.vals[src] + i);
    const float c = __ldcg(p.ps.cost + idx);
    p.out_cost[i] = c;
    if (p.out_nodes) {
      cpg_path_node nd;
      nd.level = __ldcg(p.ps.level + idx);
      nd.from = __ldcg(p.ps.from + idx);
      nd.to = __ldcg(p.ps.to + idx);
      const int par = __ldcg(p.ps.parent + idx);
      nd.parent = par >= 0 ? __ldcg(p.rank_of + par) : -1;
      nd.num_children = 0;
      nd.slack = c;
      p.out_nodes[i] = nd;
    }
  }
  STAMP(7);
  // the sorted path indices stay in vals[src]; the host learns which buffer
  if (blockIdx.x == 0 && threadIdx.x == 0) p.ctr->sorted_buf = src;
}

}  // namespace

int engine_grid(int device, int limit, int* grid_out) {
  int sms = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, engine_kernel, kEngThreads, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int grid = sms * per_sm;
  if (limit > 0 && limit < grid) grid = limit;
  *grid_out = grid;
  return cudaSuccess;
}

namespace {
// A few queries' table, passed by value to the kernel that writes it.
struct QueryTable {
  EngineQuery q[kInlineQueries];
};
__global__ void set_queries_kernel(EngineQuery* dst, QueryTable t, int nq) {
  if (static_cast<int>(threadIdx.x) < nq) dst[threadIdx.x] = t.q[threadIdx.x];
}
}  // namespace

// Writes up to kInlineQueries queries' table from the launch parameters, so
// a query starts without a host-to-device copy (which would wait behind any
// large upload another stream has on the copy engine).
int launch_set_queries(EngineQuery* dst, const EngineQuery* src, int nq, void* stream) {
  if (nq < 1 || nq > kInlineQueries) return cudaErrorInvalidValue;
  QueryTable t{};
  for (int i = 0; i < nq; ++i) t.q[i] = src[i];
  set_queries_kernel<<<1, kInlineQueries, 0, static_cast<cudaStream_t>(stream)>>>(dst, t, nq);
  return cudaGetLastError();
}

int launch_engine(const EngineParams& p, int device, void* stream) {
  int grid = 0;
  cudaError_t e = static_cast<cudaError_t>(engine_grid(device, p.grid_limit, &grid));
  if (e != cudaSuccess) return e;
  EngineParams pp = p;
  void* args[] = {&pp};
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(engine_kernel), dim3(grid),
                                     dim3(kEngThreads), args, 0,
                                     static_cast<cudaStream_t>(stream));
}

}  // namespace cpg
