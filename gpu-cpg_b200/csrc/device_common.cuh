// Device helpers shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cpg_internal.hpp"

namespace cpg {

// Acquire load and release store at GPU scope: the reader of a flag sees
// every write the flag's writer made before it, without a full fence on
// either side.
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Grid-wide barrier for cooperative (co-resident) launches.  The wait is
// bounded: after `limit` polls the block records kDevTimeout in *err and
// leaves the barrier, so a lost block can never hang the GPU.  Returns false
// once any block has recorded an error before arriving: the last block to
// arrive copies *err into the barrier, and every block decides on that copy,
// so a block that leaves late does not see an error another block records
// after the barrier (it would return while the others wait for it at the
// next one).
//
// If snap_src is given, the last block to arrive copies snap_src[0..snap_n)
// to snap_dst before releasing the others: a counter that blocks keep
// appending to after the barrier (a queue tail) can then be read as one
// agreed value by every block.
__device__ __forceinline__ bool grid_sync(GridBarrier* b, int* err,
                                          unsigned int limit,
                                          const int* snap_src = nullptr,
                                          int* snap_dst = nullptr, int snap_n = 1) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = &b->gen;
    const unsigned int g = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(&b->count, 1u);
    bool timed_out = false;
    if (arrived == gridDim.x - 1) {
      __threadfence();
      if (snap_src)
        for (int i = 0; i < snap_n; ++i)
          reinterpret_cast<volatile int*>(snap_dst)[i] =
              reinterpret_cast<const volatile int*>(snap_src)[i];
      reinterpret_cast<volatile int*>(&b->err)[0] = reinterpret_cast<volatile int*>(err)[0];
      atomicExch(&b->count, 0u);
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      unsigned int it = 0;
      while (*vgen == g) {
        if (++it > limit) {
          atomicCAS(err, kDevOk, kDevTimeout);
          timed_out = true;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = !timed_out && reinterpret_cast<volatile int*>(&b->err)[0] == kDevOk;
  }
  __syncthreads();
  return s_ok != 0;
}

// Warp-aggregated append: one atomic per warp.  Every lane of the warp must
// call it; returns the slot of this lane (meaningful only where pred).
template <typename T>
__device__ __forceinline__ T warp_append(T* counter, bool pred) {
  const unsigned mask = __ballot_sync(0xffffffffu, pred);
  if (mask == 0) return 0;
  const int leader = __ffs(mask) - 1;
  const int lane = threadIdx.x & 31;
  T base = 0;
  if (lane == leader) base = atomicAdd(counter, static_cast<T>(__popc(mask)));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + static_cast<T>(__popc(mask & lanemask_lt()));
}

__device__ __forceinline__ int warp_min_i(int v) {
  return __reduce_min_sync(0xffffffffu, v);
}
__device__ __forceinline__ int warp_max_i(int v) {
  return __reduce_max_sync(0xffffffffu, v);
}

// Order-preserving map of a float to uint32 (larger float, larger key).
__device__ __host__ __forceinline__ unsigned int float_key(float f) {
  unsigned int u;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(f);
#else
  __builtin_memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __host__ __forceinline__ float key_float(unsigned int k) {
  unsigned int u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
#ifdef __CUDA_ARCH__
  f = __uint_as_float(u);
#else
  __builtin_memcpy(&f, &u, 4);
#endif
  return f;
}

}  // namespace cpg
