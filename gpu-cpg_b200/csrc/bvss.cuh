// Device side of the BVSS (bit-vector slice set, sigma = 8) form: the binary
// tensor-core tile that counts, for the 128 slices of one VSS, how many of
// each slice's columns lie in the frontier byte of the VSS's interval.
//
// Layout (host builder in bvss_host.cpp): slice i of a VSS sits in lane
// i % 32, chunk i / 32: bits 8*chunk..8*chunk+7 of masks[vss*32 + lane] and
// rows[vss*128 + lane*4 + chunk].
//
// Tile (the placement of gpucpg/tc_sfxt_bvss.cuh:366-386): one m8n8k128 b1
// MMA with AND-popc accumulation computes C[r][j] = popc(A[r][:] & B[:][j]).
// Lane l supplies A row l/4, k range 32*(l%4)..+31; put its chunks 0 and 1 in
// the low 16 bits.  B column j is supplied by lanes 4j..4j+3 (k range 32*t);
// placing the frontier byte at k = 32*s + 8*h of column 2s+h, i.e. in lane
// 9s + 4h (lane % 9 == 0: the byte, lane % 9 == 4: the byte << 8), makes
// C[r][2s+h] = popc(chunk h of lane 4r+s & byte), and lane l receives
// C[l/4][2(l%4)] and C[l/4][2(l%4)+1]: exactly its own chunk 0 and 1 counts.
// A second MMA on the high 16 bits gives chunks 2 and 3.
#pragma once

#include <stdint.h>

namespace cpg {

__device__ __forceinline__ void mma_b1_and_popc(unsigned* c, unsigned a, unsigned b) {
  asm volatile(
      "mma.sync.aligned.m8n8k128.row.col.s32.b1.b1.s32.and.popc "
      "{%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+r"(c[0]), "+r"(c[1])
      : "r"(a), "r"(b));
}

// Counts of this lane's four slices against frontier byte fb.  All 32 lanes
// call it with warp-uniform fb / tensor / upper.  upper == false skips the
// second MMA (a VSS with at most 64 slices has nothing in chunks 2, 3).
// Returns the number of MMAs issued.
__device__ __forceinline__ int bvss_counts(unsigned mask, unsigned fb, bool tensor, bool upper,
                                           unsigned out[4]) {
  if (tensor) {
    const unsigned res = (threadIdx.x & 31) % 9;
    const unsigned b = res == 0 ? fb : (res == 4 ? (fb << 8) : 0u);
    unsigned c[4] = {0u, 0u, 0u, 0u};
    mma_b1_and_popc(&c[0], mask & 0x0000ffffu, b);
    if (upper) mma_b1_and_popc(&c[2], mask >> 16, b);
    out[0] = c[0];
    out[1] = c[1];
    out[2] = c[2];
    out[3] = c[3];
    return upper ? 2 : 1;
  }
#pragma unroll
  for (int ch = 0; ch < 4; ++ch) out[ch] = __popc((mask >> (8 * ch)) & fb & 0xffu);
  return 0;
}

// The density test: a tile goes to the tensor cores when its frontier byte
// has at least min_bits bits and the VSS more than min_slices slices; mode 1
// forces the tensor cores, mode 2 the scalar path.
__device__ __forceinline__ bool bvss_use_tensor(int mode, unsigned fb, int slices,
                                                int min_bits, int min_slices) {
  if (mode == 1) return true;
  if (mode == 2) return false;
  return __popc(fb) >= min_bits && slices > min_slices;
}

__device__ __forceinline__ unsigned frontier_byte(const unsigned int* words, int interval) {
  return (__ldcg(words + (interval >> 2)) >> ((interval & 3) * 8)) & 0xffu;
}

}  // namespace cpg
