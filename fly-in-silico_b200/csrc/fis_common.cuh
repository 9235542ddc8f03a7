// Shared device helpers of the B200 LIF engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fis.h"

namespace fis {

constexpr int kWarp = 32;

// Philox4x32-10, the counter-based generator of Salmon, Moraes, Dror and
// Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of
// two 32x32->64 multiplies, the key bumped by the Weyl constants between
// rounds.
// All four output words of Philox4x32-10.  The drive uses one call per four
// steps of a neuron: counter (neuron, own_step / 4 low, own_step / 4 high,
// trial lane), word own_step % 4 is the draw of that step.
struct Philox4 {
  uint32_t x[4];
};

__host__ __device__ __forceinline__ Philox4 philox4(uint32_t c0, uint32_t c1, uint32_t c2,
                                                    uint32_t c3, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
#ifdef __CUDA_ARCH__
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2);
#else
    const uint32_t hi0 = (uint32_t)(((uint64_t)0xD2511F53u * c0) >> 32);
    const uint32_t hi1 = (uint32_t)(((uint64_t)0xCD9E8D57u * c2) >> 32);
#endif
    const uint32_t lo0 = 0xD2511F53u * c0;
    const uint32_t lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  Philox4 r;
  r.x[0] = c0;
  r.x[1] = c1;
  r.x[2] = c2;
  r.x[3] = c3;
  return r;
}

// Packed edge: postsynaptic index in the high 18 bits, signed count low 14.
__device__ __forceinline__ int edge_post(uint32_t w) { return (int)(w >> 14); }
__device__ __forceinline__ int edge_count(uint32_t w) {
  return ((int32_t)(w << 18)) >> 18;
}

// Spike-list entry: presynaptic index << 8 | chunk index.
constexpr uint32_t kDeadEntry = 0xFFFFFFFFu;
__device__ __forceinline__ uint32_t entry_pre(uint32_t e) { return e >> 8; }
__device__ __forceinline__ uint32_t entry_chunk(uint32_t e) { return e & 0xFFu; }

__host__ __device__ __forceinline__ int64_t mod_pos(int64_t a, int64_t m) {
  int64_t r = a % m;
  return r < 0 ? r + m : r;
}

}  // namespace fis
