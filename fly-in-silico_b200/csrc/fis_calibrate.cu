// Calibration kernel: the sustained rate of 32-bit atomic adds (red.add) into
// a buffer that lives in L2, the ceiling of the engine's scatter, whose
// every pushed synapse is one such add into the scratch ring.  The bench
// times it once and states the scatter's achieved rate against it, as the
// HBM roofline states achieved bytes against a measured copy bandwidth.

#include <cuda_runtime.h>
#include <stdint.h>

#include "fis.h"

namespace {

constexpr int kThreads = 256;

// Each thread adds 1 at `iters` pseudo-random word addresses (a 32-bit
// multiply-xorshift hash of thread and iteration), eight adds in flight per
// loop turn; every address lies in [0, words).
__global__ void __launch_bounds__(kThreads)
k_red_rate(uint32_t* __restrict__ buf, uint32_t words, int iters) {
  uint32_t h = (blockIdx.x * kThreads + threadIdx.x) * 0x9E3779B1u + 0x7F4A7C15u;
  for (int i = 0; i < iters; i += 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      h ^= h >> 15;
      h *= 0x2C1B3C6Du;
      h ^= h >> 12;
      asm volatile("red.global.add.u32 [%0], 1;\n" ::"l"(buf + (h % words)) : "memory");
    }
  }
}

}  // namespace

extern "C" int fis_red_rate(uint32_t* buf, int64_t words, int32_t iters, int32_t ctas,
                            void* stream) {
  if (!buf || words < 1 || words > 0x7FFFFFFFLL || iters < 8 || (iters % 8) != 0 || ctas < 1)
    return FIS_E_ARG;
  k_red_rate<<<ctas, kThreads, 0, (cudaStream_t)stream>>>(buf, (uint32_t)words, iters);
  return (int)cudaGetLastError();
}
