// Drop-in for the reference's event SpMV FFI (lab/flybrain/ev_spmv.cu).
//
//   out[b, col[k]] += val[k] * (sp[b, pre] * mo[b, pre])   for k in row pre
//
// over the CSR of W transposed (row = presynaptic neuron).  Same exported
// names, argument meaning and return convention as the reference, so its
// ctypes loader (evspmv.py:832-930) can bind this library unchanged.
//
// Launch shape (the reference launches one 128-thread block per presynaptic
// neuron and per trial, almost all of which exit at once): here every thread
// tests one (trial, neuron) pair, a warp ballots its 32 candidates, and the
// whole warp then walks each spiking row in turn, 32 consecutive edges per
// pass.  The grid is fixed by (n, batch) alone, so the call captures into a
// CUDA graph like the reference's.  Float atomics of integral values are
// exact in any order under the reference's exactness conditions
// (evspmv.py:957-994); the product val*s is formed exactly as the reference
// forms it.

#include <cuda_runtime.h>
#include <stdint.h>

#include "fis.h"

namespace {

constexpr int kThreads = 256;

template <typename I>
__global__ void __launch_bounds__(kThreads)
k_ev_spmv(const I* __restrict__ crow, const I* __restrict__ col,
          const float* __restrict__ val, const float* __restrict__ sp,
          const float* __restrict__ mo, float* __restrict__ out, int n,
          int batch) {
  const int64_t total = (int64_t)n * batch;
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (kThreads / 32);
  for (int64_t base = ((int64_t)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5)) * 32;
       base < total; base += warps * 32) {
    const int64_t x = base + lane;
    float s = 0.f;
    if (x < total) s = __fmul_rn(sp[x], mo[x]);
    unsigned live = __ballot_sync(0xFFFFFFFFu, s != 0.f);
    while (live) {
      const int src = __ffs(live) - 1;
      live &= live - 1;
      const int64_t xs = base + src;
      const float ss = __shfl_sync(0xFFFFFFFFu, s, src);
      const int64_t b = xs / n;
      const int64_t pre = xs - b * n;
      float* o = out + b * n;
      const I a = crow[pre], e = crow[pre + 1];
      for (I k = a + (I)lane; k < e; k += (I)32)
        atomicAdd(o + (int64_t)col[k], __fmul_rn(val[k], ss));
    }
  }
}

int grid_for(int64_t total) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    sms = 148;
  int64_t g = (total + kThreads - 1) / kThreads;
  const int64_t cap = (int64_t)sms * 8;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

extern "C" {

int ev_spmv_i32(const int* crow, const int* col, const float* val, const float* sp,
                const float* mo, float* out, int n, int batch, int threads,
                void* stream) {
  (void)threads;
  if (n < 1 || batch < 1) return (int)cudaErrorInvalidValue;
  k_ev_spmv<int><<<grid_for((int64_t)n * batch), kThreads, 0, (cudaStream_t)stream>>>(
      crow, col, val, sp, mo, out, n, batch);
  return (int)cudaGetLastError();
}

int ev_spmv_i64(const long long* crow, const long long* col, const float* val,
                const float* sp, const float* mo, float* out, int n, int batch,
                int threads, void* stream) {
  (void)threads;
  if (n < 1 || batch < 1) return (int)cudaErrorInvalidValue;
  k_ev_spmv<long long><<<grid_for((int64_t)n * batch), kThreads, 0, (cudaStream_t)stream>>>(
      crow, col, val, sp, mo, out, n, batch);
  return (int)cudaGetLastError();
}

int ev_spmv_abi(void) { return 3; }

}  // extern "C"
