// Drop-in for the reference's event SpMV FFI (lab/flybrain/ev_spmv.cu).
//
//   out[b, col[k]] += val[k] * (sp[b, pre] * mo[b, pre])   for k in row pre
//
// over the CSR of W transposed (row = presynaptic neuron).  Same exported
// names, argument meaning and return convention as the reference, so its
// ctypes loader (evspmv.py:832-930) can bind this library unchanged.
//
// Launch shape.  The reference launches one 128-thread block per
// presynaptic neuron and per trial, almost all of which exit at once, and a
// spiking row is walked by its block alone.  Here each CTA tests 256
// consecutive (trial, neuron) candidates, one per thread, and:
//
//  * a warp collects the row bounds of all its spiking candidates at once
//    (one round trip for up to 32 rows), then walks the concatenation of
//    those rows in passes of 32 consecutive edges, four passes' loads in
//    flight per lane before their atomics: the work of a warp is its edge
//    count, not its row count, and rows shorter than a pass share one;
//  * rows longer than kLong edges are set aside in shared memory and walked
//    by all eight warps of the CTA, kLong edges per warp in turn, so one
//    Pareto-tail row does not hold a single warp for its whole length.
//
// The grid is fixed by (n, batch) alone, so the call captures into a CUDA
// graph like the reference's.  Float atomics of integral values are exact in
// any order under the reference's exactness conditions (evspmv.py:957-994);
// each term val * s is formed exactly as the reference forms it.

#include <cuda_runtime.h>
#include <stdint.h>

#include "fis.h"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kUnroll = 4;    // passes whose loads are issued before their atomics
constexpr int kLong = 1024;   // longer rows are shared by the CTA's warps
constexpr unsigned kFull = 0xFFFFFFFFu;

// Walk the concatenated edges of the rows held by the warp's lanes: lane l
// holds row bounds [a, a + d) (d = 0: no row), the factor s and the trial b.
// Pass p covers edges 32 p .. 32 p + 31 of the concatenation; lane l takes
// edge 32 p + l and finds its row by a binary search over the lanes'
// exclusive prefix sums of d (the largest lane whose rows start at or before
// the edge; lanes without a row start where the next one does, so the search
// never stops on them).
template <typename I>
__device__ __forceinline__ void warp_walk(I a, int d, float s, int b, const I* __restrict__ col,
                                          const float* __restrict__ val, float* __restrict__ out,
                                          int64_t n, int lane) {
  int inc = d;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int t = __shfl_up_sync(kFull, inc, off);
    if (lane >= off) inc += t;
  }
  const int total = __shfl_sync(kFull, inc, 31);
  const int ex = inc - d;
  for (int j0 = 0; j0 < total; j0 += 32 * kUnroll) {
    I k[kUnroll];
    float sc[kUnroll];
    int bb[kUnroll];
    bool ok[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int j = j0 + 32 * u + lane;
      int r = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int c = r + step;
        if (__shfl_sync(kFull, ex, c) <= j) r = c;
      }
      ok[u] = j < total;
      k[u] = __shfl_sync(kFull, a, r) + (I)(j - __shfl_sync(kFull, ex, r));
      sc[u] = __shfl_sync(kFull, s, r);
      bb[u] = __shfl_sync(kFull, b, r);
    }
    I cc[kUnroll];
    float vv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (ok[u]) {
        cc[u] = col[k[u]];
        vv[u] = val[k[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
      if (ok[u]) atomicAdd(out + (int64_t)bb[u] * n + (int64_t)cc[u], __fmul_rn(vv[u], sc[u]));
  }
}

template <typename I>
__global__ void __launch_bounds__(kThreads)
k_ev_spmv(const I* __restrict__ crow, const I* __restrict__ col,
          const float* __restrict__ val, const float* __restrict__ sp,
          const float* __restrict__ mo, float* __restrict__ out, int n,
          int batch) {
  __shared__ I la[kThreads];      // long rows set aside by the warps: start,
  __shared__ int ld[kThreads];    // length,
  __shared__ float ls[kThreads];  // factor and
  __shared__ int lb[kThreads];    // trial
  __shared__ int nlong;
  const int64_t total = (int64_t)n * batch;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  // a CTA-uniform loop: every thread runs every iteration (barriers inside)
  for (int64_t base = (int64_t)blockIdx.x * kThreads; base < total;
       base += (int64_t)gridDim.x * kThreads) {
    if (threadIdx.x == 0) nlong = 0;
    __syncthreads();
    const int64_t x = base + threadIdx.x;
    float s = 0.f;
    if (x < total) s = __fmul_rn(sp[x], mo[x]);
    I a = 0;
    int d = 0, b = 0;
    if (s != 0.f) {
      b = (int)(x / n);
      const int64_t pre = x - (int64_t)b * n;
      a = crow[pre];
      const I e = crow[pre + 1];
      d = (int)(e - a);
      if (d > kLong) {
        const int q = atomicAdd(&nlong, 1);
        la[q] = a;
        ld[q] = d;
        ls[q] = s;
        lb[q] = b;
        d = 0;
      }
    }
    if (__any_sync(kFull, d > 0)) warp_walk<I>(a, d, s, b, col, val, out, n, lane);
    __syncthreads();
    // the long rows, kLong edges per warp in turn
    const int nl = nlong;
    for (int q = 0; q < nl; ++q) {
      const int len = ld[q];
      const int pieces = (len + kLong - 1) / kLong;
      for (int c = warp; c < pieces; c += kWarps) {
        const int lo = c * kLong;
        const int span = min(kLong, len - lo);
        // lane 0 holds the piece as one row; the others hold none
        warp_walk<I>(la[q] + (I)lo, lane == 0 ? span : 0, ls[q], lb[q], col, val, out, n, lane);
      }
    }
    __syncthreads();  // the long-row slots are reused by the next iteration
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
