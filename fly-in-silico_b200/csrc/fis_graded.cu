// Graded-spike mode of the whole-brain LIF step, sm_100a.
//
// The exact engine (fis_engine.cu) carries whole spikes as integer counts.  A
// caller that writes fractional values into the spike state before a step
// (visdyn.py:660-676: photoreceptor rates and graded lamina/medulla output)
// needs the reference's float product instead:
//
//   recurrent = w_scale * (W @ (spikes * m_out))        sim.py:910-913 (csrmv)
//   refrac    = (refrac + 1) * (1 - spikes)             sim.py:921
//
// followed by the rest of the step (sim.py:921-953) on a float delay ring
// [B][buf_len][N] with the reference's read-then-write slot `ptr`.  Two
// kernels per step:
//
//  * k_graded_nz marks, per trial, the neurons whose spikes * m_out is not
//    zero, one bit each;
//  * k_graded_pull: one warp per (trial, postsynaptic neuron) accumulates the
//    neuron's in-edges in ascending presynaptic order with one fused
//    multiply-add per edge -- the order and fusing of torch's CPU kernel for a
//    CSR matrix times a dense one, which the reference's csrmv path runs, so
//    the sums carry the reference's bits.  Terms with a zero factor change
//    nothing: fma(v, +-0, acc) = acc for every acc the chain can hold (it
//    starts at +0, and a rounded sum is -0 only when both addends are -0).
//    So each CTA holds its trial's bit mask in shared memory; a warp streams
//    32 consecutive presynaptic indices of the row at a time, tests them in
//    the mask, and gathers value and weight only for the few set ones (spikes
//    are rare and graded values sit on a few hundred neurons), folding them
//    lowest lane (lowest presynaptic index) first, every lane carrying the
//    same sum.
//  * k_graded_step: one thread per (trial, neuron), the reference's
//    operations in its order, one float32 rounding at a time; masks, the
//    refractory steps and the Poisson drive come from the engine's flag bits,
//    parameters and per-trial Philox stream, as in the exact engine.
//
// The pull reads every edge once per trial and step (8 B per edge), so a step
// costs about E * 8 B * B of L2/HBM traffic: this mode is for the interactive
// single-trial callers that need it, not for the batched path.

#include <cuda_runtime.h>
#include <stdint.h>

#include "fis.h"
#include "fis_common.cuh"

namespace fis {
namespace {

constexpr int kGradedThreads = 256;

// spikes * m_out (sim.py:912): m_out is 0 for a neuron whose output is cut or
// which is silenced in this trial
__device__ __forceinline__ float graded_x(const float* spikes, const uint8_t* flags, int64_t at) {
  const float m = (flags[at] & (FIS_FL_OUT_OFF | FIS_FL_SILENCED)) ? 0.f : 1.f;
  return __fmul_rn(spikes[at], m);
}

// nz[b][i / 32] bit i % 32: spikes * m_out of neuron i in trial b is not zero
__global__ void __launch_bounds__(kGradedThreads)
k_graded_nz(const float* __restrict__ spikes, const uint8_t* __restrict__ flags, const int n,
            const int words, uint32_t* __restrict__ nz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t o = (int64_t)blockIdx.y * n;
  const bool on = i < n && graded_x(spikes, flags, o + i) != 0.f;
  const uint32_t word = __ballot_sync(0xFFFFFFFFu, on);
  if ((threadIdx.x & (kWarp - 1)) == 0 && (i >> 5) < words)
    nz[(int64_t)blockIdx.y * words + (i >> 5)] = word;
}

__global__ void __launch_bounds__(kGradedThreads)
k_graded_pull(const int64_t* __restrict__ t_ptr, const int32_t* __restrict__ t_pre,
              const float* __restrict__ t_val, const float* __restrict__ spikes,
              const uint8_t* __restrict__ flags, const uint32_t* __restrict__ nz,
              const int n, const int words, const float w, float* __restrict__ rec) {
  extern __shared__ uint32_t smask[];  // this trial's nz words
  const int b = blockIdx.y;
  const int64_t o = (int64_t)b * n;
  for (int j = threadIdx.x; j < words; j += blockDim.x) smask[j] = nz[(int64_t)b * words + j];
  __syncthreads();
  const int lane = threadIdx.x & (kWarp - 1);
  const int warps = kGradedThreads / kWarp;
  for (int post = blockIdx.x * warps + (int)(threadIdx.x / kWarp); post < n;
       post += gridDim.x * warps) {  // warp-uniform
    float acc = 0.f;
    const int64_t k0 = t_ptr[post], k1 = t_ptr[post + 1];
    for (int64_t base = k0; base < k1; base += kWarp) {
      const int64_t k = base + lane;
      int pre = 0;
      bool on = false;
      if (k < k1) {
        pre = t_pre[k];
        on = (smask[pre >> 5] >> (pre & 31)) & 1u;
      }
      unsigned bits = __ballot_sync(0xFFFFFFFFu, on);
      float v = 0.f, x = 0.f;
      if (on) {
        v = t_val[k];
        x = graded_x(spikes, flags, o + pre);
      }
      while (bits) {
        const int j = __ffs(bits) - 1;
        bits &= bits - 1;
        acc = __fmaf_rn(__shfl_sync(0xFFFFFFFFu, v, j), __shfl_sync(0xFFFFFFFFu, x, j), acc);
      }
    }
    if (lane == 0) rec[o + post] = __fmul_rn(w, acc);
  }
}

__global__ void __launch_bounds__(kGradedThreads)
k_graded_step(const fis_engine E, const int64_t step, float* __restrict__ spikes,
              float* __restrict__ ring, const int ptr, const float* __restrict__ rec,
              const float* __restrict__ vstim) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = E.n;
  if (i >= n) return;
  const int b = blockIdx.y;
  const int64_t x = (int64_t)b * n + i;
  const uint32_t fl = E.flags[x];
  const fis_trial tr = E.trials[b];

  // the drive of this step (sim.py:848-861): given, or the Philox draw of the
  // exact engine -- word own % 4 of Philox4x32-10 at counter (i, own / 4,
  // trial lane) keyed by the trial's seed, a kick iff
  // float(word >> 8) * 2**-24 < f32(rate) * f32(DT / 1000)
  float vs = 0.f;
  if (vstim) {
    vs = vstim[x];
  } else {
    const float prob = __fmul_rn(E.rates[x], E.p.prob_scale);
    if (prob > 0.f) {
      const int64_t own = step - tr.start;
      const uint64_t quad = (uint64_t)(own >> 2);
      const Philox4 r4 = philox4((uint32_t)i, (uint32_t)quad, (uint32_t)(quad >> 32), tr.stream,
                                 (uint32_t)tr.seed, (uint32_t)(tr.seed >> 32));
      const int wsel = (int)(own & 3);
      const uint32_t word = wsel & 2 ? (wsel & 1 ? r4.x[3] : r4.x[2])
                                     : (wsel & 1 ? r4.x[1] : r4.x[0]);
      if (__fmul_rn((float)(word >> 8), 0x1p-24f) < prob) vs = E.p.kick;
    }
  }

  // refractory counter and gate with the (possibly graded) previous spikes
  const float s_prev = spikes[x];
  const float r = __fmul_rn(__fadd_rn(E.refrac[x], 1.f), __fsub_rn(1.f, s_prev));
  const float rs = (fl & FIS_FL_NOREFRAC) ? 0.f : E.p.refrac_steps;
  const float gate = r >= rs ? 1.f : 0.f;
  // delayed input of slot ptr, then the slot takes this step's product
  const float m_in = (fl & (FIS_FL_IN_OFF | FIS_FL_SILENCED)) ? 0.f : 1.f;
  float* slot = ring + ((int64_t)b * E.p.buf_len + ptr) * n + i;
  const float delayed = __fmul_rn(*slot, m_in);
  const float g = E.g[x];
  const float gn = __fadd_rn(__fmul_rn(g, E.p.a_syn), __fmul_rn(delayed, gate));
  *slot = rec[x];
  // membrane with the previous conductance, hold, threshold, reset
  float v = __fadd_rn(E.v[x], vs);
  v = __fadd_rn(v, __fmul_rn(E.p.a_mem, __fsub_rn(g, __fsub_rn(v, E.p.v_rest))));
  const bool hold = (fl & FIS_FL_HOLD) != 0;
  v = __fadd_rn(__fmul_rn(v, hold ? 0.f : 1.f), hold ? tr.v_clamp : 0.f);
  const float m_fire = (fl & FIS_FL_FIRE_OFF) ? 0.f : 1.f;
  const float s = __fmul_rn(v > E.p.v_th ? 1.f : 0.f, m_fire);
  v = __fsub_rn(v, __fmul_rn(__fsub_rn(v, E.p.v_reset), s));
  E.v[x] = v;
  E.refrac[x] = r;
  E.g[x] = __fsub_rn(gn, __fmul_rn(gn, s));
  spikes[x] = s;
}

}  // namespace
}  // namespace fis

using namespace fis;

extern "C" {

int fis_graded_step(const fis_engine* e, int64_t step, const int64_t* t_ptr,
                    const int32_t* t_pre, const float* t_val, float* spikes, float* ring,
                    int32_t ptr, float* rec, const float* vstim, void* stream) {
  if (!e || !t_ptr || !t_pre || !t_val || !spikes || !ring || !rec) return FIS_E_ARG;
  if (!e->v || !e->g || !e->refrac || !e->flags || !e->rates || !e->trials) return FIS_E_ARG;
  if (e->n < 1 || e->batch < 1 || e->batch > 65535) return FIS_E_ARG;
  if (e->p.buf_len < 1 || ptr < 0 || ptr >= e->p.buf_len) return FIS_E_BOUNDS;
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid((e->n + kGradedThreads - 1) / kGradedThreads, e->batch);
  // the nonzero mask lives after the [B][N] product in the scratch
  const int words = (e->n + kWarp - 1) / kWarp;
  uint32_t* nz = reinterpret_cast<uint32_t*>(rec + (int64_t)e->batch * e->n);
  k_graded_nz<<<grid, kGradedThreads, 0, st>>>(spikes, e->flags, e->n, words, nz);
  // a few CTAs per SM share the rows of a trial, each loading the mask once
  int sms = 0, dev = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
    sms = 148;
  const int per_trial = (sms * 8 + e->batch - 1) / e->batch;
  const int rows_cta = kGradedThreads / kWarp;
  const int need = (e->n + rows_cta - 1) / rows_cta;
  const dim3 pgrid(per_trial < need ? per_trial : need, e->batch);
  const size_t smem = (size_t)words * sizeof(uint32_t);
  if (smem > 48 * 1024) {
    cudaError_t a = cudaFuncSetAttribute(k_graded_pull, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (a != cudaSuccess) return (int)a;
  }
  k_graded_pull<<<pgrid, kGradedThreads, smem, st>>>(t_ptr, t_pre, t_val, spikes, e->flags, nz,
                                                     e->n, words, e->p.w_scale, rec);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return (int)err;
  k_graded_step<<<grid, kGradedThreads, 0, st>>>(*e, step, spikes, ring, ptr, rec, vstim);
  return (int)cudaGetLastError();
}

}  // extern "C"
