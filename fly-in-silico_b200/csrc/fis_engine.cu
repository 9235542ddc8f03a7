// The fused LIF engine for sm_100a.
//
// What one block of K steps (K <= the axonal lag L = buf_len + 1 = 20) does:
//
//   phase A  k_scatter   the spikes of steps t0-L .. t0+K-1-L reach the
//                        conductance exactly at steps t0 .. t0+K-1 (written
//                        into the reference's ring one step after the spike,
//                        read buf_len steps later; sim.py:887-897).  Their CSR
//                        rows are pushed into a scratch ring of K int32 slots
//                        with integer atomics, a warp per (spike, chunk of
//                        the row).  Integer sums make the order irrelevant.
//   phase B  k_update    every neuron of every trial advances K steps with
//                        its state in registers: refractory counter and gate,
//                        delayed input, conductance, Poisson drive (Philox),
//                        membrane, hold, threshold, reset (sim.py:921-952).
//                        Nothing inside a block depends on a spike of the same
//                        block, because a spike needs L steps to arrive; so
//                        the dense state is read and written once per K steps
//                        instead of once per step.
//
// The reference applies m_out to the spikes of step u at step u+1
// (sim.py:910-913).  Inside a block that mask is the block's own; for the last
// step of a block it is the next block's, so the last list is written
// unfiltered and phase A of the next block filters it.
//
// Floating point follows the reference's operation order one rounding at a
// time (__f*_rn intrinsics, never contracted into FMA): the result is the same
// bits as the reference's float32 torch arithmetic.

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "fis_common.cuh"

namespace fis {
namespace {

constexpr int kUpdThreads = 256;
constexpr int kScatThreads = 256;
constexpr int kScatWarps = kScatThreads / kWarp;
constexpr int kMaxLists = 11264;  // prefix entries in dynamic shared memory (44 KB)

// Bulk asynchronous shared -> global copy (sm_90+ cp.async.bulk, the TMA
// engine): both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_store(void* gmem, const void* smem, unsigned bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(gmem),
               "r"(sa), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}
// Order this thread's generic-proxy shared-memory writes before later
// async-proxy (bulk copy) reads of them.
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// x mod m for 0 <= x < 4m (slot arithmetic on small offsets).
__device__ __forceinline__ int wrap(int x, int m) {
  while (x >= m) x -= m;
  return x;
}

// mbarrier and bulk (TMA) loads into shared memory.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                   smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
// Bulk copy global -> shared, completing `bytes` transactions on `bar`.
__device__ __forceinline__ void bulk_load(void* smem, const void* gmem, unsigned bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_addr(smem)),
      "l"(gmem), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Wait for phase `parity` of `bar`, giving up after `limit` polls (each poll
// may suspend the thread briefly).  Returns whether the phase completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned limit) {
  const unsigned a = smem_addr(bar);
  for (unsigned it = 0; it < limit; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
constexpr unsigned kWaitPolls = 1u << 22;   // far beyond any copy's latency

// Ring rows are padded per trial to a whole number of update tiles.
constexpr int kTile = 256;
__host__ __device__ __forceinline__ int ring_row(int n) { return (n + kTile - 1) / kTile * kTile; }

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cached[dev] = v;
  }
  return cached[dev];
}

// ---------------------------------------------------------------------------
// phase A: scatter spike lists into the scratch ring
// ---------------------------------------------------------------------------

// Source list kk (0 <= kk < nsrc) holds the spikes of step u = u_first + kk;
// its rows go to ring slot kk, or (slot_mode 1) to the slot of the reference's
// delay ring that holds the input of step u + lag, which is (u + 1) % buf_len.  With `filter_last`, the
// list of step t0-1 (the last one written by the previous block) is checked
// against m_out: when it is also a source, its dead entries are skipped; when
// it is not (K < L), its dead entries are marked for the block that will
// consume it.
struct ScatterArgs {
  int b0, nb;
  int nsrc;
  int64_t u_off;      // u_first = clock + u_off
  int slot_mode;      // 0: slot kk; 1: the reference ring slot (u + 1) % buf_len
  int zero_next;      // zero list_len of steps clock .. clock+zero_next-1
  int filter_last;    // handle the list of step clock-1 as described above
  int32_t* ring;      // slot stride nb*trial_stride elements
  int trial_stride;   // elements per trial row of `ring`
  int half;           // elements are biased uint16 (see fis.h), else int32
};

// The value that marks an empty pair of biased uint16 ring elements.
constexpr uint32_t kEmptyPair = 0x80008000u;

__global__ void __launch_bounds__(kScatThreads)
k_scatter(const fis_engine E, const ScatterArgs A) {
  extern __shared__ int32_t pre_sum[];
  const int n = E.n;
  const int B = E.batch;
  const int L = E.p.lag;
  const fis_clock ck = *E.clock;
  const int64_t t0 = ck.step;
  const int64_t u_first = t0 + A.u_off;  // u_off is -lag: u_first = t0 mod lag
  const int64_t u_last = t0 - 1;
  // slots of step u_first + kk: (ck.slot + kk) mod L and (ck.slot2 + L + kk) mod 2L
  const int slot_last = wrap(ck.slot + L - 1, L);
  const int slot2_last = wrap(ck.slot2 + 2 * L - 1, 2 * L);
  const int t_mod_r = A.slot_mode ? (int)mod_pos(t0, E.p.buf_len) : 0;
  // Is the list of step t0-1 one of the sources?
  const int kk_last = (int)(u_last - u_first);
  const bool last_is_src = A.filter_last && kk_last >= 0 && kk_last < A.nsrc;
  const bool extra = A.filter_last && !last_is_src && u_last >= 0;
  const int nlists = (A.nsrc + (extra ? 1 : 0)) * A.nb;

  // Prefix sum of the list lengths: entries [j*..] of list j, j = kk*nb + bl.
  {
    const int per = (nlists + kScatThreads - 1) / kScatThreads;
    const int j0 = threadIdx.x * per;
    int32_t acc = 0;
    for (int j = j0; j < j0 + per && j < nlists; ++j) {
      const int kk = j / A.nb, bl = j - kk * A.nb;
      const int64_t u = (kk < A.nsrc) ? u_first + kk : u_last;
      const int s2 = (kk < A.nsrc) ? wrap(ck.slot2 + L + kk, 2 * L) : slot2_last;
      int32_t len = 0;
      if (u >= 0) len = E.list_len[s2 * B + A.b0 + bl];
      pre_sum[j] = len;  // provisional
      acc += len;
    }
    __shared__ int32_t part[kScatThreads];
    part[threadIdx.x] = acc;
    __syncthreads();
    // inclusive scan of the per-thread partial sums (Hillis-Steele)
    for (int off = 1; off < kScatThreads; off <<= 1) {
      const int32_t x = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
      __syncthreads();
      part[threadIdx.x] += x;
      __syncthreads();
    }
    int32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0;
    for (int j = j0; j < j0 + per && j < nlists; ++j) {
      const int32_t len = pre_sum[j];
      pre_sum[j] = run;
      run += len;
    }
    __syncthreads();
    if (threadIdx.x == 0) pre_sum[nlists] = part[kScatThreads - 1];
    __syncthreads();
  }
  const int32_t total = pre_sum[nlists];

  // Lists that the following update phase will write start empty.
  if (blockIdx.x == 0) {
    for (int j = threadIdx.x; j < A.zero_next * A.nb; j += blockDim.x) {
      const int kk = j / A.nb, bl = j - kk * A.nb;
      E.list_len[wrap(ck.slot2 + kk, 2 * L) * B + A.b0 + bl] = 0;
    }
  }

  const int lane = threadIdx.x & (kWarp - 1);
  const int warp = threadIdx.x / kWarp;
  const int64_t slot_stride = (int64_t)A.nb * A.trial_stride;
  for (int32_t w = blockIdx.x * kScatWarps + warp; w < total; w += gridDim.x * kScatWarps) {
    // list holding work item w: largest j with pre_sum[j] <= w
    int lo = 0, hi = nlists - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pre_sum[mid] <= w) lo = mid; else hi = mid - 1;
    }
    const int j = lo;
    const int kk = j / A.nb, bl = j - kk * A.nb;
    const int b = A.b0 + bl;
    const bool is_src = kk < A.nsrc;
    const int64_t u = is_src ? u_first + kk : u_last;
    const int su = is_src ? wrap(ck.slot + kk, L) : slot_last;
    uint32_t* lst = E.lists + ((int64_t)su * B + b) * E.list_cap;
    const int32_t idx = w - pre_sum[j];
    if (idx >= E.list_cap) continue;
    const uint32_t e = lst[idx];
    const uint32_t pre = entry_pre(e);
    if (e == kDeadEntry || pre >= (uint32_t)n) continue;
    if (A.filter_last && u == u_last) {
      const uint8_t fl = E.flags[(int64_t)b * n + pre];
      if (fl & (FIS_FL_OUT_OFF | FIS_FL_SILENCED)) {
        if (!is_src && lane == 0) lst[idx] = kDeadEntry;
        continue;
      }
    }
    if (!is_src) continue;
    const int64_t r0 = E.row_ptr[pre], r1 = E.row_ptr[pre + 1];
    const int64_t lo_e = r0 + (int64_t)entry_chunk(e) * E.chunk;
    const int64_t hi_e = min(r1, lo_e + (int64_t)E.chunk);
    if (lo_e >= hi_e) continue;
    // slot_mode 1: (u + 1) mod buf_len = (t0 + kk) mod buf_len, as lag = buf_len + 1
    const int slot = A.slot_mode ? wrap(t_mod_r + kk, E.p.buf_len) : kk;
    const int64_t row = slot * slot_stride + (int64_t)bl * A.trial_stride;
    int32_t* dst = A.ring + row;
    uint16_t* dst16 = reinterpret_cast<uint16_t*>(A.ring) + row;
    // 16-byte vector loads: four edges per lane, 128 edges per warp pass.
    for (int64_t p = (lo_e & ~(int64_t)3) + 4 * lane; p < hi_e; p += 4 * kWarp) {
      const uint4 q = __ldg(reinterpret_cast<const uint4*>(E.edges + p));
      const uint32_t wv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int64_t pe = p + c;
        if (pe >= lo_e && pe < hi_e) {
          const int post = edge_post(wv[c]);
          if (post < n) {
            if (A.half) {
              // the pair (post & ~1, post | 1) shares one 32-bit word (rows
              // are even-sized, so pairs never straddle a row)
              uint32_t* w = reinterpret_cast<uint32_t*>(dst16 + (post & ~1));
              atomicAdd(w, (uint32_t)edge_count(wv[c]) << ((post & 1) * 16));
            } else {
              atomicAdd(dst + post, edge_count(wv[c]));
            }
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// phase B: K fused steps per neuron
// ---------------------------------------------------------------------------

// One neuron's state for the step loop.
struct Neuron {
  float v, g, r;      // membrane, conductance, refractory counter
  float keep;         // 1 - spike of the previous step
  float m_fire, m_in, m_hold, v_hold, rs;
  float v_th;         // threshold; +inf under the fire mask (see lif_step)
  bool silenced;
};

// One step of sim.py:921-952 for one neuron, the reference's operation order
// one rounding at a time.  Returns the spike (0 or 1).
__device__ __forceinline__ float lif_step(Neuron& s, const fis_lif_params& P, int32_t c_in,
                                          float vstim) {
  // refractory counter and gate (sim.py:921-923)
  s.r = __fmul_rn(__fadd_rn(s.r, 1.f), s.keep);
  const float gate = (s.r >= s.rs) ? 1.f : 0.f;
  // delayed input and the new conductance (sim.py:928-929); a silenced neuron
  // has no incoming synapses (sim.py:324-336)
  const int32_t ck = s.silenced ? 0 : c_in;
  const float delayed = __fmul_rn(__fmul_rn(P.w_scale, __int2float_rn(ck)), s.m_in);
  const float gn = __fadd_rn(__fmul_rn(s.g, P.a_syn), __fmul_rn(delayed, gate));
  // membrane with the previous conductance (sim.py:936-938)
  float v = __fadd_rn(s.v, vstim);
  v = __fadd_rn(v, __fmul_rn(P.a_mem, __fsub_rn(s.g, __fsub_rn(v, P.v_rest))));
  // hold, threshold, reset (sim.py:943-952).  spikes = (v > v_th) * m_fire
  // with m_fire in {0, 1} is +0 or 1; comparing against +inf where m_fire is
  // 0 gives the same bits (a finite v never exceeds +inf) without the multiply.
  v = __fadd_rn(__fmul_rn(v, s.m_hold), s.v_hold);
  const bool fire = v > s.v_th;
  const float sp = fire ? 1.f : 0.f;
  s.v = __fsub_rn(v, __fmul_rn(__fsub_rn(v, P.v_reset), sp));
  s.g = __fsub_rn(gn, __fmul_rn(gn, sp));
  s.keep = fire ? 0.f : 1.f;
  return sp;
}

// The step loop over K steps: `kDrive` selects whether any lane of the warp is
// driven, so warps without drive carry no drive logic at all.  Returns the
// number of spikes of this neuron (exact in float).
// The staged input of step k for this thread: an int32 column, or (kHalf) the
// thread's half of a biased uint16 pair, masked to zero for silenced neurons
// and padding lanes.
struct Staged {
  const int32_t* col;  // this thread's word of slot 0; slot k is kUpdThreads words further
  int shift;           // kHalf: 16 for the high half of the pair, else 0
  int32_t mask;        // kHalf: 0 for a silenced neuron, else all ones
};

template <bool kHalf>
__device__ __forceinline__ int32_t staged(const Staged& s, int k) {
  const int32_t w = s.col[k * kUpdThreads];
  if (kHalf) return ((int32_t)(((uint32_t)w >> s.shift) & 0xFFFFu) - 0x8000) & s.mask;
  return w & s.mask;
}

template <bool kTape, bool kDrive, bool kHalf>
__device__ __forceinline__ float step_loop(Neuron& st, const fis_engine& E, int K, int ka,
                                           int kb, bool valid, uint32_t dmask,
                                           const Staged& in, uint32_t* sbal, int64_t sidx) {
  const float kick = E.p.kick;
  // fired steps as bits, the latest step lowest: m = 2 m + spike per step, an
  // exact float of at most 20 bits (bookkeeping, not model state, so one fused
  // multiply-add is fine here)
  float nspk = 0.f;
  // Every lane stores the warp's ballot word (the same value to the same
  // address), so the store needs no lane predicate.
  if (ka == 0 && kb == K) {
    // Lanes past the last neuron run the same arithmetic on inert values
    // (never above an infinite threshold) and store nothing.
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
      const int32_t c_in = staged<kHalf>(in, k);
      float vstim = 0.f;
      if (kTape) vstim = valid ? E.vstim[sidx] : 0.f;
      else if (kDrive) vstim = ((dmask >> k) & 1u) ? kick : 0.f;
      const float sp = lif_step(st, E.p, c_in, vstim);
      sbal[k] = __ballot_sync(0xFFFFFFFFu, sp != 0.f);
      nspk = __fmaf_rn(nspk, 2.f, sp);
    }
  } else {
#pragma unroll 1
    for (int k = 0; k < K; ++k) {
      const int32_t c_in = staged<kHalf>(in, k);
      float sp = 0.f;
      if (valid && k >= ka && k < kb) {
        float vstim = 0.f;
        if (kTape) vstim = E.vstim[sidx];
        else if (kDrive) vstim = ((dmask >> k) & 1u) ? kick : 0.f;
        sp = lif_step(st, E.p, c_in, vstim);
      }
      sbal[k] = __ballot_sync(0xFFFFFFFFu, sp != 0.f);
      nspk = __fmaf_rn(nspk, 2.f, sp);
    }
  }
  return nspk;
}

// Grid: one CTA per (trial of the group, tile of 256 neurons); the trial's
// rows of the scratch ring are padded to ring_row(n), so each CTA's slice of
// a ring slot is one aligned 1 KB line of the async bulk copy engine.
template <bool kTape, bool kHalf>
__global__ void __launch_bounds__(kUpdThreads, 5)
k_update(const fis_engine E, const int b0, const int nb, const int K,
         int32_t* __restrict__ ring, float* __restrict__ spikes_out,
         const int bump) {
  // The block's delayed input, one column per thread: staged here so the step
  // loop stays rolled (a compact body that fits the instruction cache) and can
  // index it by step.  With kHalf the staged values are the ring's biased
  // uint16 pairs, decoded into sring in place.
  __shared__ __align__(16) int32_t sring[FIS_MAX_BLOCK][kUpdThreads];
  __shared__ __align__(16) uint32_t szero[kUpdThreads];            // source of the clearing
  __shared__ uint32_t sdrive[kUpdThreads];                         // kick bit per step
  __shared__ float sprob[kUpdThreads];                             // Bernoulli p per lane
  __shared__ uint32_t sbal[kUpdThreads / kWarp][FIS_MAX_BLOCK];    // raster words per step
  __shared__ __align__(8) uint64_t sbar;                           // staging barrier
  const int n = E.n;
  const int L = E.p.lag;
  const int Wd = (n + kWarp - 1) / kWarp;
  const int NR = ring_row(n);
  const int bl = blockIdx.y;    // trial of the group
  const int tile = blockIdx.x;  // 256-neuron tile
  const int i = tile * kTile + threadIdx.x;
  const int b = b0 + bl;
  const int lane = threadIdx.x & (kWarp - 1);
  const int wib = threadIdx.x / kWarp;
  const bool valid = i < n;
  const bool warp_valid = (i - lane) < n;
  const fis_clock ck = *E.clock;
  const int64_t t0 = ck.step;
  const fis_trial tr = E.trials[b];
  const int ka = (int)max((int64_t)0, min(tr.start - t0, (int64_t)K));
  const int kb = (int)max((int64_t)0, min(tr.end - t0, (int64_t)K));
  const int64_t sidx = (int64_t)b * n + i;

  if (ka >= kb) {
    // The trial does not run in this block (not started, or finished and
    // frozen in place): only return its ring slots to empty, as scatters of
    // its last spikes may still land there.  Uniform across the CTA.
    if (threadIdx.x == 0) {
      int32_t* rt = ring + (int64_t)bl * NR + tile * kTile;
      uint16_t* rt16 = reinterpret_cast<uint16_t*>(ring) + (int64_t)bl * NR + tile * kTile;
      for (int j = threadIdx.x; j < kTile; ++j) szero[j] = kHalf ? kEmptyPair : 0u;
      fence_proxy_async_shared();
      const int sst = nb * NR;
      for (int k = 0; k < K; ++k) {
        if (kHalf) bulk_store(rt16 + (int64_t)k * sst, szero, kTile * 2);
        else bulk_store(rt + (int64_t)k * sst, szero, kTile * 4);
      }
      bulk_commit();
      bulk_wait_all();
    }
  } else {
  if (threadIdx.x == 0) {
    mbar_init(&sbar, 1);
    fence_mbar_init();
  }
  __syncthreads();  // the barrier exists before anyone arrives or waits
  uint32_t fl = 0;
  float rate = 0.f;
  Neuron st;
  st.v = st.g = st.r = 0.f;
  if (valid && ka < kb) {
    st.v = E.v[sidx];
    st.g = E.g[sidx];
    st.r = E.refrac[sidx];
    fl = E.flags[sidx];
    rate = E.rates[sidx];
  }
  st.silenced = fl & FIS_FL_SILENCED;

  // Stage the delayed input of the K steps: lanes 0..K-1 of warp 0 each
  // bulk-copy one slot of this tile (TMA) into shared memory, completing on
  // one mbarrier that every thread then waits on.  A silenced neuron has no
  // incoming synapses (sim.py:324-336): its input is masked to zero per step.
  const int sstride = nb * NR;  // elements; < 2**31 / FIS_MAX_BLOCK, checked on the host
  int32_t* rtile = ring + (int64_t)bl * NR + tile * kTile;                 // int32 ring
  uint16_t* rtile16 = reinterpret_cast<uint16_t*>(ring) + (int64_t)bl * NR + tile * kTile;
  const unsigned slot_bytes = kHalf ? kTile * 2 : kTile * 4;
  if (threadIdx.x < kWarp) {
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&sbar, slot_bytes * (unsigned)K);
    __syncwarp();
    if (threadIdx.x < K && !E.inject_stall) {
      const void* src = kHalf ? (const void*)(rtile16 + (int64_t)threadIdx.x * sstride)
                              : (const void*)(rtile + (int64_t)threadIdx.x * sstride);
      bulk_load(&sring[threadIdx.x][0], src, slot_bytes, &sbar);
    }
  }

  const int slot0 = ck.slot;  // ring-of-lists slot of step t0
  // this warp's raster words, one per slot: bits[b][word][slot]
  uint32_t* bitrow = E.bits + ((int64_t)b * Wd + (i >> 5)) * L;
  bool s_prev = false;
  if (warp_valid && t0 - 1 >= tr.start && t0 >= 1)
    s_prev = (bitrow[slot0 == 0 ? L - 1 : slot0 - 1] >> lane) & 1u;
  st.keep = s_prev ? 0.f : 1.f;
  st.m_fire = (!valid || (fl & FIS_FL_FIRE_OFF)) ? 0.f : 1.f;
  st.v_th = st.m_fire != 0.f ? E.p.v_th : __int_as_float(0x7f800000);
  st.m_in = (fl & FIS_FL_IN_OFF) ? 0.f : 1.f;
  const bool hold = fl & FIS_FL_HOLD;
  st.m_hold = hold ? 0.f : 1.f;
  st.v_hold = hold ? tr.v_clamp : 0.f;
  st.rs = (fl & FIS_FL_NOREFRAC) ? 0.f : E.p.refrac_steps;
  const int64_t own0 = t0 - tr.start;  // the trial's own step at k = 0

  // Wait for the staged input.  If any thread's wait runs out, the whole CTA
  // (decided together, so every warp stays whole for its ballots) flags the
  // error for the host, waits once more for copies still writing its shared
  // memory, and skips the update, still reaching the final barrier.
  const unsigned polls = E.wait_polls ? E.wait_polls : kWaitPolls;
  const bool staged_ok = mbar_wait(&sbar, 0, polls);
  if (__syncthreads_or(!staged_ok)) {
    if (threadIdx.x == 0) atomicOr(E.done + 1, (uint32_t)FIS_ERR_STAGE);
    if (!staged_ok) mbar_wait(&sbar, 0, polls);
  } else {
  // The staged slots are in shared memory: warp 0 returns them to empty in
  // the ring with one bulk store per slot (lanes 0..K-1), so the scratch ring
  // needs no clearing pass and the step loop no stores.
  if (threadIdx.x < kWarp) {
    const uint32_t empty = kHalf ? kEmptyPair : 0u;
#pragma unroll
    for (int j = 0; j < kTile / kWarp; ++j) szero[j * kWarp + threadIdx.x] = empty;
    fence_proxy_async_shared();
    __syncwarp();
    if (threadIdx.x < K) {
      const int k = threadIdx.x;
      if (kHalf) bulk_store(rtile16 + (int64_t)k * sstride, szero, kTile * 2);
      else bulk_store(rtile + (int64_t)k * sstride, szero, kTile * 4);
      bulk_commit();
    }
  }

  // Every lane of a warp runs the same loop (the choice depends on the trial
  // and on the warp's ballot only), so every lane reaches each ballot.
  // Poisson drive of the whole block (sim.py:859-861), before the step loop:
  // draw j of neuron i is word j % 4 of Philox4x32-10 at counter
  // (i, j / 4, trial lane); the (neuron, quad) pairs of the warp's driven
  // neurons are spread over all 32 lanes, and each pair ORs its kick bits into
  // the neuron's mask.
  uint32_t dmask = 0;
  bool warp_driven = false;
  if (!kTape) {
    const float prob = __fmul_rn(rate, E.p.prob_scale);
    const unsigned D = __ballot_sync(0xFFFFFFFFu, valid && ka < kb && prob > 0.f);
    warp_driven = D != 0u;
    if (D) {
      sdrive[threadIdx.x] = 0u;
      sprob[threadIdx.x] = prob;
      __syncwarp();
      const int64_t q0 = (own0 + ka) >> 2;
      const int nq = (int)(((own0 + kb - 1) >> 2) - q0) + 1;
      const int total = __popc(D) * nq;
      const int wbase = threadIdx.x - lane;
      for (int it = lane; it < total; it += kWarp) {
        const int jd = it / nq, qq = it - jd * nq;
        unsigned m = D;
        for (int t = 0; t < jd; ++t) m &= m - 1;
        const int j = __ffs(m) - 1;
        const int64_t quad = q0 + qq;
        const Philox4 r4 = philox4((uint32_t)(i - lane + j), (uint32_t)quad,
                                   (uint32_t)((uint64_t)quad >> 32), tr.stream,
                                   (uint32_t)tr.seed, (uint32_t)(tr.seed >> 32));
        const float pj = sprob[wbase + j];
        uint32_t bits = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int k = (int)(quad * 4 + q - own0);
          if (k >= ka && k < kb && __fmul_rn((float)(r4.x[q] >> 8), 0x1p-24f) < pj)
            bits |= 1u << k;
        }
        if (bits) atomicOr(&sdrive[wbase + j], bits);
      }
      __syncwarp();
      dmask = sdrive[threadIdx.x];
    }
  }

  // Each thread waited for the staged copies itself (with kHalf it reads its
  // neighbour's word too).  The drive precompute runs after the wait, so warps
  // without driven neurons do not wait for those that have.
  Staged in;
  in.col = kHalf ? &sring[0][threadIdx.x >> 1] : &sring[0][threadIdx.x];
  in.shift = (threadIdx.x & 1) * 16;
  in.mask = st.silenced ? 0 : -1;
  float nspk;
  if (kTape)
    nspk = step_loop<true, false, kHalf>(st, E, K, ka, kb, valid, 0u, in, sbal[wib], sidx);
  else if (warp_driven)
    nspk = step_loop<false, true, kHalf>(st, E, K, ka, kb, valid, dmask, in, sbal[wib], sidx);
  else
    nspk = step_loop<false, false, kHalf>(st, E, K, ka, kb, valid, 0u, in, sbal[wib], sidx);
  __syncwarp();
  // the raster words of the K steps into the ring of the last L steps
  if (lane < K && warp_valid) {
    const int sl = slot0 + lane < L ? slot0 + lane : slot0 + lane - L;
    bitrow[sl] = sbal[wib][lane];
  }

  if (valid && ka < kb) {
    E.v[sidx] = st.v;
    E.g[sidx] = st.g;
    E.refrac[sidx] = st.r;
  }
  if (spikes_out && valid) spikes_out[sidx] = (st.keep == 0.f) ? 1.f : 0.f;

  // Spike lists and recording for the (rare) steps this neuron fired.
  uint32_t fired = (uint32_t)nspk;  // bit j is step K-1-j
  if (fired) {
    const int B = E.batch;
    const bool out_on = !(fl & (FIS_FL_OUT_OFF | FIS_FL_SILENCED));
    const int nch = E.nchunks[i];
    const int slot20 = ck.slot2;
    while (fired) {
      const int k = K - __ffs(fired);
      fired &= fired - 1;
      const int sl = slot0 + k < L ? slot0 + k : slot0 + k - L;
      const int sl2 = slot20 + k < 2 * L ? slot20 + k : slot20 + k - 2 * L;
      if ((out_on || k == K - 1) && nch > 0) {
        const int32_t pos = atomicAdd(E.list_len + (int64_t)sl2 * B + b, nch);
        uint32_t* dst = E.lists + ((int64_t)sl * B + b) * E.list_cap;
        for (int q = 0; q < nch; ++q)
          if (pos + q < E.list_cap) dst[pos + q] = ((uint32_t)i << 8) | (uint32_t)q;
      }
      if (tr.rec >= 0 && tr.rec < E.n_recs && tr.bin_steps > 0) {
        const int64_t own = own0 + k;
        const int64_t bin = own < 0x7FFFFFFF ? (int64_t)((int)own / tr.bin_steps)
                                              : own / tr.bin_steps;
        if (bin < tr.n_bins) atomicAdd(E.recs[tr.rec] + bin * n + i, 1);
      }
    }
  }

  // The clearing copies complete before the CTA ends (szero must stay valid
  // while they read it, and the next scatter adds into these lines).
  if (threadIdx.x < K) bulk_wait_all();
  }  // the staged input arrived
  }  // the trial runs in this block

  if (bump) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned prev = atomicAdd(E.done, 1u);
      if (prev == gridDim.x * gridDim.y - 1) {
        *E.done = 0u;
        fis_clock next;
        next.step = t0 + K;
        next.slot = wrap(ck.slot + K, L);
        next.slot2 = wrap(ck.slot2 + K, 2 * L);
        *E.clock = next;
        __threadfence();
      }
    }
  }
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------

// scratch [buf_len][nb][n] int32 -> out [nb][buf_len][n] float, w_scale * count
__global__ void k_ring_to_f32(const fis_engine E, int b0, int nb,
                              const int32_t* __restrict__ scratch,
                              float* __restrict__ out) {
  const int n = E.n, R = E.p.buf_len;
  const int64_t total = (int64_t)nb * R * n;
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(x % n);
    const int64_t rest = x / n;
    const int s = (int)(rest % R);
    const int bl = (int)(rest / R);
    const uint8_t fl = E.flags[(int64_t)(b0 + bl) * n + i];
    const int32_t cnt = (fl & FIS_FL_SILENCED) ? 0 : scratch[((int64_t)s * nb + bl) * n + i];
    out[x] = __fmul_rn(E.p.w_scale, __int2float_rn(cnt));
  }
}

__global__ void k_spikes_f32(const fis_engine E, int b0, int nb, int64_t step,
                             float* __restrict__ out) {
  const int n = E.n, L = E.p.lag;
  const int Wd = (n + kWarp - 1) / kWarp;
  const int64_t total = (int64_t)nb * n;
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int bl = (int)(x / n), i = (int)(x % n);
    const uint32_t wv = E.bits[((int64_t)(b0 + bl) * Wd + (i >> 5)) * L + mod_pos(step, L)];
    out[x] = ((wv >> (i & 31)) & 1u) ? 1.f : 0.f;
  }
}

__global__ void k_load_spikes(const fis_engine E, int b0, int nb,
                              const float* __restrict__ sp) {
  const int n = E.n, B = E.batch, L = E.p.lag;
  const int Wd = (n + kWarp - 1) / kWarp;
  const fis_clock ck = *E.clock;
  const int64_t u = ck.step - 1;
  const int su = wrap(ck.slot + L - 1, L), su2 = wrap(ck.slot2 + 2 * L - 1, 2 * L);
  const int64_t npad = (int64_t)Wd * kWarp;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u < 0 || gid >= (int64_t)nb * npad) return;
  const int bl = (int)(gid / npad);
  const int i = (int)(gid - (int64_t)bl * npad);
  const int b = b0 + bl;
  const bool fired = i < n && sp[(int64_t)bl * n + i] != 0.f;
  const unsigned bal = __ballot_sync(0xFFFFFFFFu, fired);
  if ((threadIdx.x & 31) == 0) E.bits[((int64_t)b * Wd + (i >> 5)) * L + su] = bal;
  if (fired) {
    const int nch = E.nchunks[i];
    if (nch > 0) {
      const int32_t pos = atomicAdd(E.list_len + (int64_t)su2 * B + b, nch);
      uint32_t* dst = E.lists + ((int64_t)su * B + b) * E.list_cap;
      for (int q = 0; q < nch; ++q)
        if (pos + q < E.list_cap) dst[pos + q] = ((uint32_t)i << 8) | (uint32_t)q;
    }
  }
}

// dst[r][b][i] += src[r][b][i] with separate row and trial strides; with
// `half` the destination is the biased uint16 ring (each element is written
// by one thread only, so a plain 16-bit add is exact).
__global__ void k_add_rows(int n, int nb, int rows, const int32_t* __restrict__ src, int64_t ss,
                           int64_t st, int32_t* __restrict__ dst, int64_t ds, int64_t dt,
                           int half) {
  const int64_t total = (int64_t)rows * nb * n;
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(x % n);
    const int64_t rb = x / n;
    const int bb = (int)(rb % nb);
    const int64_t r = rb / nb;
    const int32_t v = src[r * ss + bb * st + i];
    if (half) {
      uint16_t* d = reinterpret_cast<uint16_t*>(dst) + r * ds + bb * dt + i;
      *d = (uint16_t)(*d + (uint16_t)v);
    } else {
      dst[r * ds + bb * dt + i] += v;
    }
  }
}

__global__ void k_fill32(uint32_t* __restrict__ dst, int64_t words, uint32_t value) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < words;
       x += (int64_t)gridDim.x * blockDim.x)
    dst[x] = value;
}

int launch_status() {
  const cudaError_t err = cudaGetLastError();
  return (int)err;
}

int grid_for(int64_t total, int threads) {
  const int64_t cap = (int64_t)sm_count() * 16;
  int64_t g = (total + threads - 1) / threads;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

int check_range(const fis_engine* e, int32_t b0, int32_t nb) {
  if (b0 < 0 || nb < 1 || (int64_t)b0 + nb > e->batch) return FIS_E_BOUNDS;
  return FIS_OK;
}

}  // namespace
}  // namespace fis

using namespace fis;

extern "C" {

int fis_abi(void) { return FIS_ABI_VERSION; }
int fis_sizeof_engine(void) { return (int)sizeof(fis_engine); }
int fis_sizeof_trial(void) { return (int)sizeof(fis_trial); }

int fis_check(const fis_engine* e) {
  if (!e) return FIS_E_ARG;
  if (!e->row_ptr || !e->edges || !e->nchunks || !e->v || !e->g || !e->refrac ||
      !e->flags || !e->rates || !e->trials || !e->lists || !e->list_len ||
      !e->bits || !e->clock || !e->done)
    return FIS_E_ARG;
  if (e->n < 1 || e->n > (1 << 18) || e->batch < 1 || e->nnz < 0) return FIS_E_ARG;
  if (e->chunk < 128 || (e->chunk % 128) != 0) return FIS_E_ARG;
  if (e->list_cap < 1) return FIS_E_ARG;
  if (e->p.lag < 2 || e->p.buf_len != e->p.lag - 1) return FIS_E_ARG;
  if (e->n_recs < 0 || (e->n_recs > 0 && !e->recs)) return FIS_E_ARG;
  if (!aligned16(e->edges)) return FIS_E_ALIGN;
  return FIS_OK;
}

static int check_block(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps,
                       const int32_t* ring) {
  int rc = fis_check(e);
  if (rc) return rc;
  if ((rc = check_range(e, b0, nb))) return rc;
  if (!ring) return FIS_E_ARG;
  if (k_steps < 1 || k_steps > FIS_MAX_BLOCK || k_steps > e->p.lag) return FIS_E_BOUNDS;
  if (e->vstim && k_steps != 1) return FIS_E_BOUNDS;
  if ((k_steps + 1) * nb + 1 > kMaxLists) return FIS_E_BOUNDS;
  const int64_t rows = (int64_t)nb * ring_row(e->n);
  if (rows * FIS_MAX_BLOCK > 0x7FFFFFFFLL) return FIS_E_BOUNDS;
  if (((uintptr_t)ring & 15u) != 0) return FIS_E_ALIGN;
  return FIS_OK;
}

int fis_scatter(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps, int32_t* ring,
                void* stream) {
  const int rc = check_block(e, b0, nb, k_steps, ring);
  if (rc) return rc;
  ScatterArgs A;
  A.b0 = b0;
  A.nb = nb;
  A.nsrc = k_steps;
  A.u_off = -(int64_t)e->p.lag;
  A.slot_mode = 0;
  A.zero_next = k_steps;
  A.filter_last = 1;
  A.ring = ring;
  A.trial_stride = ring_row(e->n);
  A.half = e->ring16 ? 1 : 0;
  const size_t smem = sizeof(int32_t) * (size_t)((k_steps + 1) * nb + 1);
  k_scatter<<<sm_count() * 8, kScatThreads, smem, (cudaStream_t)stream>>>(*e, A);
  return launch_status();
}

int fis_update(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps, int32_t* ring,
               float* spikes_out, int32_t last_group, void* stream) {
  const int rc = check_block(e, b0, nb, k_steps, ring);
  if (rc) return rc;
  const dim3 ugrid(ring_row(e->n) / kTile, nb);
  const int bump = last_group ? 1 : 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (e->vstim) {
    if (e->ring16)
      k_update<true, true><<<ugrid, kUpdThreads, 0, st>>>(*e, b0, nb, k_steps, ring, spikes_out, bump);
    else
      k_update<true, false><<<ugrid, kUpdThreads, 0, st>>>(*e, b0, nb, k_steps, ring, spikes_out, bump);
  } else {
    if (e->ring16)
      k_update<false, true><<<ugrid, kUpdThreads, 0, st>>>(*e, b0, nb, k_steps, ring, spikes_out, bump);
    else
      k_update<false, false><<<ugrid, kUpdThreads, 0, st>>>(*e, b0, nb, k_steps, ring, spikes_out, bump);
  }
  return launch_status();
}

int fis_block(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps, int32_t* ring,
              float* spikes_out, int32_t last_group, void* stream) {
  const int rc = fis_scatter(e, b0, nb, k_steps, ring, stream);
  if (rc) return rc;
  return fis_update(e, b0, nb, k_steps, ring, spikes_out, last_group, stream);
}

static int record_if(bool on, void* const* events, int64_t idx, cudaStream_t st) {
  if (!on) return FIS_OK;
  return (int)cudaEventRecord((cudaEvent_t)events[idx], st);
}

int fis_advance(const fis_engine* e, int64_t steps, int32_t group, int32_t rows, int32_t* ring,
                float* spikes_out, void* const* events, int32_t n_pairs, int32_t every,
                void* stream) {
  int rc = fis_check(e);
  if (rc) return rc;
  if (steps < 0 || group < 1 || rows < 0 || !ring) return FIS_E_ARG;
  if (events && (n_pairs < 0 || every < 1)) return FIS_E_ARG;
  const int32_t B = (rows > 0 && rows < e->batch) ? rows : e->batch;
  const int kmax = e->p.lag < FIS_MAX_BLOCK ? e->p.lag : FIS_MAX_BLOCK;
  cudaStream_t st = (cudaStream_t)stream;
  int64_t left = steps;
  int64_t launch = 0;
  while (left > 0) {
    const int k = (int)(left < kmax ? left : kmax);
    float* sp = (left == k) ? spikes_out : nullptr;
    for (int32_t g0 = 0; g0 < B; g0 += group) {
      const int32_t nb = (B - g0) < group ? (B - g0) : group;
      if ((rc = fis_scatter(e, g0, nb, k, ring, stream))) return rc;
      const bool timed = events && (launch % every) == 0 && (launch / every) < n_pairs;
      if ((rc = record_if(timed, events, 2 * (launch / every), st))) return rc;
      if ((rc = fis_update(e, g0, nb, k, ring, sp, g0 + nb == B, stream))) return rc;
      if ((rc = record_if(timed, events, 2 * (launch / every) + 1, st))) return rc;
      ++launch;
    }
    left -= k;
  }
  return FIS_OK;
}

}  // extern "C"

namespace {
// Per-device side stream and events of fis_advance_overlap, created on first
// use and kept for the life of the process.
struct OverlapRes {
  cudaStream_t side = nullptr;
  cudaEvent_t after_sc[2] = {nullptr, nullptr};   // scatter of group gi done
  cudaEvent_t after_upd[2] = {nullptr, nullptr};  // update of group gi done
  cudaEvent_t block_done = nullptr;               // clock and lists of the block final
};
constexpr int kMaxOverlapDevices = 64;
std::mutex g_overlap_mu;  // held for a whole call: the events are shared
OverlapRes g_overlap[kMaxOverlapDevices];

int overlap_res(OverlapRes** out) {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return (int)err;
  if (dev < 0 || dev >= kMaxOverlapDevices) return FIS_E_ARG;
  OverlapRes& r = g_overlap[dev];
  if (!r.block_done) {
    if ((err = cudaStreamCreateWithFlags(&r.side, cudaStreamNonBlocking))) return (int)err;
    for (int j = 0; j < 2; ++j) {
      if ((err = cudaEventCreateWithFlags(&r.after_sc[j], cudaEventDisableTiming)))
        return (int)err;
      if ((err = cudaEventCreateWithFlags(&r.after_upd[j], cudaEventDisableTiming)))
        return (int)err;
    }
    if ((err = cudaEventCreateWithFlags(&r.block_done, cudaEventDisableTiming))) return (int)err;
  }
  *out = &r;
  return FIS_OK;
}
}  // namespace

extern "C" {

int fis_advance_overlap(const fis_engine* e, int64_t steps, int32_t group, int32_t rows,
                        int32_t* ring2, float* spikes_out, void* const* events,
                        int32_t n_pairs, int32_t every, void* stream) {
  int rc = fis_check(e);
  if (rc) return rc;
  if (steps < 0 || group < 1 || rows < 0 || !ring2) return FIS_E_ARG;
  if (events && (n_pairs < 0 || every < 1)) return FIS_E_ARG;
  const int32_t B = (rows > 0 && rows < e->batch) ? rows : e->batch;
  const int kmax = e->p.lag < FIS_MAX_BLOCK ? e->p.lag : FIS_MAX_BLOCK;
  const int32_t gmax = group < B ? group : B;
  const size_t elem = e->ring16 ? 2 : 4;
  int32_t* rings[2] = {ring2, reinterpret_cast<int32_t*>(
                                  reinterpret_cast<char*>(ring2) +
                                  (size_t)kmax * gmax * ring_row(e->n) * elem)};
  std::lock_guard<std::mutex> lk(g_overlap_mu);
  OverlapRes* R = nullptr;
  if ((rc = overlap_res(&R))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // Scatters run on the side stream, updates on the caller's stream; group gi
  // uses ring gi & 1, so the scatter of group gi + 1 overlaps the update of
  // group gi.  Scatter gi waits for the update that last drained its ring
  // (group gi - 2), or for the previous block's last update (gi < 2), which
  // finalised the clock and the spike lists the scatter reads.
  if ((rc = (int)cudaEventRecord(R->block_done, st))) return rc;
  int64_t left = steps;
  int64_t launch = 0;
  while (left > 0) {
    const int k = (int)(left < kmax ? left : kmax);
    float* sp = (left == k) ? spikes_out : nullptr;
    int gi = 0;
    for (int32_t g0 = 0; g0 < B; g0 += group, ++gi) {
      const int32_t nb = (B - g0) < group ? (B - g0) : group;
      const bool last = g0 + nb == B;
      int32_t* ring = rings[gi & 1];
      cudaEvent_t dep = gi >= 2 ? R->after_upd[gi & 1] : R->block_done;
      if ((rc = (int)cudaStreamWaitEvent(R->side, dep, 0))) return rc;
      if ((rc = fis_scatter(e, g0, nb, k, ring, R->side))) return rc;
      if ((rc = (int)cudaEventRecord(R->after_sc[gi & 1], R->side))) return rc;
      if ((rc = (int)cudaStreamWaitEvent(st, R->after_sc[gi & 1], 0))) return rc;
      const bool timed = events && (launch % every) == 0 && (launch / every) < n_pairs;
      if ((rc = record_if(timed, events, 2 * (launch / every), st))) return rc;
      if ((rc = fis_update(e, g0, nb, k, ring, sp, last, stream))) return rc;
      if ((rc = record_if(timed, events, 2 * (launch / every) + 1, st))) return rc;
      if ((rc = (int)cudaEventRecord(last ? R->block_done : R->after_upd[gi & 1], st)))
        return rc;
      ++launch;
    }
    left -= k;
  }
  return FIS_OK;
}

int fis_delay_buffer(const fis_engine* e, int32_t b0, int32_t nb, int32_t* scratch,
                     float* out, void* stream) {
  int rc = fis_check(e);
  if (rc) return rc;
  if ((rc = check_range(e, b0, nb))) return rc;
  if (!scratch || !out) return FIS_E_ARG;
  const int R = e->p.buf_len, L = e->p.lag;
  if ((R + 1) * nb + 1 > kMaxLists) return FIS_E_BOUNDS;
  cudaStream_t st = (cudaStream_t)stream;
  // Pending at clock t: spikes of steps t-L .. t-2; step u lands in slot (u+1) % R.
  ScatterArgs A;
  A.b0 = b0;
  A.nb = nb;
  A.nsrc = R;
  A.u_off = -(int64_t)L;
  A.slot_mode = 1;
  A.zero_next = 0;
  A.filter_last = 0;
  A.ring = scratch;
  A.trial_stride = e->n;
  A.half = 0;  // the delay-ring scratch is int32
  const size_t smem = sizeof(int32_t) * (size_t)((R + 1) * nb + 1);
  k_scatter<<<sm_count() * 4, kScatThreads, smem, st>>>(*e, A);
  if ((rc = launch_status())) return rc;
  const int64_t total = (int64_t)nb * R * e->n;
  k_ring_to_f32<<<grid_for(total, 256), 256, 0, st>>>(*e, b0, nb, scratch, out);
  return launch_status();
}

int fis_spikes_f32(const fis_engine* e, int32_t b0, int32_t nb, int64_t step, float* out,
                   void* stream) {
  int rc = fis_check(e);
  if (rc) return rc;
  if ((rc = check_range(e, b0, nb))) return rc;
  if (!out) return FIS_E_ARG;
  const int64_t total = (int64_t)nb * e->n;
  k_spikes_f32<<<grid_for(total, 256), 256, 0, (cudaStream_t)stream>>>(*e, b0, nb, step, out);
  return launch_status();
}

int fis_load_spikes(const fis_engine* e, int32_t b0, int32_t nb, const float* spikes,
                    void* stream) {
  int rc = fis_check(e);
  if (rc) return rc;
  if ((rc = check_range(e, b0, nb))) return rc;
  if (!spikes) return FIS_E_ARG;
  const int Wd = (e->n + kWarp - 1) / kWarp;
  const int64_t threads = (int64_t)nb * Wd * kWarp;
  const int64_t grid = (threads + 255) / 256;
  k_load_spikes<<<(unsigned)grid, 256, 0, (cudaStream_t)stream>>>(*e, b0, nb, spikes);
  return launch_status();
}

int fis_add_rows(const fis_engine* e, int32_t nb, int32_t rows, const int32_t* src,
                 int64_t src_row_stride, int64_t src_trial_stride, int32_t* dst,
                 int64_t dst_row_stride, int64_t dst_trial_stride, void* stream) {
  if (!e || !src || !dst || nb < 1 || rows < 0) return FIS_E_ARG;
  if (rows == 0) return FIS_OK;
  if (src_trial_stride < e->n || dst_trial_stride < e->n ||
      src_row_stride < (int64_t)(nb - 1) * src_trial_stride + e->n ||
      dst_row_stride < (int64_t)(nb - 1) * dst_trial_stride + e->n)
    return FIS_E_BOUNDS;
  const int64_t total = (int64_t)rows * nb * e->n;
  k_add_rows<<<grid_for(total, 256), 256, 0, (cudaStream_t)stream>>>(
      e->n, nb, rows, src, src_row_stride, src_trial_stride, dst, dst_row_stride,
      dst_trial_stride, e->ring16 ? 1 : 0);
  return launch_status();
}

int fis_ring_row(int32_t n) { return n < 1 ? FIS_E_ARG : ring_row(n); }

}  // extern "C"

// ---------------------------------------------------------------------------
// fis_block_noalloc: the block step with the scratch ring inside the library
// ---------------------------------------------------------------------------
//
// Some callers cannot allocate device memory for the scratch ring that
// fis_block takes: a closed-loop controller that steps the brain inside a hard
// real-time budget per control step (a device allocation can synchronize the
// whole GPU and stall for milliseconds), or a host that binds only this C ABI
// from another language and has no device allocator of its own to hand out a
// buffer.  For them the ring is a fixed array in this library:
//
//  * it holds FIS_NOALLOC_RING_INTS int32 (12 MiB): one trial of the
//    138,639-neuron connectome in 20-step blocks; a call that needs more
//    (k_steps * nb * fis_ring_row(n) elements) is refused with FIS_E_BOUNDS;
//  * every GPU that loads this library holds the array until the process
//    exits;
//  * all calls on one device share it, so calls that overlap on the GPU (from
//    other streams or threads) race on it and must not be issued concurrently;
//  * each call clears the part it uses before its scatter, so it never
//    depends on what an earlier, possibly failed, call left there;
//  * the first call on each device looks up the array's device address with
//    that device current; make that first call before any stream capture.

namespace {

__device__ __align__(256) int32_t g_noalloc_ring[FIS_NOALLOC_RING_INTS];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
int32_t* g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_ring on the current device, looked up once per
// device (host code cannot use the symbol itself as a device pointer).
int noalloc_ring(int32_t** out) {
  int dev = -1;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return (int)err;
  if (dev < 0 || dev >= kMaxDevices) return FIS_E_ARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    err = cudaGetSymbolAddress(&p, g_noalloc_ring);
    if (err != cudaSuccess) return (int)err;
    g_noalloc_addr[dev] = static_cast<int32_t*>(p);
  }
  *out = g_noalloc_addr[dev];
  return FIS_OK;
}

}  // namespace

extern "C" int fis_block_noalloc(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps,
                                 float* spikes_out, int32_t last_group, void* stream) {
  int rc = fis_check(e);
  if (rc) return rc;
  if (nb < 1 || k_steps < 1) return FIS_E_BOUNDS;
  const int64_t elems = (int64_t)k_steps * nb * ring_row(e->n);
  const int64_t need = e->ring16 ? elems / 2 : elems;  // 32-bit words
  if (need > (int64_t)FIS_NOALLOC_RING_INTS) return FIS_E_BOUNDS;
  int32_t* ring = nullptr;
  if ((rc = noalloc_ring(&ring))) return rc;
  if (e->ring16) {
    k_fill32<<<grid_for(need, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<uint32_t*>(ring), need, kEmptyPair);
    rc = launch_status();
  } else {
    rc = (int)cudaMemsetAsync(ring, 0, sizeof(int32_t) * (size_t)need, (cudaStream_t)stream);
  }
  if (rc) return rc;
  return fis_block(e, b0, nb, k_steps, ring, spikes_out, last_group, stream);
}
