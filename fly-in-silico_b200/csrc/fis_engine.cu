// The fused LIF engine for sm_100a.
//
// What one block of K steps (K <= the axonal lag L = buf_len + 1 = 20) does:
//
//   phase A  k_scatter   the spikes of steps t0-L .. t0+K-1-L reach the
//                        conductance exactly at steps t0 .. t0+K-1 (written
//                        into the reference's ring one step after the spike,
//                        read buf_len steps later; sim.py:887-897).  Their CSR
//                        rows are pushed into a scratch ring of K slots of
//                        integer counts (int32, or two trials' biased int16
//                        counts per word) with integer atomics, a warp per
//                        (spike, chunk of the row).  Integer sums make the
//                        order irrelevant.
//   phase B  k_update    every neuron of every trial advances K steps with
//                        its state in registers, two trials per thread in
//                        packed float pairs: refractory counter and gate,
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
#include <vector>

#include "fis_common.cuh"

namespace fis {
namespace {

constexpr int kUpdThreads = 256;
constexpr int kScatThreads = 256;
constexpr int kScatWarps = kScatThreads / kWarp;
constexpr int kMaxLists = 11264;  // prefix entries in dynamic shared memory (44 KB)

// L2 eviction priorities (createpolicy, sm_80+).  The scratch ring is kept in
// L2 between the scatter that fills it, the update that drains and clears it
// and the next scatter (evict_last); the trial state streams through once
// per block (evict_first), so it does not push the ring out.
__device__ __forceinline__ uint64_t policy_keep() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_stream() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ float ld_hint(const float* a, uint64_t pol) {
  float v;
  asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;\n" : "=f"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_hint(const uint32_t* a, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.L2::cache_hint.u32 %0, [%1], %2;\n" : "=r"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_hint(const uint8_t* a, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.L2::cache_hint.u8 %0, [%1], %2;\n" : "=r"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_hint(float* a, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;\n" ::"l"(a), "f"(v), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void red_hint(uint32_t* a, uint32_t v, uint64_t pol) {
  asm volatile("red.global.add.L2::cache_hint.u32 [%0], %1, %2;\n" ::"l"(a), "r"(v), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void red_hint(int32_t* a, int32_t v, uint64_t pol) {
  asm volatile("red.global.add.L2::cache_hint.s32 [%0], %1, %2;\n" ::"l"(a), "r"(v), "l"(pol)
               : "memory");
}

// Bulk asynchronous shared -> global copy (sm_90+ cp.async.bulk, the TMA
// engine): both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_store(void* gmem, const void* smem, unsigned bytes,
                                           uint64_t pol) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;\n" ::
                   "l"(gmem),
               "r"(sa), "r"(bytes), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
// Wait until the committed bulk copies have read their shared-memory source
// (the CTA may then end; the global writes complete before the grid does).
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
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
                                          uint64_t* bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;\n" ::"r"(smem_addr(smem)),
      "l"(gmem), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
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
  fis_clock clk;      // the block's clock when clk_given, else *E.clock
  int clk_given;
};

// The value that marks an empty pair of biased uint16 ring elements.
constexpr uint32_t kEmptyPair = 0x80008000u;

// Prefix sum of the lengths of the scatter's source lists into pre_sum
// (entries [pre_sum[j], pre_sum[j+1]) of the concatenation are list j, j =
// kk*nb + bl; list kk < nsrc holds step u_first + kk, the one after them the
// list of step u_last); returns the total.  All threads of the CTA call it.
__device__ __forceinline__ int32_t list_prefix(const fis_engine& E, const ScatterArgs& A,
                                               const fis_clock& ck, int64_t u_first,
                                               int64_t u_last, int slot2_last, int nlists,
                                               int32_t* pre_sum) {
  const int B = E.batch;
  const int L = E.p.lag;
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
    // exclusive scan of the per-thread partial sums: within each warp by
    // shuffles, then over the eight warp totals
    __shared__ int32_t wsum[kScatWarps];
    const int ln = threadIdx.x & (kWarp - 1), wp = threadIdx.x / kWarp;
    int32_t inc = acc;
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1) {
      const int32_t x = __shfl_up_sync(0xFFFFFFFFu, inc, off);
      if (ln >= off) inc += x;
    }
    if (ln == kWarp - 1) wsum[wp] = inc;
    __syncthreads();
    int32_t before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kScatWarps; ++w) {
      before += w < wp ? wsum[w] : 0;
      all += wsum[w];
    }
    int32_t run = before + inc - acc;
    for (int j = j0; j < j0 + per && j < nlists; ++j) {
      const int32_t len = pre_sum[j];
      pre_sum[j] = run;
      run += len;
    }
    if (threadIdx.x == 0) pre_sum[nlists] = all;
    __syncthreads();
  }
  return pre_sum[nlists];
}

// The scatter's work for CTA `bid` of `nblk`; `pre_sum` holds (K+1)*nb+1 ints.
__device__ __forceinline__ void scatter_body(const fis_engine& E, const ScatterArgs& A,
                                             const int bid, const int nblk, int32_t* pre_sum) {
  const int n = E.n;
  const int B = E.batch;
  const int L = E.p.lag;
  const fis_clock ck = A.clk_given ? A.clk : *E.clock;
  const uint64_t keep = policy_keep();  // the ring stays in L2 for the update
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
  const int32_t total = list_prefix(E, A, ck, u_first, u_last, slot2_last, nlists, pre_sum);

  // Lists that the following update phase will write start empty.
  if (bid == 0) {
    for (int j = threadIdx.x; j < A.zero_next * A.nb; j += blockDim.x) {
      const int kk = j / A.nb, bl = j - kk * A.nb;
      E.list_len[wrap(ck.slot2 + kk, 2 * L) * B + A.b0 + bl] = 0;
    }
  }

  const int lane = threadIdx.x & (kWarp - 1);
  const int warp = threadIdx.x / kWarp;
  // int32 ring: [slot][trial][trial_stride]; paired int16 ring (half):
  // [slot][pair][trial_stride] 32-bit words, trial 2p in the low half of each
  // word and trial 2p + 1 in the high half.
  const int64_t slot_stride = (int64_t)(A.half ? (A.nb + 1) >> 1 : A.nb) * A.trial_stride;
  for (int32_t w = bid * kScatWarps + warp; w < total; w += nblk * kScatWarps) {
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
    const int64_t row = slot * slot_stride + (int64_t)(A.half ? bl >> 1 : bl) * A.trial_stride;
    int32_t* dst = A.ring + row;
    const int shift = (bl & 1) * 16;  // the trial's half of a paired word
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
              // a signed count added to the low half carries into the high
              // half and back out, leaving it unchanged, while the biased
              // sums stay inside 0 .. 0xFFFF (exact below 2**15)
              red_hint(reinterpret_cast<uint32_t*>(dst) + post,
                       (uint32_t)edge_count(wv[c]) << shift, keep);
            } else {
              red_hint(dst + post, edge_count(wv[c]), keep);
            }
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// phase A': the block's Poisson drive
// ---------------------------------------------------------------------------

// Poisson drive of one block (sim.py:859-861) for trials [b0, b0+nb): draw j
// of neuron i in a trial is word j % 4 of Philox4x32-10 at counter
// (i, j / 4, trial lane) keyed by the trial's seed, and the neuron is kicked at
// step j iff float(word >> 8) * 2**-24 < f32(rate) * f32(DT / 1000).  Each warp
// takes 256 neurons of one trial, lists its driven ones in shared memory and
// spreads their (neuron, four-step quad) draws over its 32 lanes, so the
// Philox work is packed whatever the density of driven neurons.  The kick
// steps of the block go to kicks[b][i] as bits (bit k = step t0 + k), written
// for neurons with a positive rate only: the update reads them only there.
// With the caller's lists of driven neurons (drive_idx / drive_len) a warp
// takes 256 list entries of one trial instead of 256 neurons, so the drive
// reads the rates of the listed neurons only; the draws are the same.
constexpr int kDriveThreads = 256;
constexpr int kDriveSpan = 256;  // neurons per warp task

// kAllLoads: read the span's eight rate words before the first ballot (one
// round trip per task) instead of four at a time.
// The drive's per-warp lists in shared memory (declared once in k_phase_a,
// shared by both forms of the drive): the driven entries of the warp's task
// (offsets in the span), their kick probabilities and their kick bits.
struct DriveSmem {
  uint16_t (*slist)[kDriveSpan];
  float (*sprob)[kDriveSpan];
  uint32_t (*sbits)[kDriveSpan];
};

template <bool kAllLoads>
__device__ __forceinline__ void drive_body(const fis_engine& E, const int b0, const int nb,
                                           const int K, const fis_clock& clk,
                                           const int clk_given, const int bid, const int nblk,
                                           const DriveSmem& sm) {
  uint16_t (*slist)[kDriveSpan] = sm.slist;
  float (*sprob)[kDriveSpan] = sm.sprob;
  uint32_t (*sbits)[kDriveSpan] = sm.sbits;
  const int n = E.n;
  const int lane = threadIdx.x & (kWarp - 1);
  const int w = threadIdx.x / kWarp;
  const fis_clock ck = clk_given ? clk : *E.clock;
  const int64_t t0 = ck.step;
  const int spans = (n + kDriveSpan - 1) / kDriveSpan;
  const uint64_t stream = policy_stream();  // rates are read once per block
  const int64_t tasks = (int64_t)nb * spans;
  const int64_t nw = (int64_t)nblk * (kDriveThreads / kWarp);
  for (int64_t task = (int64_t)bid * (kDriveThreads / kWarp) + w; task < tasks;
       task += nw) {
    const int bl = (int)(task / spans);
    const int i0 = (int)(task - (int64_t)bl * spans) * kDriveSpan;
    const int b = b0 + bl;
    const fis_trial tr = E.trials[b];
    const int ka = (int)max((int64_t)0, min(tr.start - t0, (int64_t)K));
    const int kb = (int)max((int64_t)0, min(tr.end - t0, (int64_t)K));
    if (ka >= kb) continue;  // uniform across the warp
    const float* rates = E.rates + (int64_t)b * n;
    int cnt = 0;
    float pr[kDriveSpan / kWarp];
    if (kAllLoads) {
#pragma unroll
      for (int c = 0; c < kDriveSpan / kWarp; ++c) {
        const int i = i0 + c * kWarp + lane;
        pr[c] = i < n ? ld_hint(rates + i, stream) : 0.f;
      }
    }
#pragma unroll(kAllLoads ? kDriveSpan / kWarp : 4)
    for (int c = 0; c < kDriveSpan / kWarp; ++c) {
      const int i = i0 + c * kWarp + lane;
      const float rate = kAllLoads ? pr[c] : (i < n ? ld_hint(rates + i, stream) : 0.f);
      const float p = i < n ? __fmul_rn(rate, E.p.prob_scale) : 0.f;
      const bool d = p > 0.f;
      const unsigned m = __ballot_sync(0xFFFFFFFFu, d);
      if (d) {
        const int pos = cnt + __popc(m & ((1u << lane) - 1u));
        slist[w][pos] = (uint16_t)(c * kWarp + lane);
        sprob[w][pos] = p;
        sbits[w][pos] = 0u;
      }
      cnt += __popc(m);
    }
    if (cnt == 0) continue;
    __syncwarp();
    const int64_t own0 = t0 - tr.start;  // the trial's own step at k = 0
    const int64_t q0 = (own0 + ka) >> 2;
    const int nq = (int)(((own0 + kb - 1) >> 2) - q0) + 1;
    for (int itq = lane; itq < cnt * nq; itq += kWarp) {
      const int jd = itq / nq, qq = itq - jd * nq;
      const int64_t quad = q0 + qq;
      const Philox4 r4 = philox4((uint32_t)(i0 + slist[w][jd]), (uint32_t)quad,
                                 (uint32_t)((uint64_t)quad >> 32), tr.stream,
                                 (uint32_t)tr.seed, (uint32_t)(tr.seed >> 32));
      const float pj = sprob[w][jd];
      const int kq = (int)(quad * 4 - own0);  // step of word 0
      uint32_t bits = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = kq + q;
        if (k >= ka && k < kb && __fmul_rn((float)(r4.x[q] >> 8), 0x1p-24f) < pj)
          bits |= 1u << k;
      }
      if (bits) atomicOr(&sbits[w][jd], bits);
    }
    __syncwarp();
    uint32_t* kicks = E.kicks + (int64_t)b * n + i0;
    for (int j = lane; j < cnt; j += kWarp) kicks[slist[w][j]] = sbits[w][j];
    __syncwarp();  // the lists are reused by the warp's next task
  }
}
// The drive over the caller's lists of driven neurons (drive_idx /
// drive_len).  A task is kListSpan entries of one running trial's list: all
// of them are usually driven, so a task holds about as many draws as a
// scan task of kDriveSpan neurons holds in a trial where a few percent of
// the neurons are driven, and the draws spread over as many warps.
// Every warp reads the group's trial records and list lengths itself, 32
// trials at a time (one round trip per 32 trials), scans the trials' task
// counts across its lanes and takes tasks gw, gw + W, ... of the group's
// sequence, so no warp spends a round trip on a task that holds nothing.
// Within a task: the entries' neuron indices, then their rates, each as one
// round of loads; then the same draws as drive_body.
__device__ __forceinline__ void drive_list_body(const fis_engine& E, const int b0, const int nb,
                                                const int K, const fis_clock& clk,
                                                const int clk_given, const int bid,
                                                const int nblk, const DriveSmem& sm) {
  constexpr unsigned kAll = 0xFFFFFFFFu;
  constexpr int kListSpan = kWarp;  // entries per task
  constexpr int kPer = kListSpan / kWarp;
  const int n = E.n;
  const int lane = threadIdx.x & (kWarp - 1);
  const int w = threadIdx.x / kWarp;
  const fis_clock ck = clk_given ? clk : *E.clock;
  const int64_t t0 = ck.step;
  const uint64_t stream = policy_stream();
  const int W = nblk * (kDriveThreads / kWarp);      // warps of the drive
  const int gw = bid * (kDriveThreads / kWarp) + w;  // this warp among them
  int acc = 0;  // tasks of the trials before this chunk of 32
  for (int base = 0; base < nb; base += kWarp) {
    const int bl = base + lane;
    int nt = 0, len = 0;
    if (bl < nb) {
      const fis_trial t = E.trials[b0 + bl];
      const int ka = (int)max((int64_t)0, min(t.start - t0, (int64_t)K));
      const int kb = (int)max((int64_t)0, min(t.end - t0, (int64_t)K));
      len = min(max(E.drive_len[b0 + bl], 0), n);
      nt = ka < kb ? (len + kListSpan - 1) / kListSpan : 0;
    }
    int incl = nt;
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1) {
      const int x = __shfl_up_sync(kAll, incl, off);
      if (lane >= off) incl += x;
    }
    const int excl = incl - nt;
    const int total = __shfl_sync(kAll, incl, kWarp - 1);
    // this warp's tasks: t in [acc, acc + total) with t = gw (mod W)
    for (int t = acc + ((gw - acc) % W + W) % W; t < acc + total; t += W) {
      const int local = t - acc;
      const int j = __ffs(__ballot_sync(kAll, excl <= local && local < incl)) - 1;
      const int b = b0 + base + j;
      const int e0 = (local - __shfl_sync(kAll, excl, j)) * kListSpan;
      const int lenj = __shfl_sync(kAll, len, j);
      const fis_trial tr = E.trials[b];  // read above by lane j: from L1
      const int ka = (int)max((int64_t)0, min(tr.start - t0, (int64_t)K));
      const int kb = (int)max((int64_t)0, min(tr.end - t0, (int64_t)K));
      const int32_t* lst = E.drive_idx + (int64_t)b * n;
      const float* rates = E.rates + (int64_t)b * n;
      int ids[kPer];
      float pr[kPer];
#pragma unroll
      for (int c = 0; c < kPer; ++c) {
        const int e = e0 + c * kWarp + lane;
        ids[c] = e < lenj ? lst[e] : -1;
      }
#pragma unroll
      for (int c = 0; c < kPer; ++c)
        pr[c] = (unsigned)ids[c] < (unsigned)n ? ld_hint(rates + ids[c], stream) : 0.f;
      int cnt = 0;
#pragma unroll
      for (int c = 0; c < kPer; ++c) {
        const float p = (unsigned)ids[c] < (unsigned)n ? __fmul_rn(pr[c], E.p.prob_scale) : 0.f;
        const bool d = p > 0.f;
        const unsigned m = __ballot_sync(kAll, d);
        if (d) {
          const int pos = cnt + __popc(m & ((1u << lane) - 1u));
          sm.slist[w][pos] = (uint16_t)(c * kWarp + lane);
          sm.sprob[w][pos] = p;
          sm.sbits[w][pos] = 0u;
        }
        cnt += __popc(m);
      }
      if (cnt == 0) continue;
      __syncwarp();
      const int64_t own0 = t0 - tr.start;  // the trial's own step at k = 0
      const int64_t q0 = (own0 + ka) >> 2;
      const int nq = (int)(((own0 + kb - 1) >> 2) - q0) + 1;
      for (int itq = lane; itq < cnt * nq; itq += kWarp) {
        const int jd = itq / nq, qq = itq - jd * nq;
        const int64_t quad = q0 + qq;
        const Philox4 r4 = philox4((uint32_t)lst[e0 + sm.slist[w][jd]], (uint32_t)quad,
                                   (uint32_t)((uint64_t)quad >> 32), tr.stream,
                                   (uint32_t)tr.seed, (uint32_t)(tr.seed >> 32));
        const float pj = sm.sprob[w][jd];
        const int kq = (int)(quad * 4 - own0);  // step of word 0
        uint32_t bits = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int k = kq + q;
          if (k >= ka && k < kb && __fmul_rn((float)(r4.x[q] >> 8), 0x1p-24f) < pj)
            bits |= 1u << k;
        }
        if (bits) atomicOr(&sm.sbits[w][jd], bits);
      }
      __syncwarp();
      uint32_t* kicks = E.kicks + (int64_t)b * n;
      for (int jj = lane; jj < cnt; jj += kWarp) kicks[lst[e0 + sm.slist[w][jj]]] = sm.sbits[w][jj];
      __syncwarp();  // the lists are reused by the warp's next task
    }
    acc += total;
  }
}

// ---------------------------------------------------------------------------
// phase A, balanced form (scatter_mode 1): a warp per task of up to 32 items
// ---------------------------------------------------------------------------
//
// The same work as scatter_body -- the same lists, filtering and atomics --
// with the memory round trips of a task of work items taken together.  Each
// lane resolves one item (its list by binary search over pre_sum, its entry,
// its row bounds: three round trips for the whole task), and the warp walks the
// concatenation of the items' edges as 16-byte quads, 32 quads per pass and
// kScatUnroll passes' loads in flight per lane before their atomics.  A lane
// finds the item of its quad by a binary search over the lanes' exclusive
// prefix sums of quad counts.  Item ranges start anywhere in the edge array;
// a quad is read from its 16-byte aligned address and only the edges inside
// the item's range are pushed.
constexpr int kScatUnroll = 4;

__device__ __forceinline__ void scatter_body_warp(const fis_engine& E, const ScatterArgs& A,
                                                  const int bid, const int nblk,
                                                  int32_t* pre_sum) {
  const int n = E.n;
  const int B = E.batch;
  const int L = E.p.lag;
  const fis_clock ck = A.clk_given ? A.clk : *E.clock;
  const uint64_t keep = policy_keep();
  const int64_t t0 = ck.step;
  const int64_t u_first = t0 + A.u_off;
  const int64_t u_last = t0 - 1;
  const int slot_last = wrap(ck.slot + L - 1, L);
  const int slot2_last = wrap(ck.slot2 + 2 * L - 1, 2 * L);
  const int t_mod_r = A.slot_mode ? (int)mod_pos(t0, E.p.buf_len) : 0;
  const int kk_last = (int)(u_last - u_first);
  const bool last_is_src = A.filter_last && kk_last >= 0 && kk_last < A.nsrc;
  const bool extra = A.filter_last && !last_is_src && u_last >= 0;
  const int nlists = (A.nsrc + (extra ? 1 : 0)) * A.nb;
  const int32_t total = list_prefix(E, A, ck, u_first, u_last, slot2_last, nlists, pre_sum);
  if (bid == 0) {
    for (int j = threadIdx.x; j < A.zero_next * A.nb; j += blockDim.x) {
      const int kk = j / A.nb, bl = j - kk * A.nb;
      E.list_len[wrap(ck.slot2 + kk, 2 * L) * B + A.b0 + bl] = 0;
    }
  }
  const int lane = threadIdx.x & (kWarp - 1);
  const int warp = threadIdx.x / kWarp;
  const int rows_per_slot = A.half ? (A.nb + 1) >> 1 : A.nb;
  constexpr unsigned kAll = 0xFFFFFFFFu;
  // Items per warp task: about two tasks per warp of the grid, 1 to 32.  A
  // light load (one step of one trial) spreads over many warps as one item
  // each; a heavy one packs 32 items into each task.
  const int tw = nblk * kScatWarps;
  const int per = max(1, min(kWarp, total / (2 * tw)));
  const int32_t tasks = (total + per - 1) / per;
  for (int32_t task = bid * kScatWarps + warp; task < tasks; task += tw) {
    // this lane's work item: quads [q0, q0 + nq) of edges, of which edges
    // [q0*4 + lo, q0*4 + hi) are the item's, pushed into ring row `row`
    const int32_t w = task * per + lane;
    int64_t q0 = 0;
    int nq = 0;
    uint32_t span = 0;  // lo | hi << 2 (lo < 4, hi <= chunk + 3)
    uint32_t row = 0;   // ring row | (upper half of a paired word) << 31
    if (lane < per && w < total) {
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
      uint32_t e = kDeadEntry;
      if (idx < E.list_cap) e = lst[idx];
      const uint32_t pre = entry_pre(e);
      bool live = e != kDeadEntry && pre < (uint32_t)n;
      if (live && A.filter_last && u == u_last) {
        const uint8_t fl = E.flags[(int64_t)b * n + pre];
        if (fl & (FIS_FL_OUT_OFF | FIS_FL_SILENCED)) {
          if (!is_src) lst[idx] = kDeadEntry;
          live = false;
        }
      }
      if (live && is_src) {
        const int64_t r0 = E.row_ptr[pre], r1 = E.row_ptr[pre + 1];
        const int64_t lo_e = r0 + (int64_t)entry_chunk(e) * E.chunk;
        const int64_t hi_e = min(r1, lo_e + (int64_t)E.chunk);
        if (lo_e < hi_e) {
          q0 = lo_e >> 2;
          nq = (int)(((hi_e + 3) >> 2) - q0);
          span = (uint32_t)(lo_e - q0 * 4) | ((uint32_t)(hi_e - q0 * 4) << 2);
          const int slot = A.slot_mode ? wrap(t_mod_r + kk, E.p.buf_len) : kk;
          row = (uint32_t)(slot * rows_per_slot + (A.half ? bl >> 1 : bl)) |
                ((uint32_t)(A.half && (bl & 1)) << 31);
        }
      }
    }
    if (!__any_sync(kAll, nq > 0)) continue;
    int inc = nq;
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1) {
      const int t = __shfl_up_sync(kAll, inc, off);
      if (lane >= off) inc += t;
    }
    const int all = __shfl_sync(kAll, inc, kWarp - 1);
    const int ex = inc - nq;
    for (int j0 = 0; j0 < all; j0 += kWarp * kScatUnroll) {
      uint4 q[kScatUnroll];
      int lo[kScatUnroll], hi[kScatUnroll];
      uint32_t rw[kScatUnroll];
#pragma unroll
      for (int v = 0; v < kScatUnroll; ++v) {
        const int j = j0 + kWarp * v + lane;
        int r = 0;
#pragma unroll
        for (int step = kWarp / 2; step > 0; step >>= 1) {
          const int c = r + step;
          if (__shfl_sync(kAll, ex, c) <= j) r = c;
        }
        const int qi = j - __shfl_sync(kAll, ex, r);
        const int64_t qa = __shfl_sync(kAll, q0, r) + qi;
        const uint32_t sp = __shfl_sync(kAll, span, r);
        rw[v] = __shfl_sync(kAll, row, r);
        lo[v] = (int)(sp & 3u) - 4 * qi;
        hi[v] = j < all ? (int)(sp >> 2) - 4 * qi : 0;  // hi <= 0: nothing to push
        if (hi[v] > 0) q[v] = __ldg(reinterpret_cast<const uint4*>(E.edges) + qa);
      }
#pragma unroll
      for (int v = 0; v < kScatUnroll; ++v) {
        if (hi[v] <= 0) continue;
        const uint32_t wv[4] = {q[v].x, q[v].y, q[v].z, q[v].w};
        const int64_t base = (int64_t)(rw[v] & 0x7FFFFFFFu) * A.trial_stride;
        const int shift = (rw[v] >> 31) ? 16 : 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (c >= lo[v] && c < hi[v]) {
            const int post = edge_post(wv[c]);
            if (post < n) {
              if (A.half)
                red_hint(reinterpret_cast<uint32_t*>(A.ring + base) + post,
                         (uint32_t)edge_count(wv[c]) << shift, keep);
              else
                red_hint(A.ring + base + post, edge_count(wv[c]), keep);
            }
          }
        }
      }
    }
  }
}

// The scatter alone (the delay-ring readout uses it).
__global__ void __launch_bounds__(kScatThreads)
k_scatter(const fis_engine E, const ScatterArgs A) {
  extern __shared__ int32_t pre_sum[];
  if (E.scatter_mode == 1)
    scatter_body_warp(E, A, blockIdx.x, gridDim.x, pre_sum);
  else
    scatter_body(E, A, blockIdx.x, gridDim.x, pre_sum);
}

// Phase A of a block as one grid: CTAs [0, scat) scatter, the rest draw the
// Poisson drive.  Both are latency-bound; in one grid their CTAs share the
// SMs and fill each other's waits, and the block needs one launch less.  It
// runs beside the previous group's update, whose CTAs fill the register
// file: at 32 registers a thread (a few bytes of the Philox draw spill to L1)
// two phase-A CTAs take the room of one update CTA instead of 1.5.
// The balanced scatter (kMode 1) keeps four passes of quads in flight and is
// held to 48 registers a thread instead (five CTAs in the room of four
// update CTAs); it needs fewer CTAs for the same work.
static_assert(kScatThreads == kDriveThreads, "one block size for both roles");
template <int kMode>
__global__ void __launch_bounds__(kScatThreads, kMode ? 5 : 7)
k_phase_a(const fis_engine E, const ScatterArgs A, const int scat) {
  extern __shared__ int32_t pre_sum[];
  if ((int)blockIdx.x < scat) {
    if (kMode == 1)
      scatter_body_warp(E, A, blockIdx.x, scat, pre_sum);
    else
      scatter_body(E, A, blockIdx.x, scat, pre_sum);
  } else {
    __shared__ uint16_t slist[kDriveThreads / kWarp][kDriveSpan];
    __shared__ float sprob[kDriveThreads / kWarp][kDriveSpan];
    __shared__ uint32_t sbits[kDriveThreads / kWarp][kDriveSpan];
    const DriveSmem sm{slist, sprob, sbits};
    if (E.drive_idx)
      drive_list_body(E, A.b0, A.nb, A.nsrc, A.clk, A.clk_given, blockIdx.x - scat,
                      gridDim.x - scat, sm);
    else
      drive_body<kMode == 1>(E, A.b0, A.nb, A.nsrc, A.clk, A.clk_given, blockIdx.x - scat,
                             gridDim.x - scat, sm);
  }
}

// ---------------------------------------------------------------------------
// phase B: K fused steps per neuron, two trials per thread
// ---------------------------------------------------------------------------

// Packed float pairs.  sm_100 executes add/sub/mul/fma on .f32x2 operands:
// two independent IEEE binary32 operations per instruction, each lane rounded
// to nearest even with subnormals kept -- the same bits as two __f*_rn calls,
// for half the issue slots.  Lane 0 (low word) is trial A of the thread's
// pair, lane 1 trial B.
//
// One caution: the code generator contracts a .f32x2 multiply into the
// .f32x2 add or subtract that consumes it (one rounding instead of two), even
// with explicit .rn and with contraction disabled -- measured on B200 with
// CUDA 12.9, about half of all random operands then differ in the last bit.
// So a product is never added with add/sub here: addp/subp add it with an FMA
// by a unit factor known only at run time, p * 1 + c, which is exactly the
// rounded sum p + c (p * 1 is exact, signed zeros included), and which the
// code generator cannot fold back into the multiply.
typedef unsigned long long f2;

__device__ __forceinline__ f2 pk2(float a, float b) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void up2(f2 x, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x));
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// The state of one neuron in the thread's two trials, and the per-trial
// constants its flags select.
struct Pair {
  f2 v, g, r;        // membrane, conductance, refractory counter
  f2 keep;           // 1 - spike of the previous step
  f2 m_hold, v_hold;
  float rs0, rs1;    // refractory steps (0 for driven neurons)
  float vth0, vth1;  // threshold; +inf under the fire mask (see lif_step2)
};

// The model constants as pairs (both lanes equal).  `one`/`mone` are +-1
// built from a kernel argument (see addp).
struct Consts {
  f2 one, mone, w, a_syn, a_mem, v_rest, v_reset;
};

// c + p and c - p for a product p, each rounded once as a plain add.
__device__ __forceinline__ f2 addp(const Consts& C, f2 p, f2 c) { return fma2(p, C.one, c); }
__device__ __forceinline__ f2 subp(const Consts& C, f2 c, f2 p) { return fma2(p, C.mone, c); }

// One step of sim.py:921-952 for the neuron in both trials, the reference's
// operation order one rounding at a time.  f0/f1: the spikes; sp: them as
// floats.
//
// c0/c1 are the step's delayed input counts, already zero where the input
// mask m_in is 0 (and for a silenced neuron, which has no incoming synapses,
// sim.py:324-336).  The reference forms (w * count) * m_in * gate and adds it
// to g * a_syn; here the refractory gate and m_in select the count itself
// and w * count is added.  Where both factors are 1 the products are the
// same bits; where one is 0 the reference adds a signed zero and this adds
// +0, which can change only the sign of a zero sum -- and the conductance
// reset below, gn - gn * spike, turns either zero into +0.  So the stored
// state is the same bits, for two multiplies fewer per step.
//
// kStim: add the step's external drive `vstim`.  kHold: apply the hold.  For
// a warp with no driven and no held lane both are identities once v is not
// -0 (v + 0 and v * 1 + 0 leave any other v unchanged), and v never becomes
// -0 inside the loop: x + y is -0 only when both are -0, so neither the
// membrane update v + p nor the reset v - d * spike (d = v - v_reset, x - x
// = +0) turns a v that is not -0 into -0.  The loop adds +0 once before its
// first step (the reference's own v + 0) and then leaves both out.
template <bool kStim = true, bool kHold = true>
__device__ __forceinline__ void lif_step2(Pair& s, const Consts& C, int32_t c0, int32_t c1,
                                          f2 vstim, bool& f0, bool& f1, f2& sp) {
  // refractory counter and gate (sim.py:921-923); r is the previous step's
  // product, so its increment is an addp
  s.r = mul2(addp(C, s.r, C.one), s.keep);
  float r0, r1;
  up2(s.r, r0, r1);
  const int32_t g0 = r0 >= s.rs0 ? c0 : 0, g1 = r1 >= s.rs1 ? c1 : 0;
  // delayed input and the new conductance (sim.py:928-929)
  const f2 delayed = mul2(C.w, pk2(__int2float_rn(g0), __int2float_rn(g1)));
  const f2 gn = addp(C, mul2(s.g, C.a_syn), delayed);
  // membrane with the previous conductance (sim.py:936-938)
  f2 v = kStim ? add2(s.v, vstim) : s.v;
  v = addp(C, mul2(C.a_mem, sub2(s.g, sub2(v, C.v_rest))), v);
  // hold, threshold, reset (sim.py:943-952).  spikes = (v > v_th) * m_fire
  // with m_fire in {0, 1} is +0 or 1; comparing against +inf where m_fire is
  // 0 gives the same bits (a finite v never exceeds +inf) without the multiply.
  if (kHold) v = addp(C, mul2(v, s.m_hold), s.v_hold);
  float v0, v1;
  up2(v, v0, v1);
  f0 = v0 > s.vth0;
  f1 = v1 > s.vth1;
  sp = pk2(f0 ? 1.f : 0.f, f1 ? 1.f : 0.f);
  s.v = subp(C, v, mul2(sub2(v, C.v_reset), sp));
  s.g = subp(C, gn, mul2(gn, sp));
  s.keep = sub2(C.one, sp);  // 1 - 0 = 1, 1 - 1 = +0: the bits of the select
}

// The staged input of step k for this thread.  kHalf: one word of the paired
// ring, trial A's biased count in the low half and trial B's in the high
// half; flipping each half's top bit turns 0x8000 + c into c as an int16.
// Otherwise two int32 columns, one per trial.  `mask` zeroes the counts of a
// silenced neuron and of one whose input mask is off, per trial.
struct Staged2 {
  const int32_t* col;  // this thread's word of slot 0 (kHalf) or of trial A's row
  uint32_t mask0, mask1;
};

// 32-bit words of one staged slot: a pair row (kHalf) or two trial rows
template <bool kHalf>
struct StagedRow {
  static constexpr int kWords = kHalf ? kTile : 2 * kTile;
};

template <bool kHalf>
__device__ __forceinline__ void staged2(const Staged2& s, int k, int32_t& c0, int32_t& c1) {
  if (kHalf) {
    const uint32_t w = ((uint32_t)s.col[k * kTile] ^ kEmptyPair) & (s.mask0 | s.mask1);
    c0 = (int32_t)(int16_t)(w & 0xFFFFu);
    c1 = (int32_t)w >> 16;
  } else {
    c0 = (int32_t)((uint32_t)s.col[k * 2 * kTile] & s.mask0);
    c1 = (int32_t)((uint32_t)s.col[k * 2 * kTile + kTile] & s.mask1);
  }
}

// The step loop over K steps.  `kDrive` selects whether any lane of the warp
// is driven in either trial, so warps without drive carry no drive logic.
// `kPartial`: a trial starts or ends inside this block (or only one of the
// two runs), so each step commits only the lanes whose trial runs at that
// step.  `kRaster`: store every step's raster words (else the caller keeps
// only the last step's).  Returns the fired steps of each trial as bits, the
// last step in bit 0 (exact in float).
template <bool kTape, bool kDrive, bool kHalf, bool kPartial, bool kRaster = true,
          bool kHold = true>
__device__ __forceinline__ f2 step_loop2(Pair& st, const Consts& C, const fis_engine& E, int K,
                                         int ka0, int kb0, int ka1, int kb1, uint32_t dm0,
                                         uint32_t dm1, const Staged2& in, uint32_t* sbal0,
                                         uint32_t* sbal1, int64_t sidx0, int64_t sidx1,
                                         bool valid) {
  const float kick = E.p.kick;
  // fired steps as bits: m = 2 m + spike per step, an exact float of at most
  // 20 bits (bookkeeping, not model state, so the fused multiply-add is fine)
  f2 nspk = pk2(0.f, 0.f);
  const f2 two = pk2(2.f, 2.f);
  // no external drive in this warp: its per-step v + 0 is done once here
  constexpr bool kStim = kTape || kDrive || kPartial;
  if (!kStim) st.v = add2(st.v, pk2(0.f, 0.f));
  // Lanes past the last neuron run the same arithmetic on inert values (never
  // above an infinite threshold) and store nothing.  Every lane stores the
  // warp's ballot word (the same value to the same address), so the store
  // needs no lane predicate.
#pragma unroll(kPartial ? 1 : 2)
  for (int k = 0; k < K; ++k) {
    int32_t c0, c1;
    staged2<kHalf>(in, k, c0, c1);
    f2 vstim = pk2(0.f, 0.f);
    if (kTape) {
      vstim = pk2(valid ? E.vstim[sidx0] : 0.f, valid ? E.vstim[sidx1] : 0.f);
    } else if (kDrive) {
      vstim = pk2(((dm0 >> k) & 1u) ? kick : 0.f, ((dm1 >> k) & 1u) ? kick : 0.f);
    }
    bool f0, f1;
    f2 sp;
    if (kPartial) {
      const Pair old = st;
      lif_step2(st, C, c0, c1, vstim, f0, f1, sp);
      const bool a0 = k >= ka0 && k < kb0, a1 = k >= ka1 && k < kb1;
      float x0, x1, y0, y1;
#define FIS_KEEP_LANES(field)              \
  up2(st.field, x0, x1);                   \
  up2(old.field, y0, y1);                  \
  st.field = pk2(a0 ? x0 : y0, a1 ? x1 : y1);
      FIS_KEEP_LANES(v)
      FIS_KEEP_LANES(g)
      FIS_KEEP_LANES(r)
      FIS_KEEP_LANES(keep)
#undef FIS_KEEP_LANES
      f0 = f0 && a0;
      f1 = f1 && a1;
      sp = pk2(f0 ? 1.f : 0.f, f1 ? 1.f : 0.f);
    } else {
      lif_step2<kStim, kHold || kPartial>(st, C, c0, c1, vstim, f0, f1, sp);
    }
    if (kRaster) {
      sbal0[k] = __ballot_sync(0xFFFFFFFFu, f0);
      sbal1[k] = __ballot_sync(0xFFFFFFFFu, f1);
    }
    nspk = fma2(nspk, two, sp);
  }
  return nspk;
}

// Grid: one CTA per (pair of trials of the group, tile of 256 neurons).  The
// scratch ring's rows are padded to ring_row(n), so a tile's slice of a slot
// is one aligned 1 KB line of the async bulk copy engine: one line per slot
// of the paired int16 ring, one per trial and slot of the int32 ring.
// Everything the CTA reads is requested at entry -- the staged input (bulk
// copies), the clock and trial records, the neuron state -- so their
// latencies overlap each other and the drive computation.
// Warp 0 of a CTA: stage the K slots of `tile` for trial pair `pp` into
// `srow` with bulk copies (TMA) completing on `bar`, which it sets up.
template <bool kHalf>
__device__ __forceinline__ void stage_tile(const fis_engine& E, const int32_t* ring,
                                           const int nb, const int K, const int pp,
                                           const int tile,
                                           int32_t (*srow)[StagedRow<kHalf>::kWords],
                                           uint64_t* bar) {
  const int NR = ring_row(E.n);
  const int nt = (2 * pp + 1 < nb) ? 2 : 1;
  const int np = (nb + 1) >> 1;
  const int64_t sstride = kHalf ? (int64_t)np * NR * 2 : (int64_t)nb * NR;
  const int64_t toff = kHalf ? ((int64_t)pp * NR + tile * kTile) * 2
                             : (int64_t)(2 * pp) * NR + tile * kTile;
  const int copies = kHalf ? K : K * nt;
  const uint64_t keep = policy_keep();
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(bar, (unsigned)copies * kTile * 4u);
  }
  __syncwarp();
  if (!E.inject_stall) {
    for (int c = threadIdx.x; c < copies; c += kWarp) {
      const int k = kHalf ? c : c / nt, t = kHalf ? 0 : c - k * nt;
      const int64_t off = (int64_t)k * sstride + toff + (int64_t)t * NR;
      const void* src = kHalf ? (const void*)(reinterpret_cast<const uint16_t*>(ring) + off)
                              : (const void*)(ring + off);
      bulk_load(&srow[k][t * kTile], src, kTile * 4u, bar, keep);
    }
  }
}

// Four-byte async copy global -> shared (sm_80+), and the wait for all of this
// thread's outstanding ones.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, uint64_t pol) {
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %2;\n" ::"r"(
                   smem_addr(smem)),
               "l"(gmem), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// What the prologue of an update kernel gathers for one thread's neuron in
// the two trials of its pair, for tile_compute.
struct TileState {
  float v[2], g[2], r[2], vclamp[2];
  uint32_t fl[2], dm[2];  // flags; kick steps (bit k = step k)
  int ka[2], kb[2];       // the trial's steps of this block: [ka, kb)
  bool runs[2];           // the trial runs in this block (uniform in the CTA)
  bool s_prev[2];         // the neuron fired at the step before the block
};

// The K steps of one tile for both trials of pair `pp` and the epilogue:
// state stores, raster words, spike lists and recording bins.  `srow`: the
// staged slots (the step loop's input); `sbal`: the raster words of the
// warp's steps.
template <bool kTape, bool kHalf>
__device__ __forceinline__ void tile_compute(
    const fis_engine& E, const int b0, const int K, float* __restrict__ spikes_out,
    const float unit, const fis_clock& ck, const int tile, const int pp,
    int32_t (*srow)[StagedRow<kHalf>::kWords],
    uint32_t (*sbal)[kUpdThreads / kWarp][FIS_MAX_BLOCK], const TileState& S,
    const bool warp_driven, const int64_t (&sidx)[2]) {
  const int n = E.n;
  const int L = E.p.lag;
  const int Wd = (n + kWarp - 1) / kWarp;
  const int i = tile * kTile + threadIdx.x;
  const int lane = threadIdx.x & (kWarp - 1);
  const int wib = threadIdx.x / kWarp;
  const bool valid = i < n;
  const bool warp_valid = (i - lane) < n;
  const int64_t t0 = ck.step;
  const int slot0 = ck.slot;
  const uint64_t stream = policy_stream();
  Pair st;
  float vth[2], rs[2], mhold[2], vhold[2];
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const bool on = S.runs[t] && valid && !(S.fl[t] & FIS_FL_FIRE_OFF);
    vth[t] = on ? E.p.v_th : __int_as_float(0x7f800000);
    rs[t] = (S.fl[t] & FIS_FL_NOREFRAC) ? 0.f : E.p.refrac_steps;
    const bool hold = S.fl[t] & FIS_FL_HOLD;
    mhold[t] = hold ? 0.f : 1.f;
    vhold[t] = hold ? S.vclamp[t] : 0.f;
  }
  st.v = pk2(S.v[0], S.v[1]);
  st.g = pk2(S.g[0], S.g[1]);
  st.r = pk2(S.r[0], S.r[1]);
  st.keep = pk2(S.s_prev[0] ? 0.f : 1.f, S.s_prev[1] ? 0.f : 1.f);
  st.m_hold = pk2(mhold[0], mhold[1]);
  st.v_hold = pk2(vhold[0], vhold[1]);
  st.rs0 = rs[0];
  st.rs1 = rs[1];
  st.vth0 = vth[0];
  st.vth1 = vth[1];
  Consts C;
  C.one = pk2(unit, unit);
  C.mone = pk2(-unit, -unit);
  C.w = pk2(E.p.w_scale, E.p.w_scale);
  C.a_syn = pk2(E.p.a_syn, E.p.a_syn);
  C.a_mem = pk2(E.p.a_mem, E.p.a_mem);
  C.v_rest = pk2(E.p.v_rest, E.p.v_rest);
  C.v_reset = pk2(E.p.v_reset, E.p.v_reset);

  // Every lane of a warp runs the same step loop (the choice depends on the
  // trials and on the warp's vote only), so every lane reaches each ballot.
  Staged2 in;
  in.col = &srow[0][threadIdx.x];
  in.mask0 = (S.fl[0] & (FIS_FL_SILENCED | FIS_FL_IN_OFF)) ? 0u : (kHalf ? 0x0000FFFFu : 0xFFFFFFFFu);
  in.mask1 = (S.fl[1] & (FIS_FL_SILENCED | FIS_FL_IN_OFF)) ? 0u : (kHalf ? 0xFFFF0000u : 0xFFFFFFFFu);
  // A trial slot that does not run is inert in the lanes it shares (never
  // fires, never stored), so only a trial that starts or ends inside the
  // block needs the per-step commit of the partial loop.
  const bool full = (!S.runs[0] || (S.ka[0] == 0 && S.kb[0] == K)) &&
                    (!S.runs[1] || (S.ka[1] == 0 && S.kb[1] == K));
  const bool hold_any = __any_sync(0xFFFFFFFFu, ((S.fl[0] | S.fl[1]) & FIS_FL_HOLD) != 0);
  const int ka0 = S.runs[0] ? S.ka[0] : 0, kb0 = S.runs[0] ? S.kb[0] : 0;
  const int ka1 = S.runs[1] ? S.ka[1] : 0, kb1 = S.runs[1] ? S.kb[1] : 0;
  uint32_t* sb0 = sbal[0][wib];
  uint32_t* sb1 = sbal[1][wib];
  f2 nspk;
  if (kTape)
    nspk = step_loop2<true, false, kHalf, true>(st, C, E, K, ka0, kb0, ka1, kb1, 0u, 0u, in, sb0,
                                               sb1, sidx[0], sidx[1], valid);
  else if (!full)
    nspk = step_loop2<false, true, kHalf, true>(st, C, E, K, ka0, kb0, ka1, kb1, S.dm[0], S.dm[1],
                                               in, sb0, sb1, sidx[0], sidx[1], valid);
  else if (E.raster && warp_driven)
    nspk = step_loop2<false, true, kHalf, false>(st, C, E, K, 0, K, 0, K, S.dm[0], S.dm[1], in,
                                                sb0, sb1, sidx[0], sidx[1], valid);
  else if (E.raster)
    nspk = step_loop2<false, false, kHalf, false>(st, C, E, K, 0, K, 0, K, 0u, 0u, in, sb0, sb1,
                                                 sidx[0], sidx[1], valid);
  else if (hold_any && warp_driven)
    nspk = step_loop2<false, true, kHalf, false, false>(st, C, E, K, 0, K, 0, K, S.dm[0],
                                                       S.dm[1], in, sb0, sb1, sidx[0], sidx[1],
                                                       valid);
  else if (hold_any)
    nspk = step_loop2<false, false, kHalf, false, false>(st, C, E, K, 0, K, 0, K, 0u, 0u, in,
                                                        sb0, sb1, sidx[0], sidx[1], valid);
  else if (warp_driven)  // no held lane: the hold is left out (see lif_step2)
    nspk = step_loop2<false, true, kHalf, false, false, false>(
        st, C, E, K, 0, K, 0, K, S.dm[0], S.dm[1], in, sb0, sb1, sidx[0], sidx[1], valid);
  else
    nspk = step_loop2<false, false, kHalf, false, false, false>(
        st, C, E, K, 0, K, 0, K, 0u, 0u, in, sb0, sb1, sidx[0], sidx[1], valid);
  // Without the full raster only the last step's words are kept (the next
  // block reads them for the refractory reset); the partial and tape loops
  // always store every step.
  // The last step's words are the warp's ballots of keep == 0, which every
  // lane holds: lane 0 stores them directly.
  const bool only_last = !E.raster && full && !kTape;
  if (only_last) {
    float k0, k1;
    up2(st.keep, k0, k1);
    const uint32_t w0 = __ballot_sync(0xFFFFFFFFu, k0 == 0.f);
    const uint32_t w1 = __ballot_sync(0xFFFFFFFFu, k1 == 0.f);
    if (lane == 0 && warp_valid) {
      const int sl = slot0 + K - 1 < L ? slot0 + K - 1 : slot0 + K - 1 - L;
      const int64_t wrow = (int64_t)(b0 + 2 * pp) * Wd + (i >> 5);
      if (S.runs[0]) E.bits[wrow * L + sl] = w0;
      if (S.runs[1]) E.bits[(wrow + Wd) * L + sl] = w1;
    }
  } else {
    __syncwarp();
  }

  float ov[2], og[2], orr[2], okeep[2], ospk[2];
  up2(st.v, ov[0], ov[1]);
  up2(st.g, og[0], og[1]);
  up2(st.r, orr[0], orr[1]);
  up2(st.keep, okeep[0], okeep[1]);
  up2(nspk, ospk[0], ospk[1]);
  // Addresses and trial fields are derived again here rather than kept live
  // through the step loop (its register budget); the spike path reloads
  // what it needs from L1.
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    if (!S.runs[t]) continue;
    const int b = b0 + 2 * pp + t;
    const int64_t si = (int64_t)b * n + i;
    // the raster words of the K steps into the ring of the last L steps
    if (!only_last && lane < K && warp_valid) {
      const int sl = slot0 + lane < L ? slot0 + lane : slot0 + lane - L;
      E.bits[((int64_t)b * Wd + (i >> 5)) * L + sl] = sbal[t][wib][lane];
    }
    if (valid) {
      st_hint(E.v + si, ov[t], stream);
      st_hint(E.g + si, og[t], stream);
      st_hint(E.refrac + si, orr[t], stream);
      if (spikes_out) spikes_out[si] = (okeep[t] == 0.f) ? 1.f : 0.f;
    }
    // Spike lists and recording for the (rare) steps this neuron fired.
    uint32_t fired = (uint32_t)ospk[t];  // bit j is step K-1-j
    if (fired) {
      const int B = E.batch;
      const fis_trial trl = E.trials[b];
      const uint32_t flb = E.flags[si];
      const int nch = (int)E.nchunks[i];
      int32_t* const recb = (trl.rec >= 0 && trl.rec < E.n_recs) ? E.recs[trl.rec] : nullptr;
      const bool out_on = !(flb & (FIS_FL_OUT_OFF | FIS_FL_SILENCED));
      const int slot20 = ck.slot2;
      const int64_t own0 = t0 - trl.start;
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
        if (recb && trl.bin_steps > 0) {
          const int64_t own = own0 + k;
          const int64_t bin = own < 0x7FFFFFFF ? (int64_t)((int)own / trl.bin_steps)
                                                : own / trl.bin_steps;
          if (bin < trl.n_bins) red_hint(recb + bin * n + i, 1, stream);
        }
      }
    }
  }
}

// One tile's update: everything but the issue of its staging copies (warp 0
// of the CTA has issued them into `srow`, completing on `bar`) and the clock
// bump.  `count`: this CTA counts itself in for the clock bump (into
// *arrived) after the staging barrier.
template <bool kTape, bool kHalf>
__device__ __forceinline__ void update_tile(
    const fis_engine& E, const int b0, const int nb, const int K, int32_t* __restrict__ ring,
    float* __restrict__ spikes_out, const float unit, const fis_clock& ck, const int tile,
    int32_t (*srow)[StagedRow<kHalf>::kWords], uint64_t* bar, uint32_t* szero,
    uint32_t (*sbal)[kUpdThreads / kWarp][FIS_MAX_BLOCK], const bool count, unsigned* arrived) {
  const int n = E.n;
  const int L = E.p.lag;
  const int Wd = (n + kWarp - 1) / kWarp;
  const int NR = ring_row(n);
  const int pp = blockIdx.y;    // pair of trials of the group: 2 pp, 2 pp + 1
  const int i = tile * kTile + threadIdx.x;
  const int lane = threadIdx.x & (kWarp - 1);
  const bool valid = i < n;
  const bool warp_valid = (i - lane) < n;
  const int nt = (2 * pp + 1 < nb) ? 2 : 1;  // trials in this pair
  const int np = (nb + 1) >> 1;              // pairs in the group
  // slot stride and this tile's offset, in ring elements (uint16 or int32)
  const int64_t sstride = kHalf ? (int64_t)np * NR * 2 : (int64_t)nb * NR;
  const int64_t toff = kHalf ? ((int64_t)pp * NR + tile * kTile) * 2
                             : (int64_t)(2 * pp) * NR + tile * kTile;
  const int copies = kHalf ? K : K * nt;  // 1 KB lines to stage
  const uint64_t keep = policy_keep();      // the scratch ring
  const uint64_t stream = policy_stream();  // the trial state

  __syncwarp();  // sbal of the previous tile is read before this one writes it

  // Clock, trial records and state, requested before anything depends on
  // them.  A trial slot that does not run in this block is inert: its state
  // is not used, its threshold infinite, nothing of it stored.
  fis_trial tr[2];
  int64_t sidx[2];
  uint32_t fl[2], dm[2], word[2];
  float rate[2], vv[2], gg[2], rr[2];
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int b = b0 + 2 * pp + (t < nt ? t : 0);
    tr[t] = E.trials[b];
    sidx[t] = (int64_t)b * n + i;
    // the warp's raster word of the step before the block: whether it is
    // used depends on the trial record, its address does not, so it is
    // requested now rather than after the record arrives
    word[t] = warp_valid ? E.bits[((int64_t)b * Wd + (i >> 5)) * L +
                                  (ck.slot == 0 ? L - 1 : ck.slot - 1)]
                         : 0u;
    fl[t] = dm[t] = 0;
    rate[t] = vv[t] = gg[t] = rr[t] = 0.f;
    if (valid && t < nt) {
      fl[t] = ld_hint(E.flags + sidx[t], stream);
      vv[t] = ld_hint(E.v + sidx[t], stream);
      gg[t] = ld_hint(E.g + sidx[t], stream);
      rr[t] = ld_hint(E.refrac + sidx[t], stream);
      rate[t] = ld_hint(E.rates + sidx[t], stream);
      if (!kTape && K > 1) dm[t] = ld_hint(E.kicks + sidx[t], stream);
    }
  }
  __syncthreads();  // the staging barrier exists before anyone waits on it
  const int64_t t0 = ck.step;
  int ka[2], kb[2];
  bool runs[2];
  bool s_prev[2];
  bool drv_any = false;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    ka[t] = (int)max((int64_t)0, min(tr[t].start - t0, (int64_t)K));
    kb[t] = (int)max((int64_t)0, min(tr[t].end - t0, (int64_t)K));
    runs[t] = t < nt && ka[t] < kb[t];  // uniform across the CTA
    if (!runs[t]) fl[t] = 0, rate[t] = vv[t] = gg[t] = rr[t] = 0.f;
    // kick steps were computed by phase A for neurons with a positive rate
    // (a one-step block draws its word here: word own % 4 of Philox4x32-10
    // at counter (i, own / 4, trial lane), as the phase-A drive does)
    const float prob = __fmul_rn(rate[t], E.p.prob_scale);
    if (!(runs[t] && prob > 0.f)) {
      dm[t] = 0u;
    } else if (!kTape && K == 1 && valid) {
      const int64_t own = t0 - tr[t].start;
      const uint64_t quad = (uint64_t)(own >> 2);
      const Philox4 r4 = philox4((uint32_t)i, (uint32_t)quad, (uint32_t)(quad >> 32), tr[t].stream,
                                 (uint32_t)tr[t].seed, (uint32_t)(tr[t].seed >> 32));
      const int w = (int)(own & 3);  // selected without indexing (stays in registers)
      const uint32_t x = w & 2 ? (w & 1 ? r4.x[3] : r4.x[2]) : (w & 1 ? r4.x[1] : r4.x[0]);
      dm[t] = __fmul_rn((float)(x >> 8), 0x1p-24f) < prob ? 1u : 0u;
    }
    drv_any = drv_any || (valid && runs[t] && __fmul_rn(rate[t], E.p.prob_scale) > 0.f);
    s_prev[t] = runs[t] && warp_valid && t0 - 1 >= tr[t].start - tr[t].history && t0 >= 1 &&
                ((word[t] >> lane) & 1u);
  }
  const bool warp_driven = !kTape && __any_sync(0xFFFFFFFFu, drv_any);

  // Wait for the staged input.  If any thread's wait runs out, the whole CTA
  // (decided together, so every warp stays whole for its ballots) flags the
  // error for the host, waits once more for copies still writing its shared
  // memory, and skips the update, still reaching the final barrier.
  const unsigned polls = E.wait_polls ? E.wait_polls : kWaitPolls;
  const bool staged_ok = mbar_wait(bar, 0, polls);
  const bool failed = __syncthreads_or(!staged_ok);
  // With `bump` the grid's last CTA advances the clock.  Each CTA counts
  // itself in here, after a barrier that every one of its threads reached
  // with the clock already read, and the CTA whose count completes the grid
  // -- by then every CTA has read the clock -- writes the next clock as it
  // ends; the count's round trip overlaps the rest of the CTA.
  if (count && threadIdx.x == 0) *arrived = atomicAdd(E.done, 1u) + 1u;
  if (failed) {
    // The staged lines were neither consumed nor returned to empty: the
    // host must refill the ring before it is used again.  A second wait
    // that also runs out leaves copies that may still write this CTA's
    // shared memory after it ends: FIS_ERR_STAGE_LOST, fatal for the context.
    if (threadIdx.x == 0) atomicOr(E.done + 1, (uint32_t)FIS_ERR_STAGE);
    if (!staged_ok && !mbar_wait(bar, 0, polls))
      atomicOr(E.done + 1, (uint32_t)FIS_ERR_STAGE_LOST);
  } else {
  // The staged lines are in shared memory: warp 0 returns them to empty in
  // the ring with one bulk store each, so the scratch ring needs no clearing
  // pass and the step loop no stores.  Trials that do not run in this block
  // are cleared too: scatters of their last spikes may have landed there.
  if (threadIdx.x < kWarp) {
    const uint32_t empty = kHalf ? kEmptyPair : 0u;
#pragma unroll
    for (int j = 0; j < kTile / kWarp; ++j) szero[j * kWarp + threadIdx.x] = empty;
    fence_proxy_async_shared();
    __syncwarp();
    for (int c = threadIdx.x; c < copies; c += kWarp) {
      const int k = kHalf ? c : c / nt, t = kHalf ? 0 : c - k * nt;
      const int64_t off = (int64_t)k * sstride + toff + (int64_t)t * NR;
      if (kHalf) bulk_store(reinterpret_cast<uint16_t*>(ring) + off, szero, kTile * 4u, keep);
      else bulk_store(ring + off, szero, kTile * 4u, keep);
    }
    bulk_commit();
  }

  if (runs[0] || runs[1]) {
    TileState S;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      S.v[t] = vv[t];
      S.g[t] = gg[t];
      S.r[t] = rr[t];
      S.vclamp[t] = tr[t].v_clamp;
      S.fl[t] = fl[t];
      S.dm[t] = dm[t];
      S.ka[t] = ka[t];
      S.kb[t] = kb[t];
      S.runs[t] = runs[t];
      S.s_prev[t] = s_prev[t];
    }
    tile_compute<kTape, kHalf>(E, b0, K, spikes_out, unit, ck, tile, pp, srow, sbal, S,
                               warp_driven, sidx);
  }

  // The clearing copies have read szero before the CTA ends (it must stay
  // valid while they read it); their writes into the ring are complete when
  // the grid is, before the next scatter, a later kernel, adds into them.
  if (threadIdx.x < kWarp) bulk_wait_all();
  }  // the staged input arrived
}

// The grid's last CTA to count itself in writes the next clock.
__device__ __forceinline__ void clock_bump(const fis_engine& E, const int bump,
                                           const unsigned arrived, const fis_clock& ck,
                                           const int K) {
  if (bump && threadIdx.x == 0 && arrived == gridDim.x * gridDim.y) {
    const int L = E.p.lag;
    *E.done = 0u;
    fis_clock next;
    next.step = ck.step + K;
    next.slot = wrap(ck.slot + K, L);
    next.slot2 = wrap(ck.slot2 + K, 2 * L);
    *E.clock = next;
  }
}

// One tile per CTA: grid (tiles, trial pairs).
template <bool kTape, bool kHalf>
__global__ void __launch_bounds__(kUpdThreads, 4)
k_update(const fis_engine E, const int b0, const int nb, const int K,
         int32_t* __restrict__ ring, float* __restrict__ spikes_out,
         const int bump, const float unit,  // unit: 1.0f (see addp)
         const fis_clock clk, const int clk_given) {
  // The block's delayed input, a column per thread (per trial for int32):
  // staged so the step loop stays rolled (a compact body that fits the
  // instruction cache) and can index it by step.
  __shared__ __align__(128) int32_t sring[FIS_MAX_BLOCK][StagedRow<kHalf>::kWords];
  __shared__ __align__(16) uint32_t szero[kTile];                  // source of the clearing
  __shared__ uint32_t sbal[2][kUpdThreads / kWarp][FIS_MAX_BLOCK]; // raster words per step
  __shared__ __align__(8) uint64_t sbar;                           // staging barrier
  if (threadIdx.x < kWarp) stage_tile<kHalf>(E, ring, nb, K, blockIdx.y, blockIdx.x, sring, &sbar);
  const fis_clock ck = clk_given ? clk : *E.clock;  // the block's clock
  unsigned arrived = 0;
  update_tile<kTape, kHalf>(E, b0, nb, K, ring, spikes_out, unit, ck, blockIdx.x, sring, &sbar,
                            szero, sbal, bump != 0, &arrived);
  clock_bump(E, bump, arrived, ck, K);
}

// Streamed tiles (paired int16 ring, Philox drive, blocks of 2+ steps): each
// CTA takes a near-equal run of consecutive items (trial pair, tile),
// pair-major, and pipelines them.  While item j's steps run, item j+1's input
// is already on its way: its slots into the second of two ring buffers, its
// trial records and raster words into the second of two small buffers, its
// state (v, g, refrac, rates, kicks and flags of both trials) into the one
// state buffer.  So only a CTA's first item waits for its input.
//
// No CTA-wide barrier: warps meet only through mbarriers, so a warp that
// finishes an item early starts the next one.  `full[s]` completes when
// stage s holds its item (bulk copies, TMA, counted in bytes, plus the 4-byte
// async copies of the raster words).  `taken` completes when all 8 warps
// have taken item j's state into registers -- and so have finished item
// j-1, whose buffers may then be refilled.  Warp 0 waits for it and issues
// item j+1's copies; the other warps never wait for warp 0.
//
// A trial's row of N neurons starts anywhere, so each state row is copied
// from the 16-byte boundary at or below the tile's first neuron: 1040 bytes
// of floats (kStateWords) and 272 of flags (kFlagBytes), read from an offset
// inside.  A trial whose widened rows would reach past the end of the arrays
// (the batch's last tile) is read directly by its threads instead.  The
// arrays and the trial records must start on 16-byte boundaries (checked by
// the host).
struct StreamSmem {
  static constexpr int kStateWords = kTile + 4;
  static constexpr int kFlagBytes = kTile + 16;
  static constexpr int kArrays = 5;  // v, g, refrac, rates, kicks
  static constexpr size_t kRingStage = sizeof(int32_t) * FIS_MAX_BLOCK * kTile;
  static constexpr size_t kState = 2 * kRingStage;
  static constexpr size_t kFlags = kState + sizeof(uint32_t) * 2 * kArrays * kStateWords;
  static constexpr size_t kZero = kFlags + 2 * kFlagBytes;
  static constexpr size_t kBal = kZero + sizeof(uint32_t) * kTile;
  static constexpr size_t kPrev = kBal + sizeof(uint32_t) * 2 * (kUpdThreads / kWarp) * FIS_MAX_BLOCK;
  static constexpr size_t kTrials = kPrev + sizeof(uint32_t) * 2 * 2 * (kUpdThreads / kWarp);
  static constexpr size_t kBar = kTrials + sizeof(fis_trial) * 2 * 2;
  static constexpr size_t kClock = kBar + sizeof(uint64_t) * 3;  // full[2], taken
  static constexpr size_t kAbort = kClock + sizeof(fis_clock);
  static constexpr size_t kBytes = kAbort + 16;
};
static_assert(StreamSmem::kFlags % 16 == 0 && StreamSmem::kZero % 16 == 0 &&
                  StreamSmem::kTrials % 16 == 0 && sizeof(fis_trial) % 16 == 0 &&
                  StreamSmem::kBar % 8 == 0 && StreamSmem::kClock % 8 == 0,
              "bulk copy destinations on 16-byte boundaries, barriers on 8");

// Where item `item` of the group lies.  first[t]: element index of the
// tile's first neuron in trial t's row of the [B][N] arrays; ofs/ofb: floats
// and flag bytes from the 16-byte boundary below it; direct: read by the
// threads, not staged (also for a trial slot the pair does not have).
struct ItemGeo {
  int pp, tile, nt;
  int64_t first[2];
  int ofs[2], ofb[2];
  bool direct[2];
};

__device__ __forceinline__ ItemGeo item_geo(const fis_engine& E, const int b0, const int nb,
                                            const int ntiles, const int item) {
  ItemGeo G;
  G.pp = item / ntiles;
  G.tile = item - G.pp * ntiles;
  G.nt = (2 * G.pp + 1 < nb) ? 2 : 1;
  const int64_t total = (int64_t)E.batch * E.n;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int64_t f = (int64_t)(b0 + 2 * G.pp + (t < G.nt ? t : 0)) * E.n + G.tile * kTile;
    G.first[t] = f;
    G.ofs[t] = (int)(f & 3);
    G.ofb[t] = (int)(f & 15);
    G.direct[t] = t >= G.nt || f - G.ofs[t] + StreamSmem::kStateWords > total ||
                  f - G.ofb[t] + StreamSmem::kFlagBytes > total;
  }
  return G;
}

__device__ __forceinline__ unsigned item_bytes(const ItemGeo& G, const int K) {
  unsigned b = (unsigned)K * kTile * 4u + (unsigned)G.nt * (unsigned)sizeof(fis_trial);
#pragma unroll
  for (int t = 0; t < 2; ++t)
    if (!G.direct[t])
      b += StreamSmem::kArrays * StreamSmem::kStateWords * 4u + StreamSmem::kFlagBytes;
  return b;
}

// Make `bar`'s current phase wait for this thread's earlier 4-byte async
// copies (the pending count rises by one now and falls when they land).
__device__ __forceinline__ void cp_async_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];\n" ::"r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar))
               : "memory");
}

// Warp 0: all copies of item G into ring buffer `sr`, raster-word buffer
// `sprev`, trial-record buffer `strl` and the state buffer, completing on
// `bar`.  The raster words go first: their arrivals raise the barrier's
// pending count before the expect-tx arrival that would otherwise let the
// phase complete.
__device__ __forceinline__ void stream_stage(const fis_engine& E, const int32_t* ring,
                                             const int b0, const int nb, const int K,
                                             const ItemGeo& G, int32_t (*sr)[kTile],
                                             uint32_t (*sprev)[kUpdThreads / kWarp],
                                             fis_trial* strl,
                                             float (*sst)[StreamSmem::kArrays][StreamSmem::kStateWords],
                                             uint8_t (*sfl)[StreamSmem::kFlagBytes],
                                             uint64_t* bar, const int slot_prev) {
  const int lane = threadIdx.x;
  const int Wd = (E.n + kWarp - 1) / kWarp;
  {
    const int t = lane / (kUpdThreads / kWarp), w = lane % (kUpdThreads / kWarp);
    if (t < G.nt && G.tile * kTile + w * kWarp < E.n) {
      const int64_t word = ((int64_t)(b0 + 2 * G.pp + t) * Wd + G.tile * (kTile / kWarp) + w) *
                               E.p.lag + slot_prev;
      cp_async4(&sprev[t][w], E.bits + word, policy_keep());
      cp_async_arrive(bar);
    }
  }
  __syncwarp();
  if (lane == 0) mbar_arrive_expect_tx(bar, item_bytes(G, K));
  __syncwarp();
  if (E.inject_stall) return;
  const int NR = ring_row(E.n);
  const int64_t sstride = (int64_t)((nb + 1) >> 1) * NR * 2;
  const int64_t toff = ((int64_t)G.pp * NR + G.tile * kTile) * 2;
  if (lane < K)
    bulk_load(&sr[lane][0], reinterpret_cast<const uint16_t*>(ring) + (int64_t)lane * sstride + toff,
              kTile * 4u, bar, policy_keep());
  // the pair's trial records (consecutive), then the state rows: lane =
  // trial * 6 + array (array 5 = the flags)
  if (lane == 2 * (StreamSmem::kArrays + 1))
    bulk_load(strl, E.trials + (b0 + 2 * G.pp), (unsigned)G.nt * (unsigned)sizeof(fis_trial),
              bar, policy_keep());
  const int t = lane / (StreamSmem::kArrays + 1), a = lane % (StreamSmem::kArrays + 1);
  const bool direct = t == 0 ? G.direct[0] : G.direct[1];  // selected, not indexed
  const int64_t first = t == 0 ? G.first[0] : G.first[1];
  if (t >= 2 || direct) return;
  const uint64_t pol = policy_stream();
  if (a < StreamSmem::kArrays) {
    const float* base = a == 0   ? E.v
                        : a == 1 ? E.g
                        : a == 2 ? E.refrac
                        : a == 3 ? E.rates
                                 : reinterpret_cast<const float*>(E.kicks);
    bulk_load(&sst[t][a][0], base + (first - (first & 3)), StreamSmem::kStateWords * 4u, bar,
              pol);
  } else {
    bulk_load(&sfl[t][0], E.flags + (first - (first & 15)), StreamSmem::kFlagBytes, bar, pol);
  }
}

// Grid: up to 4 CTAs per SM, each a near-equal run of the group's items.
__global__ void __launch_bounds__(kUpdThreads, 4)
k_update_stream(const fis_engine E, const int b0, const int nb, const int K,
                int32_t* __restrict__ ring, float* __restrict__ spikes_out, const int bump,
                const float unit, const fis_clock clk, const int clk_given) {
  extern __shared__ __align__(128) uint8_t dsm[];
  using S = StreamSmem;
  auto sring = reinterpret_cast<int32_t(*)[FIS_MAX_BLOCK][kTile]>(dsm);
  auto sst = reinterpret_cast<float(*)[S::kArrays][S::kStateWords]>(dsm + S::kState);
  auto sfl = reinterpret_cast<uint8_t(*)[S::kFlagBytes]>(dsm + S::kFlags);
  uint32_t* szero = reinterpret_cast<uint32_t*>(dsm + S::kZero);
  auto sbal = reinterpret_cast<uint32_t(*)[kUpdThreads / kWarp][FIS_MAX_BLOCK]>(dsm + S::kBal);
  auto sprev = reinterpret_cast<uint32_t(*)[2][kUpdThreads / kWarp]>(dsm + S::kPrev);
  auto strl = reinterpret_cast<fis_trial(*)[2]>(dsm + S::kTrials);
  uint64_t* full = reinterpret_cast<uint64_t*>(dsm + S::kBar);
  uint64_t* taken = full + 2;
  fis_clock* sck = reinterpret_cast<fis_clock*>(dsm + S::kClock);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(dsm + S::kAbort);

  const int n = E.n;
  const int ntiles = ring_row(n) / kTile;
  const int items = ((nb + 1) >> 1) * ntiles;
  const int j0 = (int)((int64_t)blockIdx.x * items / gridDim.x);
  const int j1 = (int)((int64_t)(blockIdx.x + 1) * items / gridDim.x);
  const int lane = threadIdx.x & (kWarp - 1);
  const int wib = threadIdx.x / kWarp;
  const bool w0 = threadIdx.x < kWarp;
  const unsigned polls = E.wait_polls ? E.wait_polls : kWaitPolls;
  const uint64_t stream = policy_stream();

  if (threadIdx.x == 0) {
    *sck = clk_given ? clk : *E.clock;  // the block's clock
    *abort_flag = 0;
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_init(taken, kUpdThreads / kWarp);
    fence_mbar_init();
  }
  if (w0) {
#pragma unroll
    for (int q = 0; q < kTile / kWarp; ++q) szero[q * kWarp + lane] = kEmptyPair;
    fence_proxy_async_shared();
  }
  __syncthreads();
  const fis_clock& ck = *sck;
  const int slot_prev = ck.slot == 0 ? E.p.lag - 1 : ck.slot - 1;
  // With `bump` the grid's last CTA advances the clock: each CTA counts
  // itself in once every thread can read the clock from shared memory.
  unsigned arrived = 0;
  if (bump && threadIdx.x == 0) arrived = atomicAdd(E.done, 1u) + 1u;
  int issued = j0 - 1, seen = j0 - 1;  // warp 0: items staged / waited for
  if (w0 && j0 < j1) {
    stream_stage(E, ring, b0, nb, K, item_geo(E, b0, nb, ntiles, j0), sring[0], sprev[0],
                 strl[0], sst, sfl, &full[0], slot_prev);
    issued = j0;
  }

  for (int j = j0; j < j1; ++j) {
    const int s = (j - j0) & 1;
    const unsigned par = (unsigned)((j - j0) >> 1) & 1u;
    const ItemGeo G = item_geo(E, b0, nb, ntiles, j);
    const int pp = G.pp, tile = G.tile, nt = G.nt;
    const int i = tile * kTile + threadIdx.x;
    const bool valid = i < n;
    const bool warp_valid = (i - lane) < n;
    int64_t sidx[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) sidx[t] = G.first[t] + threadIdx.x;
    // A wait that runs out ends this warp's run (decided by the whole warp,
    // which stays together for its ballots): the error goes to the host, the
    // other warps see the abort or run out in turn, and warp 0 drains the
    // copies it issued before the CTA ends.
    const bool ok = __all_sync(0xFFFFFFFFu, mbar_wait(&full[s], par, polls));
    if (!ok) {
      if (lane == 0) {
        atomicOr(E.done + 1, (uint32_t)FIS_ERR_STAGE);
        *abort_flag = 1;
      }
      break;
    }
    if (w0) seen = j;
    fis_trial tr[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) tr[t] = strl[s][t < nt ? t : 0];

    // this item's state, from the state buffer (or directly)
    uint32_t fl[2] = {0u, 0u}, dm[2] = {0u, 0u};
    float rate[2] = {0.f, 0.f}, vv[2] = {0.f, 0.f}, gg[2] = {0.f, 0.f}, rr[2] = {0.f, 0.f};
    bool bit[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      bit[t] = (sprev[s][t][wib] >> lane) & 1u;
      if (valid && t < nt) {
        if (!G.direct[t]) {
          const int o = G.ofs[t] + threadIdx.x;
          vv[t] = sst[t][0][o];
          gg[t] = sst[t][1][o];
          rr[t] = sst[t][2][o];
          rate[t] = sst[t][3][o];
          dm[t] = __float_as_uint(sst[t][4][o]);
          fl[t] = sfl[t][G.ofb[t] + threadIdx.x];
        } else {
          fl[t] = ld_hint(E.flags + sidx[t], stream);
          vv[t] = ld_hint(E.v + sidx[t], stream);
          gg[t] = ld_hint(E.g + sidx[t], stream);
          rr[t] = ld_hint(E.refrac + sidx[t], stream);
          rate[t] = ld_hint(E.rates + sidx[t], stream);
          dm[t] = ld_hint(E.kicks + sidx[t], stream);
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(taken);

    if (w0) {
      if (j + 1 < j1) {
        // every warp has taken item j's state, so has finished item j-1:
        // stage s ^ 1, the state buffer and the small buffers s ^ 1 may be
        // refilled
        const bool room = __all_sync(
            0xFFFFFFFFu, mbar_wait(taken, (unsigned)(j - j0) & 1u, polls) && !*abort_flag);
        if (room) {
          stream_stage(E, ring, b0, nb, K, item_geo(E, b0, nb, ntiles, j + 1), sring[s ^ 1],
                       sprev[s ^ 1], strl[s ^ 1], sst, sfl, &full[s ^ 1], slot_prev);
          issued = j + 1;
        } else if (lane == 0) {
          atomicOr(E.done + 1, (uint32_t)FIS_ERR_STAGE);
          *abort_flag = 1;
        }
      }
      // this item's slots back to empty in the ring (see update_tile)
      const int NR = ring_row(n);
      const int64_t sstride = (int64_t)((nb + 1) >> 1) * NR * 2;
      const int64_t toff = ((int64_t)pp * NR + tile * kTile) * 2;
      if (lane < K)
        bulk_store(reinterpret_cast<uint16_t*>(ring) + (int64_t)lane * sstride + toff, szero,
                   kTile * 4u, policy_keep());
      bulk_commit();
    }

    TileState St;
    bool drv_any = false;
    const int64_t t0 = ck.step;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      St.ka[t] = (int)max((int64_t)0, min(tr[t].start - t0, (int64_t)K));
      St.kb[t] = (int)max((int64_t)0, min(tr[t].end - t0, (int64_t)K));
      St.runs[t] = t < nt && St.ka[t] < St.kb[t];
      const bool on = St.runs[t];
      const float prob = __fmul_rn(rate[t], E.p.prob_scale);
      St.dm[t] = (on && prob > 0.f) ? dm[t] : 0u;
      drv_any = drv_any || (valid && on && prob > 0.f);
      St.fl[t] = on ? fl[t] : 0u;
      St.v[t] = on ? vv[t] : 0.f;
      St.g[t] = on ? gg[t] : 0.f;
      St.r[t] = on ? rr[t] : 0.f;
      St.vclamp[t] = tr[t].v_clamp;
      St.s_prev[t] = on && warp_valid && t0 - 1 >= tr[t].start - tr[t].history && t0 >= 1 &&
                     bit[t];
    }
    const bool warp_driven = __any_sync(0xFFFFFFFFu, drv_any);
    if (St.runs[0] || St.runs[1])
      tile_compute<false, true>(E, b0, K, spikes_out, unit, ck, tile, pp, sring[s], sbal, St,
                                warp_driven, sidx);
    if (__any_sync(0xFFFFFFFFu, *abort_flag != 0)) break;
  }
  if (w0) {
    // copies still in flight (a run cut short) land before the CTA ends
    bool lost = false;
    for (int j = seen + 1; j <= issued; ++j)
      lost |= !__all_sync(0xFFFFFFFFu, mbar_wait(&full[(j - j0) & 1],
                                                 (unsigned)((j - j0) >> 1) & 1u, polls));
    cp_async_wait_all();
    if (lost && lane == 0) atomicOr(E.done + 1, (uint32_t)FIS_ERR_STAGE_LOST);
    // the clearing copies have read szero before the CTA ends
    bulk_wait_all();
  }
  if (threadIdx.x == 0) clock_bump(E, bump, arrived, ck, K);
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

// dst[r][b][i] += src[r][b][i] with separate row and trial strides.  With
// `half` the destination is the paired biased int16 ring: row r, pair b / 2
// (stride dt words), word i, trial b in half b % 2 -- two threads may share a
// word, so the add is atomic.
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
      uint32_t* d = reinterpret_cast<uint32_t*>(dst) + r * ds + (bb >> 1) * dt + i;
      atomicAdd(d, (uint32_t)v << ((bb & 1) * 16));
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

// 32-bit words of a scratch ring of `k` slots for `nb` trials: [k][nb][NR]
// int32, or [k][ceil(nb / 2)][NR] words of paired biased int16 counts.
int64_t ring_words(const fis_engine* e, int k, int nb) {
  return (int64_t)k * (e->ring16 ? (nb + 1) / 2 : nb) * ring_row(e->n);
}

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
      !e->bits || !e->clock || !e->done || !e->kicks)
    return FIS_E_ARG;
  if (e->n < 1 || e->n > (1 << 18) || e->batch < 1 || e->nnz < 0) return FIS_E_ARG;
  if (e->chunk < 128 || (e->chunk % 128) != 0) return FIS_E_ARG;
  if (e->list_cap < 1) return FIS_E_ARG;
  if (e->p.lag < 2 || e->p.buf_len != e->p.lag - 1) return FIS_E_ARG;
  if (e->n_recs < 0 || (e->n_recs > 0 && !e->recs)) return FIS_E_ARG;
  if (e->scatter_mode < 0 || e->scatter_mode > 1) return FIS_E_ARG;
  if (e->scat_ctas < 0 || e->drive_ctas < 0 || e->scat_ctas > 256 || e->drive_ctas > 256)
    return FIS_E_ARG;
  if (e->update_streams < 0 || e->update_streams > 2) return FIS_E_ARG;
  if (e->update_tiles < 0 || e->update_tiles > 2) return FIS_E_ARG;
  if (!e->drive_idx != !e->drive_len) return FIS_E_ARG;  // both lists or neither
  if (!aligned16(e->edges)) return FIS_E_ALIGN;
  return FIS_OK;
}

// Everything fis_block checks except the ring pointer itself.
static int check_block_shape(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps) {
  int rc = fis_check(e);
  if (rc) return rc;
  if ((rc = check_range(e, b0, nb))) return rc;
  if (k_steps < 1 || k_steps > FIS_MAX_BLOCK || k_steps > e->p.lag) return FIS_E_BOUNDS;
  if (e->vstim && k_steps != 1) return FIS_E_BOUNDS;
  if ((k_steps + 1) * nb + 1 > kMaxLists) return FIS_E_BOUNDS;
  const int64_t rows = (int64_t)nb * ring_row(e->n);
  if (rows * FIS_MAX_BLOCK > 0x7FFFFFFFLL) return FIS_E_BOUNDS;
  return FIS_OK;
}

static int check_block(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps,
                       const int32_t* ring) {
  const int rc = check_block_shape(e, b0, nb, k_steps);
  if (rc) return rc;
  if (!ring) return FIS_E_ARG;
  if (((uintptr_t)ring & 15u) != 0) return FIS_E_ALIGN;
  return FIS_OK;
}

}  // extern "C"

namespace {

// The block's clock for a launch inside fis_advance*: the host knows every
// block's step there, so launches need not wait for the device clock to be
// advanced between blocks (only the call's last launch advances it).
fis_clock clock_at(const fis_engine* e, int64_t step) {
  fis_clock c;
  c.step = step;
  c.slot = (int32_t)(step % e->p.lag);
  c.slot2 = (int32_t)(step % (2 * e->p.lag));
  return c;
}

int scatter_block(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps, int32_t* ring,
                  cudaStream_t st, const fis_clock* clk) {
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
  A.clk_given = clk ? 1 : 0;
  if (clk) A.clk = *clk;
  const size_t smem = sizeof(int32_t) * (size_t)((k_steps + 1) * nb + 1);
  // up to 8 CTAs per SM; fewer for small blocks (one trial, one step), where
  // the spikes of a step fill one pass of a CTA per SM
  const int per_sm = std::min(8, std::max(1, nb * k_steps / 2));
  // An external drive replaces the Philox draw; a one-step block draws its one
  // Philox word per driven neuron inside the update (no CTAs for so little).
  // With a drive, the grid is sized for the overlapped pipeline, where it
  // runs beside the previous group's update: every resident phase-A CTA holds
  // register-file room that an update CTA would use, so the grid is the
  // smallest that still ends within an update.  Up to 1.5 scattering and 3
  // drawing CTAs per SM (4.5 per SM, one wave at 5 per SM) measured best on
  // the full connectome for trial groups of 16 to 64.
  // The balanced scatter (mode 1), which keeps more loads in flight per
  // warp, defaults to one scattering and two drawing CTAs per SM.  With the
  // caller's lists of driven neurons the drive has a few percent of the
  // rates to read, and one drawing CTA per two SMs is enough.  The
  // descriptor may set both counts (per 8 SMs, for the autotuner).
  const bool balanced = e->scatter_mode == 1;
  int drive = 0;
  if (!e->vstim && k_steps > 1) {
    const int64_t warps = (int64_t)nb * ((e->n + kDriveSpan - 1) / kDriveSpan);
    const int64_t dflt = e->drive_idx ? std::max(1, sm_count() / 2)
                                      : (int64_t)sm_count() * (balanced ? 2 : 3);
    const int64_t cap = e->drive_ctas > 0 ? std::max(1, sm_count() * e->drive_ctas / 8) : dflt;
    const int64_t blocks = (warps + kDriveThreads / kWarp - 1) / (kDriveThreads / kWarp);
    drive = (int)(blocks < cap ? blocks : cap);
  }
  int scat = drive ? std::max(sm_count(), sm_count() * std::min(per_sm, 3) / 2)
                   : sm_count() * per_sm;
  if (balanced && drive) scat = sm_count();
  if (e->scat_ctas > 0) scat = std::max(1, sm_count() * e->scat_ctas / 8);
  if (balanced)
    k_phase_a<1><<<scat + drive, kScatThreads, smem, st>>>(*e, A, scat);
  else
    k_phase_a<0><<<scat + drive, kScatThreads, smem, st>>>(*e, A, scat);
  return launch_status();
}

int update_block(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps, int32_t* ring,
                 float* spikes_out, int32_t bump, cudaStream_t st, const fis_clock* clk) {
  const int rc = check_block(e, b0, nb, k_steps, ring);
  if (rc) return rc;
  const dim3 ugrid(ring_row(e->n) / kTile, (nb + 1) / 2);  // tiles x trial pairs
  fis_clock c{};
  if (clk) c = *clk;
  const int given = clk ? 1 : 0;
  const int bp = bump ? 1 : 0;
  const auto a16 = [](const void* q) { return ((uintptr_t)q & 15u) == 0; };
  if (!e->vstim && e->ring16 && k_steps > 1 && e->update_tiles == 2 && a16(e->v) &&
      a16(e->g) && a16(e->refrac) && a16(e->rates) && a16(e->kicks) && a16(e->flags) &&
      a16(e->trials)) {
    // streamed tiles: the attributes for its dynamic shared memory are set
    // once per device
    static int sized[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !sized[dev]) {
      cudaError_t err = cudaFuncSetAttribute(
          k_update_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)StreamSmem::kBytes);
      if (err == cudaSuccess)
        err = cudaFuncSetAttribute(k_update_stream,
                                   cudaFuncAttributePreferredSharedMemoryCarveout, 100);
      if (err != cudaSuccess) return (int)err;
      sized[dev] = 1;
    }
    // as many CTAs as fit at once (4 per SM), each a near-equal run of items
    const int items = ((nb + 1) / 2) * (ring_row(e->n) / kTile);
    const int grid = std::min(items, 4 * sm_count());
    k_update_stream<<<grid, kUpdThreads, StreamSmem::kBytes, st>>>(
        *e, b0, nb, k_steps, ring, spikes_out, bp, 1.0f, c, given);
    return launch_status();
  }
  if (e->vstim) {
    if (e->ring16)
      k_update<true, true><<<ugrid, kUpdThreads, 0, st>>>(*e, b0, nb, k_steps, ring, spikes_out,
                                                          bp, 1.0f, c, given);
    else
      k_update<true, false><<<ugrid, kUpdThreads, 0, st>>>(*e, b0, nb, k_steps, ring, spikes_out,
                                                           bp, 1.0f, c, given);
  } else {
    if (e->ring16)
      k_update<false, true><<<ugrid, kUpdThreads, 0, st>>>(*e, b0, nb, k_steps, ring, spikes_out,
                                                           bp, 1.0f, c, given);
    else
      k_update<false, false><<<ugrid, kUpdThreads, 0, st>>>(*e, b0, nb, k_steps, ring,
                                                            spikes_out, bp, 1.0f, c, given);
  }
  return launch_status();
}

int record_if(bool on, void* const* events, int64_t idx, cudaStream_t st) {
  if (!on) return FIS_OK;
  return (int)cudaEventRecord((cudaEvent_t)events[idx], st);
}

int check_advance(const fis_engine* e, int64_t start, int64_t steps, int32_t group, int32_t rows,
                  const int32_t* ring, void* const* events, int32_t n_pairs, int32_t every) {
  int rc = fis_check(e);
  if (rc) return rc;
  if (start < 0 || steps < 0 || group < 1 || rows < 0 || !ring) return FIS_E_ARG;
  if (events && (n_pairs < 0 || every < 1)) return FIS_E_ARG;
  return FIS_OK;
}

// Per-device side stream and events of fis_advance_overlap, created on first
// use and kept for the life of the process.
struct OverlapRes {
  cudaStream_t side = nullptr;
  cudaStream_t upd2 = nullptr;                    // second update stream
  cudaEvent_t after_sc[2] = {nullptr, nullptr};   // scatter of launch l done (l mod 2)
  std::vector<cudaEvent_t> after_upd;             // update of launch l done (l mod size)
  cudaEvent_t start = nullptr;                    // the call's starting point
  cudaEvent_t upd2_done = nullptr;                // the second update stream's last work
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
  if (!r.start) {
    // The side stream gets the highest priority: the block scheduler then
    // dispatches a scatter's CTAs as soon as update CTAs retire instead of
    // after the whole update grid, which is what lets the two overlap.
    int least = 0, greatest = 0;
    if ((err = cudaDeviceGetStreamPriorityRange(&least, &greatest))) return (int)err;
    if ((err = cudaStreamCreateWithPriority(&r.side, cudaStreamNonBlocking, greatest)))
      return (int)err;
    for (int j = 0; j < 2; ++j) {
      if ((err = cudaEventCreateWithFlags(&r.after_sc[j], cudaEventDisableTiming)))
        return (int)err;
    }
    if ((err = cudaStreamCreateWithFlags(&r.upd2, cudaStreamNonBlocking))) return (int)err;
    if ((err = cudaEventCreateWithFlags(&r.upd2_done, cudaEventDisableTiming))) return (int)err;
    if ((err = cudaEventCreateWithFlags(&r.start, cudaEventDisableTiming))) return (int)err;
  }
  *out = &r;
  return FIS_OK;
}

// At least `n` update events in R (created on first need, kept for the process).
int overlap_events(OverlapRes* R, size_t n) {
  while (R->after_upd.size() < n) {
    cudaEvent_t ev = nullptr;
    const cudaError_t err = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (err != cudaSuccess) return (int)err;
    R->after_upd.push_back(ev);
  }
  return FIS_OK;
}

}  // namespace

extern "C" {

int fis_scatter(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps, int32_t* ring,
                void* stream) {
  return scatter_block(e, b0, nb, k_steps, ring, (cudaStream_t)stream, nullptr);
}

int fis_update(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps, int32_t* ring,
               float* spikes_out, int32_t last_group, void* stream) {
  return update_block(e, b0, nb, k_steps, ring, spikes_out, last_group, (cudaStream_t)stream,
                      nullptr);
}

int fis_block(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps, int32_t* ring,
              float* spikes_out, int32_t last_group, void* stream) {
  const int rc = fis_scatter(e, b0, nb, k_steps, ring, stream);
  if (rc) return rc;
  return fis_update(e, b0, nb, k_steps, ring, spikes_out, last_group, stream);
}

int fis_advance(const fis_engine* e, int64_t start, int64_t steps, int32_t group, int32_t rows,
                int32_t* ring, float* spikes_out, void* const* events, int32_t n_pairs,
                int32_t every, void* stream) {
  int rc = check_advance(e, start, steps, group, rows, ring, events, n_pairs, every);
  if (rc) return rc;
  const int32_t B = (rows > 0 && rows < e->batch) ? rows : e->batch;
  const int kmax = e->p.lag < FIS_MAX_BLOCK ? e->p.lag : FIS_MAX_BLOCK;
  cudaStream_t st = (cudaStream_t)stream;
  int64_t done = 0;
  int64_t launch = 0;
  while (done < steps) {
    const int k = (int)(steps - done < kmax ? steps - done : kmax);
    const bool final_block = done + k == steps;
    const fis_clock clk = clock_at(e, start + done);
    float* sp = final_block ? spikes_out : nullptr;
    for (int32_t g0 = 0; g0 < B; g0 += group) {
      const int32_t nb = (B - g0) < group ? (B - g0) : group;
      const bool last = final_block && g0 + nb == B;  // advances the device clock
      if ((rc = scatter_block(e, g0, nb, k, ring, st, &clk))) return rc;
      const bool timed = events && (launch % every) == 0 && (launch / every) < n_pairs;
      if ((rc = record_if(timed, events, 2 * (launch / every), st))) return rc;
      if ((rc = update_block(e, g0, nb, k, ring, sp, last, st, &clk))) return rc;
      if ((rc = record_if(timed, events, 2 * (launch / every) + 1, st))) return rc;
      ++launch;
    }
    done += k;
  }
  return FIS_OK;
}

int fis_advance_overlap(const fis_engine* e, int64_t start, int64_t steps, int32_t group,
                        int32_t rows, int32_t* ring2, float* spikes_out, void* const* events,
                        int32_t n_pairs, int32_t every, void* stream) {
  int rc = check_advance(e, start, steps, group, rows, ring2, events, n_pairs, every);
  if (rc) return rc;
  const int32_t B = (rows > 0 && rows < e->batch) ? rows : e->batch;
  const int kmax = e->p.lag < FIS_MAX_BLOCK ? e->p.lag : FIS_MAX_BLOCK;
  const int32_t gmax = group < B ? group : B;
  int32_t* rings[2] = {ring2, ring2 + ring_words(e, kmax, gmax)};
  std::lock_guard<std::mutex> lk(g_overlap_mu);
  OverlapRes* R = nullptr;
  if ((rc = overlap_res(&R))) return rc;
  // Launch l (over all blocks and groups, in order) uses ring l mod 2.  Its
  // scatter runs on the side stream and waits for update l - 2, which
  // drained that ring, and for update l - ngroups, the same trial group one
  // block earlier, which wrote the spike lists the scatter reads; its update
  // waits for that scatter and for update l - ngroups (the group's state).
  // So each update overlaps the scatter of the next launch, across block
  // boundaries too.  With two update streams (e->update_streams == 2 and at
  // least two trial groups), consecutive updates -- of different groups,
  // hence independent -- alternate between the caller's stream and a second
  // one, so the tail of one update grid overlaps the start of the next.
  const int64_t ngroups = (B + group - 1) / group;
  const int nstreams = (e->update_streams == 2 && ngroups >= 2) ? 2 : 1;
  const int64_t M = ngroups + 2;  // update events kept: launches l-M .. l-1
  if ((rc = overlap_events(R, (size_t)M))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaStream_t ust[2] = {st, R->upd2};
  if ((rc = (int)cudaEventRecord(R->start, st))) return rc;
  if (nstreams == 2 && (rc = (int)cudaStreamWaitEvent(R->upd2, R->start, 0))) return rc;
  int64_t done = 0;
  int64_t launch = 0;
  while (done < steps) {
    const int k = (int)(steps - done < kmax ? steps - done : kmax);
    const bool final_block = done + k == steps;
    const fis_clock clk = clock_at(e, start + done);
    float* sp = final_block ? spikes_out : nullptr;
    for (int32_t g0 = 0; g0 < B; g0 += group) {
      const int32_t nb = (B - g0) < group ? (B - g0) : group;
      const bool last = final_block && g0 + nb == B;  // advances the device clock
      const int r = (int)(launch & 1);
      cudaStream_t us = ust[nstreams == 2 ? r : 0];
      if (launch >= 2) {
        if ((rc = (int)cudaStreamWaitEvent(R->side, R->after_upd[(launch - 2) % M], 0)))
          return rc;
      } else if ((rc = (int)cudaStreamWaitEvent(R->side, R->start, 0))) {
        return rc;
      }
      cudaEvent_t same_group = launch >= ngroups ? R->after_upd[(launch - ngroups) % M]
                                                 : nullptr;
      if (same_group && (rc = (int)cudaStreamWaitEvent(R->side, same_group, 0))) return rc;
      if ((rc = scatter_block(e, g0, nb, k, rings[r], R->side, &clk))) return rc;
      if ((rc = (int)cudaEventRecord(R->after_sc[r], R->side))) return rc;
      if ((rc = (int)cudaStreamWaitEvent(us, R->after_sc[r], 0))) return rc;
      if (same_group && nstreams == 2 && (rc = (int)cudaStreamWaitEvent(us, same_group, 0)))
        return rc;
      const bool timed = events && (launch % every) == 0 && (launch / every) < n_pairs;
      if ((rc = record_if(timed, events, 2 * (launch / every), us))) return rc;
      if ((rc = update_block(e, g0, nb, k, rings[r], sp, last, us, &clk))) return rc;
      if ((rc = record_if(timed, events, 2 * (launch / every) + 1, us))) return rc;
      if ((rc = (int)cudaEventRecord(R->after_upd[launch % M], us))) return rc;
      ++launch;
    }
    done += k;
  }
  if (nstreams == 2) {  // later work on the caller's stream follows both
    if ((rc = (int)cudaEventRecord(R->upd2_done, R->upd2))) return rc;
    if ((rc = (int)cudaStreamWaitEvent(st, R->upd2_done, 0))) return rc;
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
  const int32_t drows = e->ring16 ? (nb + 1) >> 1 : nb;  // pairs or trials of dst
  if (src_trial_stride < e->n || dst_trial_stride < e->n ||
      src_row_stride < (int64_t)(nb - 1) * src_trial_stride + e->n ||
      dst_row_stride < (int64_t)(drows - 1) * dst_trial_stride + e->n)
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
//  * it holds FIS_NOALLOC_RING_INTS int32 (12 MiB): one trial (or one pair
//    of trials with the paired int16 ring) of the 138,639-neuron connectome
//    in 20-step blocks; a call whose ring needs more words is refused with
//    FIS_E_BOUNDS;
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
  // Every argument check fis_block makes, before the array is touched: a
  // refused call launches nothing.
  int rc = check_block_shape(e, b0, nb, k_steps);
  if (rc) return rc;
  const int64_t need = ring_words(e, k_steps, nb);
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
