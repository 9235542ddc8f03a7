/*
 * fis.h -- C ABI of the B200 LIF engine for fly-in-silico's whole-brain step.
 *
 * Two families of entry points live here.
 *
 * 1. Drop-in replacements for the reference's own event-SpMV FFI
 *    (lab/flybrain/ev_spmv.cu:114-137, bound by lab/flybrain/evspmv.py:832-930
 *    through ctypes): same names, same argument meaning, same return
 *    convention (a cudaError_t code, 0 = success).  A reference build can load
 *    this library in place of its own DLL.
 *
 * 2. The fused engine (fis_*), which replaces the reference's per-step Python
 *    body Engine._core (lab/flybrain/sim.py:863-953) and the Poisson drive
 *    Engine._poisson (sim.py:848-861).  Every buffer is owned by the caller
 *    and passed as a device pointer; nothing here allocates device memory.
 *    Every call takes a CUDA stream and returns a status instead of trapping.
 *
 * Status codes: 0 = success, a positive value is the cudaError_t of a failed
 * launch, a negative value is one of FIS_E_* (argument checks on the host,
 * before anything is launched).
 */
#ifndef FIS_H
#define FIS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FIS_ABI_VERSION 9

/* Largest number of steps one block may advance (registers per thread). */
#define FIS_MAX_BLOCK 20

enum {
  FIS_OK = 0,
  FIS_E_ARG = -1,     /* a pointer is null or a size is out of range */
  FIS_E_BOUNDS = -2,  /* a trial range, block length or slot is out of range */
  FIS_E_ALIGN = -3    /* an array is not 16-byte aligned */
};

/* Error bits the device sets in done[1].
 * FIS_ERR_STAGE: a CTA whose staged input did not arrive within wait_polls
 *   skipped its update; the run is then invalid, and the CTA left its lines
 *   of the scratch ring as the scatter wrote them, so the caller must refill
 *   the whole ring with its empty value (0, or 0x80008000 per word with
 *   ring16) before passing it to another call.
 * FIS_ERR_STAGE_LOST: a CTA's second bounded wait, for copies still in
 *   flight after the first ran out, ran out as well; those copies may have
 *   written shared memory after the CTA ended.  Treat the CUDA context as
 *   unusable (destroy it, or end the process). */
enum { FIS_ERR_STAGE = 1u << 0, FIS_ERR_STAGE_LOST = 1u << 1 };

/* Per-neuron flag bits, one byte per (trial, neuron). */
enum {
  FIS_FL_FIRE_OFF = 1u << 0, /* m_fire = 0: the spike is not emitted        */
  FIS_FL_OUT_OFF = 1u << 1,  /* m_out  = 0: the spike reaches no synapse    */
  FIS_FL_IN_OFF = 1u << 2,   /* m_in   = 0: delayed input is discarded      */
  FIS_FL_HOLD = 1u << 3,     /* m_hold = 0, v_hold = the trial's v_clamp    */
  FIS_FL_NOREFRAC = 1u << 4, /* refrac_steps = 0 (driven neurons)           */
  FIS_FL_SILENCED = 1u << 5  /* per-trial silencing: in and out both off    */
};

/*
 * Model constants, each computed once on the host exactly as the reference
 * derives it (sim.py:356-366): the Python double value cast to float32.
 */
typedef struct fis_lif_params {
  float a_syn;        /* f32(1 - dt/tauSyn)                                  */
  float a_mem;        /* f32(dt/tauMem)                                      */
  float w_scale;      /* f32(wScale), mV per synapse                         */
  float kick;         /* f32(wScale) * f32(scalePoisson), a float32 product  */
  float prob_scale;   /* f32(dt/1000)                                        */
  float v_rest;
  float v_reset;
  float v_th;
  float refrac_steps; /* f32(round(tRefrac/dt))                              */
  int32_t buf_len;    /* int(tDelay/dt) + 1, the reference's ring length     */
  int32_t lag;        /* buf_len + 1: steps from a spike to its g update     */
  int32_t pad_;
} fis_lif_params;

/* The device-side step counter.  `slot` and `slot2` are step mod lag and
 * step mod 2*lag, kept beside the step so kernels index the spike history
 * without 64-bit division; kernels advance all three together. */
typedef struct fis_clock {
  int64_t step;
  int32_t slot;
  int32_t slot2;
} fis_clock;

/* One trial slot.  Times are global engine steps. */
typedef struct fis_trial {
  uint64_t seed;      /* Philox key of this trial's Poisson drive            */
  int64_t start;      /* global step at which the trial's own step 0 runs    */
  int64_t end;        /* first global step that is not simulated             */
  float v_clamp;      /* v_hold value of neurons under FIS_FL_HOLD           */
  uint32_t stream;    /* Philox counter word 3 (the trial's lane)            */
  int32_t rec;        /* recording buffer index, -1 = no recording           */
  int32_t bin_steps;  /* own steps per recording bin                         */
  int32_t n_bins;     /* bins in the recording buffer                        */
  int32_t history;    /* steps before `start` whose spikes are the trial's
                         own (1 after a restore that loaded the spikes of
                         step start-1; 0 for a fresh trial, whose slot may
                         hold a previous occupant's raster)                 */
} fis_trial;

/*
 * The engine descriptor.  All pointers are device pointers owned by the
 * caller.  Layouts (B = batch, N = n, L = params.lag, W = ceil(N/32)):
 *   row_ptr  int64 [N+1]       CSR by presynaptic neuron
 *   edges    uint32 [nnz4]     post << 14 | (count & 0x3fff), 16-byte aligned,
 *                              nnz4 = nnz rounded up to a multiple of 4
 *   nchunks  uint16 [N]        ceil(out_degree / chunk), 0 for no edges
 *   v, g, refrac  float [B][N] the reference's v, conductance, refrac
 *   flags    uint8 [B][N]      FIS_FL_* bits
 *   rates    float [B][N]      Poisson rate in Hz, read once per block
 *   vstim    float [B][N]      or NULL: an external drive (the reference's
 *                              voltage_stim, sim.py:863) replacing the Philox
 *                              draw; only 1-step blocks may use it
 *   trials   fis_trial [B]
 *   lists    uint32 [L][B][list_cap]  spike entries pre << 8 | chunk
 *   list_len int32 [2L][B]     entries per (step mod 2L, trial)
 *   bits     uint32 [B][W][L]  spike raster of the last L steps (slot innermost)
 *   clock    fis_clock [1]     global steps completed (device-side)
 *   done     uint32 [2]        [0] block-completion counter, zero between
 *                              calls; [1] error bits (FIS_ERR_*), set by the
 *                              device and cleared by the host after reading
 *   recs     int32* [n_recs]   recording buffers [n_bins][N]
 *   kicks    uint32 [B][N]     scratch: the Poisson kick steps of the current
 *                              block, written by phase A for neurons with a
 *                              positive rate (others are never read)
 *   drive_idx int32 [B][N] or NULL, drive_len int32 [B]: per trial b, the
 *                              first drive_len[b] entries of row b list a
 *                              superset of the neurons whose rate is
 *                              positive (any order, each below N).  When
 *                              set, phase A's Poisson drive visits only the
 *                              listed neurons instead of scanning every
 *                              rate; the draws and kicks are the same.  A
 *                              neuron with a positive rate that is missing
 *                              from its trial's list gets stale kicks: the
 *                              caller keeps the lists in step with `rates`.
 */
typedef struct fis_engine {
  const int64_t* row_ptr;
  const uint32_t* edges;
  const uint16_t* nchunks;
  float* v;
  float* g;
  float* refrac;
  uint8_t* flags;
  const float* rates;
  const float* vstim;
  const fis_trial* trials;
  uint32_t* lists;
  int32_t* list_len;
  uint32_t* bits;
  fis_clock* clock;
  uint32_t* done;
  int32_t* const* recs;
  uint32_t* kicks;
  const int32_t* drive_idx;
  const int32_t* drive_len;
  int64_t nnz;
  int64_t list_cap;
  int32_t n;
  int32_t batch;
  int32_t chunk;      /* edges per scatter work item, a multiple of 128     */
  int32_t n_recs;
  int32_t ring16;     /* scratch ring of biased int16 counts (see below)    */
  uint32_t wait_polls;   /* bound on a CTA's wait for its staged input, in
                            polls; 0 = the default (~4M, far above any copy) */
  uint32_t inject_stall; /* test hook: nonzero = issue no staging copy, so
                            every wait runs out and sets FIS_ERR_STAGE       */
  int32_t raster;     /* nonzero: keep the raster of every step in `bits`;
                         0: only of each block's last step (all the next
                         block needs), for runs that read spikes through
                         recordings and spike lists alone                  */
  int32_t scatter_mode;  /* how the scatter spreads its work items (spike,
                            chunk of a row) over warps: 0 = one item per warp
                            at a time; 1 = 32 items per warp, resolved
                            together, their edges walked as one stream of
                            16-byte quads.  Same sums either way.          */
  int32_t scat_ctas;     /* phase-A CTAs that scatter, per 8 SMs (0 = the
                            library's default for the mode)                 */
  int32_t drive_ctas;    /* phase-A CTAs that draw the Poisson drive, per 8
                            SMs (0 = default)                                */
  int32_t update_streams;  /* fis_advance_overlap: 2 = consecutive updates
                              (of different trial groups) alternate between
                              the caller's stream and a second one; else 1 */
  int32_t update_tiles;    /* 2 = streamed tiles: up to 4 CTAs per SM, each
                              pipelining a run of (trial pair, tile) items --
                              the next item's slots, state and trial records
                              arrive by bulk copies while the current one's
                              steps run (paired int16 ring, Philox drive,
                              blocks of 2+ steps, arrays and trial records on
                              16-byte boundaries); else 1 tile per CTA      */
  int32_t pad3_;
  fis_lif_params p;
} fis_engine;

/* ---- family 1: the reference's event-SpMV FFI ------------------------- */

/* out[b, col[k]] += val[k] * sp[b, pre] * mo[b, pre] over the CSR rows of
 * spiking presynaptic neurons.  Replaces ev_spmv_i32 (ev_spmv.cu:114-122).
 * `threads` is accepted for signature compatibility; the launch shape is the
 * library's own.  Returns a cudaError_t code. */
int ev_spmv_i32(const int* crow, const int* col, const float* val,
                const float* sp, const float* mo, float* out, int n,
                int batch, int threads, void* stream);

/* Same with 64-bit indices.  Replaces ev_spmv_i64 (ev_spmv.cu:124-132). */
int ev_spmv_i64(const long long* crow, const long long* col,
                const float* val, const float* sp, const float* mo,
                float* out, int n, int batch, int threads, void* stream);

/* ABI tag checked by the loader.  Replaces ev_spmv_abi (ev_spmv.cu:136-137),
 * which returns 3; this library returns the same value. */
int ev_spmv_abi(void);

/* ---- family 2: the fused engine ---------------------------------------- */

/* ABI version of the fis_* family (FIS_ABI_VERSION). */
int fis_abi(void);

/* Size of fis_engine / fis_trial as compiled, for the binding's check. */
int fis_sizeof_engine(void);
int fis_sizeof_trial(void);

/* Host-side validation of a descriptor (no device access).  Returns FIS_OK
 * or a FIS_E_* code.  Mirrors Events._check_bounds (evspmv.py:1057-1113)
 * for what can be checked without reading device memory. */
int fis_check(const fis_engine* e);

/*
 * Advance the trials in slots [b0, b0+nb) by one block of k_steps steps
 * (1 <= k_steps <= min(FIS_MAX_BLOCK, lag)).  Two launches: the scatter of
 * the spikes that reach these steps through the delay (CSR rows of spiking
 * neurons, int32 atomics into `ring`), then the fused neuron update of all
 * k_steps steps (refractory gate, delayed input, conductance, Poisson drive,
 * membrane, hold, threshold, reset).  Replaces one call of Engine.step per
 * step (sim.py:745-771, 863-953).
 *   ring        the scratch ring, NR = fis_ring_row(N) (N rounded up to a
 *               multiple of 256), 16-byte aligned; "empty" on entry and on
 *               exit.  Either int32 counts [k_steps][nb][NR] (empty = 0), or,
 *               when e->ring16 is set, 32-bit words [k_steps][ceil(nb/2)][NR]
 *               that pair trials 2p and 2p+1 of the call: uint16 values
 *               0x8000 + count, trial 2p in the low half (empty word =
 *               0x80008000).  The pairing is exact whenever every neuron's
 *               sum of |count| over its incoming synapses is below 2**15, as
 *               then no partial sum leaves (-2**15, 2**15) and a 32-bit
 *               atomic add of a sign-extended count into the low half never
 *               disturbs the high half.  Size in 32-bit words: k_steps *
 *               (ring16 ? ceil(nb/2) : nb) * NR
 *   spikes_out  float [B][N] or NULL: the spikes of the block's last step
 *   last_group  nonzero when this call completes the block for all trial
 *               groups; the device clock then advances by k_steps
 */
int fis_block(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps,
              int32_t* ring, float* spikes_out, int32_t last_group,
              void* stream);

/* Phase A of fis_block alone: the scatter into `ring` and the block's Poisson
 * drive into e->kicks (same arguments). */
int fis_scatter(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps,
                int32_t* ring, void* stream);

/* Phase B of fis_block alone: the fused update draining `ring`. */
int fis_update(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps,
               int32_t* ring, float* spikes_out, int32_t last_group, void* stream);

/*
 * Advance slots [0, rows) by `steps` steps (rows = 0: every slot): blocks of
 * min(FIS_MAX_BLOCK, lag) steps (the last one shorter), each block running
 * fis_scatter + fis_update for the trial groups [g0, g0+group) in turn.  The
 * native form of a host loop over fis_block.  Slots at or above `rows` must
 * not be running (their trials ended); they stay frozen.  `start` is the
 * device clock's step on entry: every launch is given its block's step, so
 * no launch waits for the clock, which the call's last launch advances to
 * start + steps.
 *   ring        scratch ring of fis_block's layout for min(FIS_MAX_BLOCK,
 *               lag) slots and `group` trials, empty on entry and on return
 *   spikes_out  float [B][N] or NULL, written by the last block
 *   events      NULL, or 2*n_pairs cudaEvent_t handles: pair j is recorded
 *               around the update launch number j*every (0-based over the
 *               whole call), for timing the dominant kernel
 */
int fis_advance(const fis_engine* e, int64_t start, int64_t steps, int32_t group,
                int32_t rows, int32_t* ring, float* spikes_out, void* const* events,
                int32_t n_pairs, int32_t every, void* stream);

/*
 * fis_advance with two scratch rings, so that each scatter (on a
 * library-owned side stream, one per device) runs while the previous update
 * runs on `stream`, across block boundaries too: launch l (over all blocks
 * and groups, in order) uses ring l mod 2 and its scatter waits only for
 * update l - 2 and for the previous block's update of the same trial group.
 * With e->update_streams == 2 and two or more trial groups, consecutive
 * updates alternate between `stream` and a second library-owned stream.
 * On return all work is ordered before later work on `stream`.
 *   ring2  two consecutive rings of fis_block's layout, each for
 *          min(FIS_MAX_BLOCK, lag) slots and min(group, rows or batch)
 *          trials, empty on entry and on return
 * Other arguments as fis_advance.  Calls are serialised inside the library.
 */
int fis_advance_overlap(const fis_engine* e, int64_t start, int64_t steps, int32_t group,
                        int32_t rows, int32_t* ring2, float* spikes_out, void* const* events,
                        int32_t n_pairs, int32_t every, void* stream);

/*
 * Write the reference's pending delay ring (Engine.delay_buffer,
 * sim.py:385) for slots [b0, b0+nb): out float [nb][buf_len][N], slot
 * s mod buf_len holding w_scale * the counts that reach step s (from the
 * spikes of step s - lag), for the pending steps s = clock .. clock+buf_len-1.
 * `scratch` int32 [buf_len][nb][N] is accumulated into: the caller zeroes it
 * and may preload counts that are pending from a restored ring.
 */
int fis_delay_buffer(const fis_engine* e, int32_t b0, int32_t nb,
                     int32_t* scratch, float* out, void* stream);

/* Expand the spike bits of global step `step` into float 0/1 [nb][N]. */
int fis_spikes_f32(const fis_engine* e, int32_t b0, int32_t nb, int64_t step,
                   float* out, void* stream);

/*
 * Load a pending spike list from a float 0/1 spike tensor [nb][N] as the
 * spikes of global step clock-1 (restore path; the reference keeps these in
 * Engine.spikes).  Entries are written unfiltered, as the block that
 * consumes them filters by m_out.  Also writes the raster bits.
 */
int fis_load_spikes(const fis_engine* e, int32_t b0, int32_t nb,
                    const float* spikes, void* stream);

/* dst[r][b][i] += src[r][b][i] for r < rows, b < nb, i < N, with row and
 * trial strides given in elements (restore path: pending delayed input that a
 * restored delay ring holds for the next buf_len steps).  `dst` is a scratch
 * ring of fis_block's layout: with e->ring16 its strides count 32-bit words
 * and step over trial pairs (trial b in half b % 2 of pair b / 2). */
int fis_add_rows(const fis_engine* e, int32_t nb, int32_t rows,
                 const int32_t* src, int64_t src_row_stride,
                 int64_t src_trial_stride, int32_t* dst, int64_t dst_row_stride,
                 int64_t dst_trial_stride, void* stream);

/*
 * Graded-spike mode: one step of the reference's float path (sim.py:863-953
 * with the csrmv product of sim.py:910-913) for callers that write fractional
 * values into the spike state (visdyn.py:660-676), where whole-spike integer
 * counts no longer describe the input.  All trials [0, batch) of `e` advance
 * one step:
 *   recurrent[b][post] = w_scale * sum over in-edges, ascending pre, of
 *                        val * (spikes[b][pre] * m_out[b][pre]), one fused
 *                        multiply-add per edge (torch's CPU csrmv order)
 *   then the step with ring[b][ptr] as the delayed input, which the slot
 *   then takes over from `recurrent`; spikes[b] becomes the new 0/1 spikes.
 * e's v, g, refrac, flags (masks, silencing, no-refractory), rates, trials
 * (seed, lane, start, clamp value) and params are used as by fis_block; the
 * drive is e's Philox draw for global step `step`, or `vstim` [B][N] when
 * non-null.  t_ptr int64 [N+1] / t_pre int32 [E] / t_val float [E]: the
 * weights W[post, pre] as CSR by postsynaptic neuron, presynaptic indices
 * ascending within a row.  spikes float [B][N] (read, then written), ring
 * float [B][buf_len][N], rec scratch of B*N floats followed by
 * B*ceil(N/32) 32-bit words; 0 <= ptr < buf_len.
 * Replaces Engine._core's float path (sim.py:863-953) for graded spikes.
 */
int fis_graded_step(const fis_engine* e, int64_t step, const int64_t* t_ptr,
                    const int32_t* t_pre, const float* t_val, float* spikes, float* ring,
                    int32_t ptr, float* rec, const float* vstim, void* stream);

/* Row length NR of the scratch ring for N neurons (N rounded up to 256). */
int fis_ring_row(int32_t n);

/*
 * Measurement aid, no counterpart in the reference: `ctas` CTAs of 256
 * threads each add 1 (red.add.u32) at `iters` pseudo-random words of
 * buf[0, words) -- ctas * 256 * iters atomic adds in all.  Timed by the
 * caller, it gives the sustained L2 atomic-add rate that bounds the scatter
 * (one such add per pushed synapse).  iters: a positive multiple of 8.
 */
int fis_red_rate(uint32_t* buf, int64_t words, int32_t iters, int32_t ctas, void* stream);

/*
 * fis_block without the `ring` argument: the scratch ring is a fixed array
 * of FIS_NOALLOC_RING_INTS int32 (12 MiB) inside this library, for callers
 * that cannot allocate device memory (a real-time closed-loop controller,
 * where an allocation may stall the GPU; a foreign-language host with no
 * device allocator).  No counterpart in the reference.  Blocks whose ring
 * (fis_block's size in 32-bit words) exceeds FIS_NOALLOC_RING_INTS return
 * FIS_E_BOUNDS.  Every GPU that loads the library keeps the array until
 * exit; calls overlapping on the GPU race on it; each call clears what it
 * uses; the first call on a device looks up the array's address and should
 * come before any stream capture.  Arguments are checked as fis_block
 * checks them before anything is launched.
 */
#define FIS_NOALLOC_RING_INTS (3 << 20)
int fis_block_noalloc(const fis_engine* e, int32_t b0, int32_t nb, int32_t k_steps,
                      float* spikes_out, int32_t last_group, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FIS_H */
