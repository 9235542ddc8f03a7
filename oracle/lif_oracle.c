/*
 * lif_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's whole-brain LIF step, used as the
 * checker of the CUDA engine and as the timed CPU baseline.  Nothing in the
 * product path links or calls this file.
 *
 * It follows, one float32 operation at a time and in the same order:
 *   Engine._core     lab/flybrain/sim.py:863-953   (the 11-op step)
 *   Engine._poisson  lab/flybrain/sim.py:848-861   (drive = w * (bern * gain))
 *   ring layout      lab/flybrain/sim.py:383-385   ([B][buf_len][N], ptr)
 *   recurrent        lab/flybrain/sim.py:910-919   (w_scale * (W @ (s*m_out)))
 * The recurrent product has the reference's two algorithms: "csrmv" pulls
 * every edge by postsynaptic row (torch.sparse.mm, sim.py:911-913, the
 * reference's default path) and "event" pushes the rows of spiking
 * presynaptic neurons (ev_spmv.cu:60-79).  Both sum integers in float32,
 * which is exact in any order below 2**24 (evspmv.py:957-994).  The csrmv
 * pull accumulates as torch's CPU kernel for a CSR matrix times a dense one
 * does, one fused multiply-add per entry in ascending column order, so it
 * also matches the reference bit for bit when a caller has written
 * fractional spikes (visdyn.py:660-676), where the order and the fusing
 * decide the last bits.
 *
 * The Bernoulli draw is not torch's generator: the reference's randomness is
 * replaced by a counter-based Philox4x32-10 stream (Salmon et al., SC'11),
 * identical to the CUDA engine's, so the reference itself can be driven by
 * the same input tape (the tape helper below) and compared bit for bit.
 *
 * Parity of this file is pinned by tests/golden, generated by running the
 * reference's own sim.Engine on the same tapes.
 *
 * Build: gcc -O2 -mfma -ffp-contract=off -fno-fast-math -fopenmp -shared -fPIC ... -lm
 * (-mfma makes fmaf the hardware instruction; -ffp-contract=off keeps every
 * other product and sum rounded on its own)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct oracle_params {
  float a_syn, a_mem, w_scale, kick, prob_scale;
  float v_rest, v_reset, v_th, refrac_steps;
  int32_t buf_len;
  int32_t lag;
  int32_t pad_;
} oracle_params;

typedef struct oracle_ctx {
  int n;
  int64_t nnz;
  const int64_t* row_ptr; /* by pre */
  const int32_t* col;
  const int32_t* cnt;
  int64_t* t_ptr;         /* by post */
  int32_t* t_pre;
  float* t_val;
} oracle_ctx;

/* ---- Philox4x32-10 ------------------------------------------------------ */

static void philox_round(uint32_t c[4], const uint32_t k[2]) {
  const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
  const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
  const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
  const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
  const uint32_t n0 = hi1 ^ c[1] ^ k[0];
  const uint32_t n2 = hi0 ^ c[3] ^ k[1];
  c[0] = n0;
  c[1] = lo1;
  c[2] = n2;
  c[3] = lo0;
}

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  uint32_t k[2] = {key[0], key[1]};
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k[0] += 0x9E3779B9u;
      k[1] += 0xBB67AE85u;
    }
    philox_round(c, k);
  }
  memcpy(out, c, sizeof(c));
}

/* The draw of neuron i at own step `own`: Philox4x32-10 with counter
 * (i, own/4 low, own/4 high, stream) and key (seed low, seed high); word
 * own % 4 of the output. */
static uint32_t drive_word(int i, int64_t own, uint32_t stream, uint64_t seed) {
  const uint64_t quad = (uint64_t)own >> 2;
  const uint32_t ctr[4] = {(uint32_t)i, (uint32_t)quad, (uint32_t)(quad >> 32), stream};
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t out[4];
  oracle_philox4x32_10(ctr, key, out);
  return out[own & 3];
}

/* One draw: fire iff float(x >> 8) * 2**-24 < f32(rate) * f32(dt/1000). */
static float drive_one(float rate, float prob_scale, float kick, int i, int64_t own,
                       uint64_t seed, uint32_t stream) {
  const float p = rate * prob_scale;
  if (!(p > 0.0f)) return 0.0f * kick; /* the reference's w * (0 * gain) */
  const uint32_t x = drive_word(i, own, stream, seed);
  const float u = (float)(x >> 8) * 0x1p-24f;
  return (u < p) ? kick : 0.0f * kick;
}

/* vstim[b][i] for trial b at its own step own_t[b] (the shared input tape). */
void oracle_drive(int n, int batch, const float* rates, const uint64_t* seeds,
                  const uint32_t* streams, const int64_t* own_t, float prob_scale,
                  float kick, float* vstim) {
  for (int b = 0; b < batch; ++b)
    for (int i = 0; i < n; ++i)
      vstim[(int64_t)b * n + i] = drive_one(rates[(int64_t)b * n + i], prob_scale, kick, i,
                                            own_t[b], seeds[b], streams[b]);
}

/* ---- context: the matrix in both orientations ------------------------- */

void* oracle_create(int n, int64_t nnz, const int64_t* row_ptr, const int32_t* col,
                    const int32_t* cnt) {
  oracle_ctx* c = (oracle_ctx*)calloc(1, sizeof(oracle_ctx));
  if (!c) return NULL;
  c->n = n;
  c->nnz = nnz;
  c->row_ptr = row_ptr;
  c->col = col;
  c->cnt = cnt;
  c->t_ptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  c->t_pre = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nnz ? nnz : 1));
  c->t_val = (float*)malloc(sizeof(float) * (size_t)(nnz ? nnz : 1));
  if (!c->t_ptr || !c->t_pre || !c->t_val) {
    free(c->t_ptr);
    free(c->t_pre);
    free(c->t_val);
    free(c);
    return NULL;
  }
  for (int64_t k = 0; k < nnz; ++k) c->t_ptr[col[k] + 1]++;
  for (int i = 0; i < n; ++i) c->t_ptr[i + 1] += c->t_ptr[i];
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  memcpy(fill, c->t_ptr, sizeof(int64_t) * (size_t)n);
  for (int pre = 0; pre < n; ++pre)
    for (int64_t k = row_ptr[pre]; k < row_ptr[pre + 1]; ++k) {
      const int64_t at = fill[col[k]]++;
      c->t_pre[at] = pre;
      c->t_val[at] = (float)cnt[k];
    }
  free(fill);
  return c;
}

void oracle_destroy(void* h) {
  oracle_ctx* c = (oracle_ctx*)h;
  if (!c) return;
  free(c->t_ptr);
  free(c->t_pre);
  free(c->t_val);
  free(c);
}

/* ---- the step ----------------------------------------------------------- */

/*
 * One call of Engine._core(vstim) for all trials.  Arrays are [B][N] float32
 * except ring [B][buf_len][N]; rec is scratch [B][N].
 * mode 0: event push; mode 1: csrmv pull.
 */
static void core_one_trial(const oracle_ctx* c, const oracle_params* p, int mode, int b,
                           float* v, float* g, float* spikes, float* refrac, float* ring,
                           int ptr, const float* rs, const float* m_fire,
                           const float* m_out, const float* m_in, const float* m_hold,
                           const float* v_hold, const float* vstim, float* rec) {
  const int n = c->n;
  const int64_t o = (int64_t)b * n;
  float* R = ring + (int64_t)b * p->buf_len * n;
  /* recurrent = w_scale * (W @ (spikes * m_out))  (sim.py:910-913) */
  if (mode == 0) {
    for (int i = 0; i < n; ++i) rec[o + i] = 0.0f;
    for (int pre = 0; pre < n; ++pre) {
      const float s = spikes[o + pre] * m_out[o + pre];
      if (s == 0.0f) continue;
      for (int64_t k = c->row_ptr[pre]; k < c->row_ptr[pre + 1]; ++k)
        rec[o + c->col[k]] += (float)c->cnt[k] * s;
    }
  } else {
    for (int post = 0; post < n; ++post) {
      float acc = 0.0f;
      for (int64_t k = c->t_ptr[post]; k < c->t_ptr[post + 1]; ++k) {
        const int pre = c->t_pre[k];
        acc = fmaf(c->t_val[k], spikes[o + pre] * m_out[o + pre], acc);
      }
      rec[o + post] = acc;
    }
  }
  for (int i = 0; i < n; ++i) rec[o + i] = p->w_scale * rec[o + i];

  for (int i = 0; i < n; ++i) {
    const int64_t x = o + i;
    /* refrac.add_(1).mul_(1 - spikes); gate = refrac >= refrac_steps */
    refrac[x] = (refrac[x] + 1.0f) * (1.0f - spikes[x]);
    const float gate = (refrac[x] >= rs[x]) ? 1.0f : 0.0f;
    /* delayed = ring[:, ptr] * m_in; g_new = g*(1-dt/tauSyn) + delayed*gate */
    const float delayed = R[(int64_t)ptr * n + i] * m_in[x];
    const float gn = g[x] * p->a_syn + delayed * gate;
    /* ring[:, ptr] = recurrent */
    R[(int64_t)ptr * n + i] = rec[x];
    /* v += vstim; v += a_mem * (g - (v - v_rest))   (old g) */
    float vv = v[x] + vstim[x];
    vv = vv + p->a_mem * (g[x] - (vv - p->v_rest));
    /* v = v * m_hold + v_hold */
    vv = vv * m_hold[x] + v_hold[x];
    /* spikes = (v > v_th) * m_fire */
    const float s = ((vv > p->v_th) ? 1.0f : 0.0f) * m_fire[x];
    /* v -= (v - v_reset) * spikes; g = g_new - g_new * spikes */
    vv = vv - (vv - p->v_reset) * s;
    v[x] = vv;
    spikes[x] = s;
    g[x] = gn - gn * s;
  }
}

int oracle_core(void* h, const oracle_params* p, int batch, int mode, float* v, float* g,
                float* spikes, float* refrac, float* ring, int32_t* ptr, const float* rs,
                const float* m_fire, const float* m_out, const float* m_in,
                const float* m_hold, const float* v_hold, const float* vstim, float* rec,
                int nthreads) {
  const oracle_ctx* c = (const oracle_ctx*)h;
  if (!c || !p || batch < 1 || p->buf_len < 1) return -1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) if (batch > 1)
#endif
  for (int b = 0; b < batch; ++b)
    core_one_trial(c, p, mode, b, v, g, spikes, refrac, ring, *ptr, rs, m_fire, m_out, m_in,
                   m_hold, v_hold, vstim, rec);
  *ptr = (*ptr + 1) % p->buf_len;
  return 0;
}

/*
 * `steps` calls of Engine.step: drive from the Philox tape, then _core.
 * own_t[b] is each trial's own step at the first call and is advanced.
 * raster (optional): [steps][B][(N+7)/8] bits, neuron i in byte i/8 bit i%8.
 * csrmv mode parallelises the pull over postsynaptic rows inside a trial, the
 * way torch's CPU csrmv does; event mode runs trials in parallel.
 */
int oracle_run(void* h, const oracle_params* p, int batch, int steps, int mode, float* v,
               float* g, float* spikes, float* refrac, float* ring, int32_t* ptr,
               const float* rs, const float* m_fire, const float* m_out, const float* m_in,
               const float* m_hold, const float* v_hold, const float* rates,
               const uint64_t* seeds, const uint32_t* streams, int64_t* own_t,
               uint8_t* raster, int nthreads) {
  const oracle_ctx* c = (const oracle_ctx*)h;
  if (!c || !p || batch < 1 || steps < 0 || p->buf_len < 1) return -1;
  const int n = c->n;
  const int64_t bn = (int64_t)batch * n;
  float* vstim = (float*)malloc(sizeof(float) * (size_t)bn);
  float* rec = (float*)malloc(sizeof(float) * (size_t)bn);
  if (!vstim || !rec) {
    free(vstim);
    free(rec);
    return -2;
  }
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const int nbytes = (n + 7) / 8;
  for (int t = 0; t < steps; ++t) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t x = 0; x < bn; ++x) {
      const int b = (int)(x / n), i = (int)(x % n);
      vstim[x] = drive_one(rates[x], p->prob_scale, p->kick, i, own_t[b], seeds[b], streams[b]);
    }
    const int ptr0 = *ptr;
    if (mode == 0) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) if (batch > 1)
#endif
      for (int b = 0; b < batch; ++b)
        core_one_trial(c, p, 0, b, v, g, spikes, refrac, ring, ptr0, rs, m_fire, m_out, m_in,
                       m_hold, v_hold, vstim, rec);
    } else {
      /* csrmv: parallel pull over (trial, post), then the parallel update */
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1024)
#endif
      for (int64_t x = 0; x < bn; ++x) {
        const int b = (int)(x / n), post = (int)(x % n);
        const int64_t o = (int64_t)b * n;
        float acc = 0.0f;
        for (int64_t k = c->t_ptr[post]; k < c->t_ptr[post + 1]; ++k) {
          const int pre = c->t_pre[k];
          acc = fmaf(c->t_val[k], spikes[o + pre] * m_out[o + pre], acc);
        }
        rec[x] = p->w_scale * acc;
      }
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
      for (int64_t x = 0; x < bn; ++x) {
        const int b = (int)(x / n), i = (int)(x % n);
        float* R = ring + (int64_t)b * p->buf_len * n;
        refrac[x] = (refrac[x] + 1.0f) * (1.0f - spikes[x]);
        const float gate = (refrac[x] >= rs[x]) ? 1.0f : 0.0f;
        const float delayed = R[(int64_t)ptr0 * n + i] * m_in[x];
        const float gn = g[x] * p->a_syn + delayed * gate;
        R[(int64_t)ptr0 * n + i] = rec[x];
        float vv = v[x] + vstim[x];
        vv = vv + p->a_mem * (g[x] - (vv - p->v_rest));
        vv = vv * m_hold[x] + v_hold[x];
        const float s = ((vv > p->v_th) ? 1.0f : 0.0f) * m_fire[x];
        vv = vv - (vv - p->v_reset) * s;
        v[x] = vv;
        spikes[x] = s;
        g[x] = gn - gn * s;
      }
    }
    *ptr = (ptr0 + 1) % p->buf_len;
    for (int b = 0; b < batch; ++b) own_t[b] += 1;
    if (raster) {
      uint8_t* row = raster + (int64_t)t * batch * nbytes;
      memset(row, 0, (size_t)batch * nbytes);
      for (int b = 0; b < batch; ++b)
        for (int i = 0; i < n; ++i)
          if (spikes[(int64_t)b * n + i] != 0.0f)
            row[(int64_t)b * nbytes + (i >> 3)] |= (uint8_t)(1u << (i & 7));
    }
  }
  free(vstim);
  free(rec);
  return 0;
}

/*
 * The same equations in float64, for the error statement of the float32 path:
 * every constant is the double the reference starts from (DT/tauSyn ...
 * before its float32 cast), every operation is rounded to double, and the
 * drive fires on the same Philox draws (the firing decision itself is the
 * float32 comparison of the tape, so both runs receive the same kicks).
 * Arrays are double [B][N] (ring [B][buf_len][N]); masks and refrac_steps
 * are the float arrays of the float32 run.
 */
typedef struct oracle_params64 {
  double a_syn, a_mem, w_scale, kick, v_rest, v_reset, v_th;
  float prob_scale;
  int32_t buf_len;
} oracle_params64;

int oracle_run_f64(void* h, const oracle_params64* p, int batch, int steps, double* v,
                   double* g, double* spikes, double* refrac, double* ring, int32_t* ptr,
                   const float* rs, const float* m_fire, const float* m_out, const float* m_in,
                   const float* m_hold, const float* v_hold, const float* rates,
                   const uint64_t* seeds, const uint32_t* streams, int64_t* own_t,
                   uint8_t* raster) {
  const oracle_ctx* c = (const oracle_ctx*)h;
  if (!c || !p || batch < 1 || steps < 0 || p->buf_len < 1) return -1;
  const int n = c->n;
  const int64_t bn = (int64_t)batch * n;
  double* rec = (double*)malloc(sizeof(double) * (size_t)bn);
  if (!rec) return -2;
  const int nbytes = (n + 7) / 8;
  for (int t = 0; t < steps; ++t) {
    const int ptr0 = *ptr;
    for (int b = 0; b < batch; ++b) {
      const int64_t o = (int64_t)b * n;
      for (int i = 0; i < n; ++i) rec[o + i] = 0.0;
      for (int pre = 0; pre < n; ++pre) {
        const double s = spikes[o + pre] * (double)m_out[o + pre];
        if (s == 0.0) continue;
        for (int64_t k = c->row_ptr[pre]; k < c->row_ptr[pre + 1]; ++k)
          rec[o + c->col[k]] += (double)c->cnt[k] * s;
      }
      double* R = ring + (int64_t)b * p->buf_len * n;
      for (int i = 0; i < n; ++i) {
        const int64_t x = o + i;
        const float fr = rates[x] * p->prob_scale;
        double vstim = 0.0;
        if (fr > 0.0f) {
          const uint32_t w = drive_word(i, own_t[b], streams[b], seeds[b]);
          if ((float)(w >> 8) * 0x1p-24f < fr) vstim = p->kick;
        }
        refrac[x] = (refrac[x] + 1.0) * (1.0 - spikes[x]);
        const double gate = (refrac[x] >= (double)rs[x]) ? 1.0 : 0.0;
        const double delayed = R[(int64_t)ptr0 * n + i] * (double)m_in[x];
        const double gn = g[x] * p->a_syn + delayed * gate;
        R[(int64_t)ptr0 * n + i] = p->w_scale * rec[x];
        double vv = v[x] + vstim;
        vv = vv + p->a_mem * (g[x] - (vv - p->v_rest));
        vv = vv * (double)m_hold[x] + (double)v_hold[x];
        const double s = ((vv > p->v_th) ? 1.0 : 0.0) * (double)m_fire[x];
        vv = vv - (vv - p->v_reset) * s;
        v[x] = vv;
        spikes[x] = s;
        g[x] = gn - gn * s;
      }
    }
    *ptr = (ptr0 + 1) % p->buf_len;
    for (int b = 0; b < batch; ++b) own_t[b] += 1;
    if (raster) {
      uint8_t* row = raster + (int64_t)t * batch * nbytes;
      memset(row, 0, (size_t)batch * nbytes);
      for (int b = 0; b < batch; ++b)
        for (int i = 0; i < n; ++i)
          if (spikes[(int64_t)b * n + i] != 0.0)
            row[(int64_t)b * nbytes + (i >> 3)] |= (uint8_t)(1u << (i & 7));
    }
  }
  free(rec);
  return 0;
}

int oracle_abi(void) { return 1; }
