"""The engine's float32 error against float64 on sampled trials of the batch.

Four trials of the benchmark's trial mix (own seed, stimulus set, rate and
silencing each) run on the GPU for 100 ms; the same equations in float64
(the oracle's FP64 restatement, same Poisson draws) give the same spike
counts, and the membrane potentials differ by less than 0.1 mV (about 40 uV
measured).
The float32 engine equals the reference bit for bit (test_parity_gpu.py), so
this is the reference's float32 error as well.
"""

import copy

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEPS = 1000  # 100 ms
SAMPLED = (0, 21, 42, 63)


def test_float32_engine_against_float64_on_sampled_trials():
    import fis.connectome as C
    from fis.batch import Batch, random_specs

    conn = C.synthetic(seed=0)
    mix = random_specs(conn.n, 64, 2024, STEPS)
    specs = [mix[j] for j in SAMPLED]
    b = Batch(conn, len(specs), group=2)
    counts = b.run(specs)
    worst = 0.0
    for j, s in enumerate(specs):
        o = O.Oracle.from_connectome(conn.without(s.silenced), batch=1, no_refractory=s.stim,
                                     seed=s.seed, streams=[0])
        o.rates[0, np.asarray(s.stim)] = np.float32(s.rate_hz)
        r64 = o.run_f64(STEPS, raster=True)
        c64 = np.unpackbits(r64[:, 0], axis=1, bitorder="little")[:, :conn.n].sum(0)
        assert np.array_equal(counts[j], c64), j
        v = b.core.v[b.slots_of_run[j]].cpu().numpy().astype(np.float64)
        worst = max(worst, float(np.abs(v - o.v64[0]).max()))
    print("max |v32 - v64| over %d sampled trials after %d steps: %.3g mV"
          % (len(specs), STEPS, worst))
    assert worst < 0.1


UNEVEN_SAMPLED = (0, 85, 170, 255)


def test_uneven_mix_against_float64_on_sampled_trials():
    """The uneven 256-trial batch (durations U[500, 20,000] steps, 50-300 Hz,
    own stimulus set and silencing per trial): four sampled trials, on the
    GPU, against the same equations in float64 (same Poisson draws).  Over the
    first 100 ms the spike counts are identical and the membranes differ by
    less than 0.1 mV; over each trial's whole duration the per-neuron rates
    correlate at >= 0.99 by the reference's metric (jobs.py:956-971)."""
    import fis.connectome as C
    from fis.batch import Batch, random_specs
    from fis.metrics import compare_rates

    conn = C.synthetic(seed=0)
    mix = random_specs(conn.n, 256, 2024 + 7, (500, 20000))
    specs = [mix[j] for j in UNEVEN_SAMPLED]
    head = [copy.copy(s) for s in specs]
    for s in head:
        s.steps = min(s.steps, STEPS)
    b = Batch(conn, len(specs), group=2)
    first = b.run(head)
    v_head = [b.core.v[b.slots_of_run[j]].cpu().numpy().astype(np.float64)
              for j in range(len(specs))]
    whole = b.run(specs)
    worst, corrs = 0.0, []
    for j, s in enumerate(specs):
        o = O.Oracle.from_connectome(conn.without(s.silenced), batch=1, no_refractory=s.stim,
                                     seed=s.seed, streams=[0])
        o.rates[0, np.asarray(s.stim)] = np.float32(s.rate_hz)
        n0 = min(s.steps, STEPS)
        r = o.run_f64(n0, raster=True)
        c64 = np.unpackbits(r[:, 0], axis=1, bitorder="little")[:, :conn.n].sum(0)
        assert np.array_equal(first[j], c64), j
        worst = max(worst, float(np.abs(v_head[j] - o.v64[0]).max()))
        total = c64.astype(np.int64)
        left = s.steps - n0
        while left > 0:                  # 200 ms pieces bound the raster's size
            k = min(left, 2000)
            r = o.run_f64(k, raster=True)
            total += np.unpackbits(r[:, 0], axis=1,
                                   bitorder="little")[:, :conn.n].sum(0).astype(np.int64)
            left -= k
        seconds = s.steps * 1e-4         # 0.1 ms steps
        m = compare_rates(whole[j] / seconds, total / seconds)
        corrs.append(m["corr"])
        assert m["corr"] >= 0.99, (j, s.steps, m)
    print("uneven mix, %d sampled trials (%s steps): max |v32 - v64| at 100 ms %.3g mV, "
          "rate correlation over each trial %s"
          % (len(specs), [s.steps for s in specs], worst, ["%.4f" % c for c in corrs]))
    assert worst < 0.1
