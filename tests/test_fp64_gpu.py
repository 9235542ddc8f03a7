"""The engine's float32 error against float64 on sampled trials of the batch.

Four trials of the benchmark's trial mix (own seed, stimulus set, rate and
silencing each) run on the GPU for 100 ms; the same equations in float64
(the oracle's FP64 restatement, same Poisson draws) give the same spike
counts, and the membrane potentials differ by less than 0.1 mV (about 40 uV
measured).
The float32 engine equals the reference bit for bit (test_parity_gpu.py), so
this is the reference's float32 error as well.
"""

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
