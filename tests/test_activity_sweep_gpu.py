"""The activity sweep of the plain single trial: 0.1 %, 1 % and 10 % driven.

The full 138,639-neuron connectome with a 150 Hz Poisson drive on a seeded
0.1 %, 1 % or 10 % of the neurons, so that spikes per step range from a few
to several hundred on this synthetic connectome (the 10 % run settles near
40 Hz mean firing) and the scatter's load balance over the Pareto-tailed rows
is exercised from nearly idle to busy.  Each run is compared with the oracle
(the reference's step restated in C, pinned to the reference by
test_oracle.py) bit for bit over the configuration's full 10,000 steps (1 s):
per-neuron spike counts and the final state.
"""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEPS = 10_000  # 1 s
CHUNK = 1000    # oracle steps per call (bounds the raster it returns)


@pytest.fixture(scope="module")
def conn():
    import fis.connectome as C

    return C.synthetic(seed=0)


@pytest.mark.parametrize("frac", [0.001, 0.01, 0.10])
def test_activity_sweep_matches_oracle(conn, frac):
    from fis.batch import Batch, TrialSpec

    rng = np.random.default_rng(int(frac * 1e4) + 17)
    stim = np.sort(rng.choice(conn.n, size=int(frac * conn.n), replace=False))
    spec = TrialSpec(seed=1234 + int(frac * 1e4), steps=STEPS, stim=stim, rate_hz=150.0)
    b = Batch(conn, 1, group=1)
    counts = b.run([spec])[0]

    o = O.Oracle.from_connectome(conn, batch=1, no_refractory=stim, seed=spec.seed, streams=[0])
    o.rates[0, stim] = np.float32(150.0)
    want = np.zeros(conn.n, dtype=np.int64)
    per_step = []
    for _ in range(STEPS // CHUNK):
        raster = o.run(CHUNK, raster=True)
        bits = np.unpackbits(raster[:, 0], axis=1, bitorder="little")[:, :conn.n]
        per_step.append(bits.sum(1))
        want += bits.sum(0).astype(np.int64)
    per_step = np.concatenate(per_step)
    print("drive %.1f %%: %.1f spikes per step (max %d) over %d steps"
          % (100 * frac, per_step.mean(), per_step.max(), STEPS))
    assert per_step.max() > 0
    assert np.array_equal(counts, want)
    core = b.core
    assert np.array_equal(core.v[0].cpu().numpy(), o.v[0])
    assert np.array_equal(core.g[0].cpu().numpy(), o.conductance[0])
    assert np.array_equal(core.refrac[0].cpu().numpy(), o.refrac[0])
    if frac >= 0.10:
        assert per_step.max() > 100  # the busy end of the sweep
