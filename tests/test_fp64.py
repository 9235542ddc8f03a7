"""The float32 step against the same equations in float64.

The engine computes in float32 exactly as the reference does (bit-exact, see
test_oracle / test_parity_gpu); this file states that path's error against a
float64 restatement of the equations driven by the same Poisson draws: the
rasters stay identical for the first 100 ms, the membrane difference stays far
below a millivolt until then, and per-neuron rates over 1 s correlate at
>= 0.99 by the reference's own metric (jobs.py:956-971).
"""

import numpy as np

import scenarios as S
from oracle import oracle as O


def test_float32_against_float64_same_equations():
    from fis.metrics import compare_rates

    sc = S.SCENARIOS["small_b1"]
    c = S.connectome(sc)
    a = O.Oracle.from_connectome(c, batch=1, no_refractory=S.driven(sc), seed=sc["seed"])
    b = O.Oracle.from_connectome(c, batch=1, no_refractory=S.driven(sc), seed=sc["seed"])
    a.rates[:] = S.rates_matrix(sc)
    b.rates[:] = S.rates_matrix(sc)
    max_dv = 0.0
    r32, r64 = [], []
    for _ in range(10):                  # the first 100 ms in 10 ms pieces
        r32.append(a.run(100, raster=True))
        r64.append(b.run_f64(100, raster=True))
        max_dv = max(max_dv, float(np.abs(a.v.astype(np.float64) - b.v64).max()))
    assert np.array_equal(np.concatenate(r32), np.concatenate(r64))
    assert max_dv < 1e-2, max_dv
    rest32 = a.run(9000, raster=True)
    rest64 = b.run_f64(9000, raster=True)
    n = c.n
    cnt32 = sum(np.unpackbits(x[:, 0], axis=1, bitorder="little")[:, :n].sum(0)
                for x in r32 + [rest32])
    cnt64 = sum(np.unpackbits(x[:, 0], axis=1, bitorder="little")[:, :n].sum(0)
                for x in r64 + [rest64])
    m = compare_rates(cnt32, cnt64)
    assert m["corr"] >= 0.99 and m["jaccard"] >= 0.9, m
