"""Rate-level comparison of two runs (the reference's parity metric).

``compare_rates`` is the measure of ``jobs._compare_upstream``
(``lab/flybrain/jobs.py:956-971``): a neuron is active at >= 0.5 Hz; the
Pearson correlation of rates is taken over the union of both active sets; the
Jaccard index compares the sets themselves.
"""

from __future__ import annotations

import numpy as np


def compare_rates(rates_a, rates_b, min_rate=0.5):
    a_r = np.asarray(rates_a, dtype=np.float64)
    b_r = np.asarray(rates_b, dtype=np.float64)
    a = a_r >= min_rate
    b = b_r >= min_rate
    both = a | b
    corr = float(np.corrcoef(a_r[both], b_r[both])[0, 1]) if both.sum() > 2 else float("nan")
    return {"corr": corr, "jaccard": float((a & b).sum() / max(int(both.sum()), 1)),
            "n_active_a": int(a.sum()), "n_active_b": int(b.sum()),
            "spikes_ratio": float(a_r.sum() / b_r.sum()) if b_r.sum() else float("nan")}
