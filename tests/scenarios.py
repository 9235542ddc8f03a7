"""Parity scenarios shared by the golden generator and the tests.

Each scenario is a seeded synthetic connectome, a Poisson drive on a seeded
subset, a model-parameter set and a schedule of ``set_masks`` calls applied
before given steps.  Everything is derived from the integers below, so the
reference (here), the oracle and the CUDA engine all see the same inputs.
The mask windows follow the reference's own parity probe
(``lab/probe/lif_event.py:233-243``): each intervention alone and all four
together, with windows longer than the 19/20-step delay tails.
"""

from __future__ import annotations

import numpy as np

ALT_PARAMS = {
    "tauSyn": 4.0, "tDelay": 1.0, "v0": -55.0, "vReset": -58.0, "vRest": -52.5,
    "vThreshold": -46.3, "tauMem": 17.0, "tRefrac": 1.3, "scalePoisson": 200,
    "wScale": 0.31,
}

LIF_EVENT_PLAN = [(60, "fire"), (100, "clear"), (130, "out"), (170, "clear"),
                  (200, "inc"), (230, "clear"), (250, "hold"), (280, "clear"),
                  (300, "all"), (340, "clear")]

SCENARIOS = {
    "small_b1": dict(n=2048, e=2048 * 100, conn_seed=1, batch=1, steps=400,
                     seed=5, drive_k=300, drive_seed=2, rates=[150.0],
                     plan=[], params=None),
    "batch3_masks": dict(n=3000, e=3000 * 109, conn_seed=3, batch=3, steps=360,
                         seed=9, drive_k=400, drive_seed=4,
                         rates=[60.0, 150.0, 240.0], plan=LIF_EVENT_PLAN,
                         params=None),
    "silenced_b2": dict(n=2500, e=2500 * 110, conn_seed=5, batch=2, steps=300,
                        seed=13, drive_k=350, drive_seed=6, rates=[200.0, 120.0],
                        silenced_k=60, silenced_seed=8, plan=[], params=None),
    "alt_params": dict(n=2200, e=2200 * 105, conn_seed=7, batch=2, steps=320,
                       seed=21, drive_k=320, drive_seed=10, rates=[180.0, 90.0],
                       plan=[(40, "hold_clamp"), (90, "clear"), (150, "all"),
                             (200, "clear")], params=ALT_PARAMS),
    # Graded spikes (visdyn.py:660-676): before every step, fractional values
    # in [0, 0.9] are written into the spike state of a seeded set of neurons,
    # which the reference's csrmv product and refractory update then use.
    "graded_b2": dict(n=2400, e=2400 * 104, conn_seed=11, batch=2, steps=240, seed=17,
                      drive_k=300, drive_seed=12, rates=[150.0, 90.0],
                      plan=[(60, "all"), (150, "clear")], params=None,
                      graded_k=300, graded_seed=13),
    # The plain single-trial configuration at full size (1,000 steps).
    "full_cfg0": dict(n=138_639, e=15_091_983, conn_seed=0, batch=1, steps=1000,
                      seed=0, drive_k=2249, drive_seed=1, rates=[150.0], plan=[],
                      params=None),
    # The same configuration over 1 s (10,000 steps): rates over the run.
    "full_cfg0_1s": dict(n=138_639, e=15_091_983, conn_seed=0, batch=1, steps=10_000,
                         seed=0, drive_k=2249, drive_seed=1, rates=[150.0], plan=[],
                         params=None),
}

MILESTONES = (1, 10, 19, 20, 21, 40, 100, 200, 300, 400, 500, 1000)


def connectome(sc):
    import fis.connectome as C

    return C.synthetic(n=sc["n"], e=sc["e"], seed=sc["conn_seed"])


def driven(sc):
    rng = np.random.default_rng(sc["drive_seed"])
    return np.sort(rng.choice(sc["n"], size=sc["drive_k"], replace=False)).astype(np.int64)


def silenced(sc):
    if not sc.get("silenced_k"):
        return np.zeros(0, dtype=np.int64)
    rng = np.random.default_rng(sc["silenced_seed"])
    return np.sort(rng.choice(sc["n"], size=sc["silenced_k"], replace=False)).astype(np.int64)


def busy(sc):
    """Neurons the mask plan acts on: 300 driven ones and 300 others."""
    d = driven(sc)
    rng = np.random.default_rng(sc["drive_seed"] + 1000)
    others = np.setdiff1d(np.arange(sc["n"]), d)
    extra = rng.choice(others, size=min(300, others.size), replace=False)
    return np.concatenate([d[:300], np.sort(extra)]).astype(np.int64)


def rates_matrix(sc):
    r = np.zeros((sc["batch"], sc["n"]), dtype=np.float32)
    d = driven(sc)
    for b, hz in enumerate(sc["rates"]):
        r[b, d] = hz
    return r


def mask_call(what, idx):
    """Keyword arguments of the ``set_masks`` call for one plan entry."""
    if what == "clear":
        return dict(fire=[], out=[], inc=[], hold=[])
    if what == "all":
        return dict(fire=idx[:150], out=idx[150:300], inc=idx[300:450],
                    hold=idx[450:600])
    if what == "hold_clamp":
        return dict(hold=idx[:200], v_clamp=-61.5)
    return {what: idx}


def graded_spikes(sc, step):
    """(neurons, values [batch][k] float32) written into the spike state before
    ``step`` in a graded scenario, or None."""
    k = sc.get("graded_k")
    if not k:
        return None
    rng = np.random.default_rng(sc["graded_seed"])
    idx = np.sort(rng.choice(sc["n"], size=k, replace=False)).astype(np.int64)
    j = np.arange(k)[None, :]
    b = np.arange(sc["batch"])[:, None]
    vals = ((j * 7 + step * 3 + b * 5) % 17) / 17.0 * 0.9
    return idx, vals.astype(np.float32)


# sim.run through the experiment API (sim.py:990-1117): three stimuli whose
# windows switch on and off mid-bin and on a bin edge, per-trial Philox
# streams, silencing through the reference's own build path, a run length
# that leaves the last bin partial, and a second run that a should_stop
# callback cuts after bin ``stop_after_bin``.
RUN_SCENARIOS = {
    "run_b2": dict(n=2500, e=2500 * 110, conn_seed=21, batch=2, seed=31, t_run_s=0.0473,
                   bin_ms=5.0, silenced_k=40, silenced_seed=44, stop_after_bin=5,
                   stimuli=[dict(name="a", k=300, seed=41, rate_hz=210.0, t_on_ms=0.0,
                                 t_off_ms=20.0),
                            dict(name="b", k=250, seed=42, rate_hz=120.0, t_on_ms=12.3,
                                 t_off_ms=None),
                            dict(name="c", k=200, seed=43, rate_hz=90.0, t_on_ms=7.77,
                                 t_off_ms=31.4)]),
}


def run_stimuli(sc):
    """``(name, indices, rate_hz, t_on_ms, t_off_ms)`` of a run scenario."""
    out = []
    for s in sc["stimuli"]:
        rng = np.random.default_rng(s["seed"])
        idx = np.sort(rng.choice(sc["n"], size=s["k"], replace=False)).astype(np.int64)
        out.append((s["name"], idx, s["rate_hz"], s["t_on_ms"], s["t_off_ms"]))
    return out


# Reference snapshots (sim.py:780-814) taken mid-run, for restoring a state
# the reference wrote into this engine: scenario -> step of the snapshot.
# batch3_masks at 320 is inside the window where all four masks are set
# (hold included, so v_hold is not zero); silenced_b2 at 150 is mid-run.
SNAPSHOTS = {"batch3_masks": 320, "silenced_b2": 150}
