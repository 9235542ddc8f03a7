"""``fis.sim.run`` and ``Engine.restore`` against the reference's own outputs.

* ``run``: the reference's experiment driver (``sim.py:990-1117``) was run
  with its Poisson draw replaced by the shared Philox tape
  (``tests/golden/make_golden.py``).  Here the same stimuli, silencing and
  configuration go through this engine's ``run``, whose Philox drive is that
  tape, and the result must be the same: per-neuron counts, the binned raster,
  every ``on_bin(bin, t_ms, counts)`` call, and, in a second run, the step at
  which ``should_stop`` ends it (``timing["steps"]``).
* ``restore``: a snapshot the reference's own engine wrote mid-run
  (``sim.py:780-814``: f32 ``delay_buffer [B,19,N]``, ``ptr``, masks,
  ``v_hold``) is restored into a fresh engine, which then continues on the
  tape; the rest of the run must equal the reference's, raster and final
  state.  The snapshot's generator state is torch's and is refused unless
  dropped: the drive continues from the tape.
"""

import numpy as np
import pandas as pd
import pytest
import torch

import scenarios as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def run_inputs(name):
    from fis import sim

    sc = S.RUN_SCENARIOS[name]
    conn = S.connectome(sc)
    stims = [sim.Stimulus(indices=idx, rate_hz=rate, t_on_ms=on, t_off_ms=off, name=nm)
             for nm, idx, rate, on, off in S.run_stimuli(sc)]
    neurons = pd.DataFrame({"region": np.array(["AL", "MB", "LH", "CX"])[np.arange(sc["n"]) % 4]})
    cfg = sim.RunConfig(t_run_s=sc["t_run_s"], bin_ms=sc["bin_ms"], n_trials=sc["batch"],
                        seed=sc["seed"], device="cuda")
    return sc, conn, stims, neurons, cfg


@pytest.mark.parametrize("tag", ["full", "stop"])
def test_run_matches_reference_run(tag, golden):
    from fis import sim

    z = golden("run_b2")
    sc, conn, stims, neurons, cfg = run_inputs("run_b2")
    calls, polls = [], [0]
    stop_after = sc["stop_after_bin"] if tag == "stop" else None

    def on_bin(b, t_ms, counts):
        assert counts.dtype == np.int16 and counts.shape == (sc["n"],)
        calls.append((b, t_ms, counts.copy()))

    def should_stop():
        polls[0] += 1
        return stop_after is not None and polls[0] > stop_after

    res = sim.run(stims, silenced=S.silenced(sc), config=cfg, neurons=neurons, weights=conn,
                  progress=False, on_bin=on_bin, should_stop=should_stop)
    assert res.timing["steps"] == int(z[tag + "_steps"])
    assert [c[0] for c in calls] == list(z[tag + "_onbin_b"])
    assert [c[1] for c in calls] == list(z[tag + "_onbin_t"])
    assert np.array_equal(np.stack([c[2] for c in calls]), z[tag + "_onbin_counts"])
    assert res.counts.dtype == np.int64 and np.array_equal(res.counts, z[tag + "_counts"])
    assert res.bins.dtype == np.int16 and np.array_equal(res.bins, z[tag + "_bins"])
    assert res.n_bins == z[tag + "_bins"].shape[0]
    assert res.meta()["total_spikes"] == int(z[tag + "_counts"].sum())


def test_run_without_callbacks_matches_reference(golden):
    """Without on_bin/should_stop the run takes whole 20-step blocks across
    bin edges; bins and counts are the same."""
    from fis import sim

    z = golden("run_b2")
    sc, conn, stims, neurons, cfg = run_inputs("run_b2")
    res = sim.run(stims, silenced=S.silenced(sc), config=cfg, neurons=neurons, weights=conn,
                  progress=False)
    assert np.array_equal(res.counts, z["full_counts"])
    assert np.array_equal(res.bins, z["full_bins"])
    tl = res.region_timeline()
    assert list(tl.index) == ["AL", "MB", "LH", "CX"] and tl.shape == (4, res.n_bins)


def test_run_reads_the_flywire_folder(monkeypatch, tmp_path):
    """run(weights=None) loads the connectome the way build_engine does."""
    from fis import connectome as C
    from fis import sim

    conn = C.synthetic(n=1200, e=1200 * 60, seed=3, cache=False)
    seen = []
    monkeypatch.setenv("FIS_FLYWIRE_DATA", str(tmp_path))
    monkeypatch.setattr(C, "from_upstream", lambda d, cache=True: seen.append(d) or conn)
    stim = sim.Stimulus(indices=np.arange(0, 1200, 7), rate_hz=150.0)
    res = sim.run([stim], config=sim.RunConfig(t_run_s=0.01, device="cuda"), progress=False)
    assert seen == [str(tmp_path)] and res.counts.shape == (1200,)


@pytest.mark.parametrize("name", sorted(S.SNAPSHOTS))
def test_restore_reference_snapshot_continues_as_reference(name, golden):
    from fis import sim

    z = golden(name)
    snap = dict(golden("%s_snap%d" % (name, S.SNAPSHOTS[name])))
    at = S.SNAPSHOTS[name]
    sc = S.SCENARIOS[name]
    conn = S.connectome(sc)
    eng = sim.build_engine(weights=conn, silenced=S.silenced(sc), params=sc["params"],
                           batch=sc["batch"], seed=sc["seed"], no_refractory=S.driven(sc),
                           graphs=False)
    with pytest.raises(ValueError):
        eng.restore(snap)  # torch's generator state cannot seed the Philox drive
    done = eng.restore(snap, drop=("gen",))
    assert set(done) >= set(sim.Engine.STATE_TENSORS) | {"ptr"}
    assert int(eng.ptr) == int(snap["ptr"])
    assert np.array_equal(eng.delay_buffer.cpu().numpy(), snap["delay_buffer"])
    for mask in sim.Engine.MASK_TENSORS:
        assert np.array_equal(getattr(eng, mask).cpu().numpy(), snap[mask]), mask
    rates = S.rates_matrix(sc)
    seeds = np.full(sc["batch"], sc["seed"], dtype=np.uint64)
    streams = np.arange(sc["batch"], dtype=np.uint32)
    plan = dict(sc["plan"])
    idx = S.busy(sc)
    rows = []
    for step in range(at, sc["steps"]):
        if step in plan:
            eng.set_masks(**S.mask_call(plan[step], idx))
        tape = O.drive_tape(rates, seeds, streams, np.full(sc["batch"], step), sc["params"])
        sp = eng._core(torch.from_numpy(tape).cuda())
        rows.append(np.packbits(sp.cpu().numpy() != 0, axis=1, bitorder="little"))
    assert np.array_equal(np.stack(rows), z["raster_bits"][at:])
    for key, got in (("v", eng.v), ("g", eng.conductance), ("refrac", eng.refrac),
                     ("spikes", eng.spikes), ("ring", eng.delay_buffer)):
        assert np.array_equal(got.cpu().numpy(), z[key]), key
    assert int(eng.ptr) == int(z["ptr"])
