"""The oracle against the reference's own outputs (tests/golden).

The fixtures were produced by running the reference's ``sim.Engine`` on CPU
(``tests/golden/make_golden.py``); these tests pin the C oracle to them, bit
for bit, in both of the reference's recurrent-product algorithms.
"""

import numpy as np
import pytest

import scenarios as S
from oracle import oracle as O

SMALL = ["small_b1", "batch3_masks", "silenced_b2", "alt_params"]


def test_philox_known_answers():
    # Random123 philox4x32-10 known-answer vectors (ctr, key -> out).
    kat = [
        ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for ctr, key, want in kat:
        assert list(O.philox4x32_10(ctr, key)) == want


def run_oracle(name, mode, tape=False):
    sc = S.SCENARIOS[name]
    conn = S.connectome(sc)
    sil = S.silenced(sc)
    if sil.size:
        conn = conn.without(sil)
    o = O.Oracle.from_connectome(conn, batch=sc["batch"], params_dict=sc["params"],
                                 no_refractory=S.driven(sc), seed=sc["seed"])
    o.rates[:] = S.rates_matrix(sc)
    plan = dict(sc["plan"])
    idx = S.busy(sc)
    rows = []
    marks = {}
    for step in range(sc["steps"]):
        if step in plan:
            o.set_masks(**S.mask_call(plan[step], idx))
        gs = S.graded_spikes(sc, step)
        if gs is not None:
            o.spikes[:, gs[0]] = gs[1]
        if tape:
            vs = O.drive_tape(o.rates, o.seeds, o.streams, np.full(sc["batch"], step),
                              sc["params"])
            o.core(vs, mode=mode)
            rows.append(np.packbits(o.spikes != 0, axis=1, bitorder="little"))
        else:
            rows.append(o.run(1, mode=mode, raster=True)[0])
        if step + 1 in S.MILESTONES or step + 1 == sc["steps"]:
            marks[step + 1] = [O.fingerprint(a) for a in
                               (o.v, o.conductance, o.refrac, o.spikes, o.delay_buffer)]
    return o, np.stack(rows), marks


@pytest.mark.parametrize("name", SMALL)
@pytest.mark.parametrize("mode", [O.Oracle.EVENT, O.Oracle.CSRMV])
def test_oracle_matches_reference(name, mode, golden):
    z = golden(name)
    o, raster, marks = run_oracle(name, mode)
    assert np.array_equal(raster, z["raster_bits"])
    for key, got in (("v", o.v), ("g", o.conductance), ("refrac", o.refrac),
                     ("spikes", o.spikes), ("ring", o.delay_buffer)):
        assert np.array_equal(got, z[key]), key
    assert int(o.ptr[0]) == int(z["ptr"])
    for k, fps in zip(z["marks_steps"], z["marks"]):
        assert marks[int(k)] == list(fps), int(k)


def test_oracle_graded_spikes_match_reference(golden):
    """Fractional values written into the spike state before every step
    (visdyn.py:660-676) reach the reference's csrmv product and refractory
    update; the oracle's fused, ascending-column accumulation gives the
    reference's bits, signed zeros included."""
    z = golden("graded_b2")
    o, raster, marks = run_oracle("graded_b2", O.Oracle.CSRMV)
    assert np.array_equal(raster, z["raster_bits"])
    for key, got in (("v", o.v), ("g", o.conductance), ("refrac", o.refrac),
                     ("spikes", o.spikes), ("ring", o.delay_buffer)):
        assert np.array_equal(np.ascontiguousarray(got).view(np.uint32),
                              np.ascontiguousarray(z[key]).view(np.uint32)), key
    assert int(o.ptr[0]) == int(z["ptr"])
    for k, fps in zip(z["marks_steps"], z["marks"]):
        assert marks[int(k)] == list(fps), int(k)
    # the graded values reached the state: (r + 1) * (1 - s) with a
    # fractional s leaves fractional refractory counts
    assert np.any(z["refrac"] != np.round(z["refrac"]))


def test_oracle_tape_path_matches(golden):
    """Driving ``core`` with the explicit tape equals the built-in drive."""
    z = golden("batch3_masks")
    _, raster, _ = run_oracle("batch3_masks", O.Oracle.EVENT, tape=True)
    assert np.array_equal(raster, z["raster_bits"])


def test_oracle_full_size_config0(golden):
    """1,000 steps of the full 138,639-neuron connectome, raster and fingerprints."""
    z = golden("full_cfg0")
    sc = S.SCENARIOS["full_cfg0"]
    conn = S.connectome(sc)
    o = O.Oracle.from_connectome(conn, batch=1, no_refractory=S.driven(sc), seed=sc["seed"])
    o.rates[:] = S.rates_matrix(sc)
    raster = o.run(sc["steps"], mode=O.Oracle.EVENT, raster=True)
    st, b, i = np.nonzero(np.unpackbits(raster, axis=2, bitorder="little")[:, :, :sc["n"]])
    assert np.array_equal(st, z["spike_step"])
    assert np.array_equal(i, z["spike_neuron"])
    last = z["marks"][-1]
    assert [O.fingerprint(a) for a in (o.v, o.conductance, o.refrac, o.spikes,
                                       o.delay_buffer)] == list(last)


def test_oracle_catches_planted_mistakes(golden):
    """The comparison can fail: three mistakes planted in the oracle are caught.

    The reference's own forgeries (lab/probe/lif_event.py:301-412): one synapse
    count of a spiking row off by one, an all-ones m_out under an ``out``
    mask, and the ring pointer shifted by one slot.
    """
    name = "batch3_masks"
    z = golden(name)
    sc = S.SCENARIOS[name]
    ref = z["raster_bits"]

    def diverges(spoil):
        conn = S.connectome(sc)
        o = O.Oracle.from_connectome(conn, batch=sc["batch"], no_refractory=S.driven(sc),
                                     seed=sc["seed"])
        o.rates[:] = S.rates_matrix(sc)
        plan = dict(sc["plan"])
        idx = S.busy(sc)
        first = None
        for step in range(sc["steps"]):
            if step in plan:
                o.set_masks(**S.mask_call(plan[step], idx))
            spoil(o, step)
            row = o.run(1, raster=True)[0]
            if first is None and not np.array_equal(row, ref[step]):
                first = step
        state_differs = not (np.array_equal(o.v, z["v"]) and
                             np.array_equal(o.conductance, z["g"]))
        return first if first is not None else ("state" if state_differs else None)

    hot = int(S.driven(sc)[0])
    conn0 = S.connectome(sc)
    k = int(conn0.row_ptr[hot])

    def one_count(o, step):
        if step == 0:
            o.cnt[k] += 1  # the row of a driven (spiking) neuron

    def ones_mask(o, step):
        if 130 <= step < 170:
            o.m_out[:] = 1.0  # ignore the ``out`` intervention

    def ring_shift(o, step):
        if step == 50:
            o.ptr[0] = (o.ptr[0] + 1) % o.buf_len

    assert diverges(one_count) is not None
    assert diverges(ones_mask) is not None
    assert diverges(ring_shift) is not None


def oracle_sim_run(name, stop_after=None):
    """The experiment driver of sim.py:990-1083 over the oracle's step: the
    rate schedule, int16 bins summed over trials, the on_bin stream and the
    should_stop cut, written out here from the reference's description."""
    sc = S.RUN_SCENARIOS[name]
    conn = S.connectome(sc).without(S.silenced(sc))
    stims = S.run_stimuli(sc)
    steps = int(round(sc["t_run_s"] * 1000.0 / O.DT))
    bin_steps = max(1, int(round(sc["bin_ms"] / O.DT)))
    n_bins = -(-steps // bin_steps)
    switches = []
    for _, idx, rate, on, off in stims:
        switches.append((int(round(on / O.DT)), idx, rate))
        stop = steps if off is None else int(round(off / O.DT))
        if stop < steps:
            switches.append((stop, idx, 0.0))
    switches.sort(key=lambda e: e[0])
    o = O.Oracle.from_connectome(conn, batch=sc["batch"], seed=sc["seed"],
                                 no_refractory=np.concatenate([s[1] for s in switches]))
    bins = np.zeros((n_bins, sc["n"]), dtype=np.int64)
    calls = []
    polls = 0
    for step in range(steps):
        for at, idx, rate in switches:
            if at == step:
                o.rates[:, idx] = rate
        vs = O.drive_tape(o.rates, o.seeds, o.streams, np.full(sc["batch"], step))
        o.core(vs, mode=O.Oracle.CSRMV)
        b = step // bin_steps
        bins[b] += o.spikes.sum(0).astype(np.int64)
        if (step + 1) % bin_steps == 0 or step == steps - 1:
            calls.append((b, (step + 1) * O.DT, bins[b].astype(np.int16)))
            polls += 1
            if stop_after is not None and polls > stop_after:
                steps = step + 1
                break
    return bins, calls, steps


@pytest.mark.parametrize("tag", ["full", "stop"])
def test_oracle_sim_run_matches_reference(tag, golden):
    """The run golden (the reference's own sim.run on the tape) against the
    oracle stepping the same schedule: pins the fixture's drive convention
    (one Philox stream per trial, keyed by the run seed, own step = call)."""
    z = golden("run_b2")
    sc = S.RUN_SCENARIOS["run_b2"]
    bins, calls, steps = oracle_sim_run("run_b2", sc["stop_after_bin"] if tag == "stop" else None)
    assert steps == int(z[tag + "_steps"])
    assert np.array_equal(bins.astype(np.int16), z[tag + "_bins"])
    assert np.array_equal(bins.sum(0), z[tag + "_counts"])
    assert [c[0] for c in calls] == list(z[tag + "_onbin_b"])
    assert [c[1] for c in calls] == list(z[tag + "_onbin_t"])
    assert np.array_equal(np.stack([c[2] for c in calls]), z[tag + "_onbin_counts"])


@pytest.mark.parametrize("name", sorted(S.SNAPSHOTS))
def test_reference_snapshot_continues_in_oracle(name, golden):
    """The reference's mid-run snapshot, put into the oracle's state, continues
    to the reference's final raster and state."""
    z = golden(name)
    at = S.SNAPSHOTS[name]
    snap = golden("%s_snap%d" % (name, at))
    sc = S.SCENARIOS[name]
    conn = S.connectome(sc)
    sil = S.silenced(sc)
    if sil.size:
        conn = conn.without(sil)
    o = O.Oracle.from_connectome(conn, batch=sc["batch"], params_dict=sc["params"],
                                 no_refractory=S.driven(sc), seed=sc["seed"])
    o.rates[:] = S.rates_matrix(sc)
    for key in ("v", "conductance", "spikes", "refrac", "delay_buffer", "m_fire", "m_out",
                "m_in", "m_hold", "v_hold"):
        getattr(o, key)[...] = snap[key]
    o.ptr[0] = int(snap["ptr"])
    plan = dict(sc["plan"])
    idx = S.busy(sc)
    rows = []
    for step in range(at, sc["steps"]):
        if step in plan:
            o.set_masks(**S.mask_call(plan[step], idx))
        vs = O.drive_tape(o.rates, o.seeds, o.streams, np.full(sc["batch"], step), sc["params"])
        o.core(vs, mode=O.Oracle.EVENT)
        rows.append(np.packbits(o.spikes != 0, axis=1, bitorder="little"))
    assert np.array_equal(np.stack(rows), z["raster_bits"][at:])
    assert np.array_equal(o.v, z["v"]) and np.array_equal(o.delay_buffer, z["ring"])
