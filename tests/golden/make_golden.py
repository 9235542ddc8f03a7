"""Generate the golden parity fixtures by running the REFERENCE engine.

Runs only where the reference tree is present (it is read, never copied):

    python tests/golden/make_golden.py [scenario ...]

For every scenario of ``tests/scenarios.py`` (or those named) it builds the reference's own
``sim.Engine`` (``lab/flybrain/sim.py:348``) on CPU with the synthetic
connectome as its weight matrix, silences through the reference's own
``sim._silence`` (``sim.py:324-336``), applies the mask plan through
``Engine.set_masks`` (``sim.py:510``), and steps it with ``Engine._core``
(``sim.py:863``) fed by the shared Philox input tape, the way the
reference's parity probes drive it; a graded scenario first writes its
fractional values into ``Engine.spikes``, as ``visdyn.py:660-676`` does.  It records the spike raster of every step
and fingerprints of the full state at milestones, plus the final state arrays
for the small scenarios, and for the scenarios of ``SNAPSHOTS`` the
reference's own ``Engine.snapshot()`` (``sim.py:780-814``) taken mid-run.
For the scenarios of ``RUN_SCENARIOS`` it runs the reference's experiment
driver ``sim.run`` (``sim.py:990-1117``) with ``Engine._poisson`` replaced
by the same tape, and records the result, every ``on_bin`` call and the
step at which a ``should_stop`` callback ends a second run.  The fixtures
pin the C oracle (CPU tests) and the CUDA engine (GPU tests).
"""

from __future__ import annotations

import hashlib
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF_LAB = Path("/root/reference/lab")
sys.path.insert(0, str(ROOT / "fly-in-silico_b200"))
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT))

import scenarios as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def fp(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def tape_source(sc_seed, params):
    """A stand-in for ``Engine._poisson`` (sim.py:848-861) that returns the
    shared Philox tape of the engine's current step: trial ``b`` draws from
    stream ``b`` keyed by the run's seed, as this engine's ``build_engine``
    seeds its trials."""
    import torch

    def poisson(self, rates):
        r = rates.detach().cpu().numpy()
        B = r.shape[0]
        tape = O.drive_tape(r, np.full(B, sc_seed, np.uint64), np.arange(B, dtype=np.uint32),
                            np.full(B, self.calls - 1, np.int64), params)
        return torch.from_numpy(tape)

    return poisson


def run_sim_run(name):
    """The reference's own ``sim.run`` (sim.py:990-1117) on a run scenario,
    its Poisson draw replaced by the shared tape: the result's counts and
    bins, every ``on_bin`` call, and a second run cut by ``should_stop``."""
    import pandas as pd
    import torch

    sys.path.insert(0, str(REF_LAB))
    from flybrain import sim

    torch.set_num_threads(8)
    sc = S.RUN_SCENARIOS[name]
    conn = S.connectome(sc)
    n = sc["n"]
    W = conn.to_torch_weights()
    sil = S.silenced(sc)
    stims = [sim.Stimulus(indices=idx, rate_hz=rate, t_on_ms=on, t_off_ms=off, name=nm)
             for nm, idx, rate, on, off in S.run_stimuli(sc)]
    neurons = pd.DataFrame({"region": np.array(["AL", "MB", "LH", "CX"])[np.arange(n) % 4]})
    cfg = sim.RunConfig(t_run_s=sc["t_run_s"], bin_ms=sc["bin_ms"], n_trials=sc["batch"],
                        seed=sc["seed"], device="cpu", spmv=sim.SPMV_CSR)
    saved = sim.Engine._poisson
    sim.Engine._poisson = tape_source(sc["seed"], None)
    out = {}
    try:
        for tag, stop_after in (("full", None), ("stop", sc["stop_after_bin"])):
            calls = []
            polls = [0]

            def on_bin(b, t_ms, counts):
                calls.append((b, t_ms, counts.copy()))

            def should_stop():
                polls[0] += 1
                return stop_after is not None and polls[0] > stop_after

            t0 = time.time()
            res = sim.run(stims, silenced=sil, config=cfg, neurons=neurons, weights=W,
                          progress=False, on_bin=on_bin, should_stop=should_stop)
            out.update({
                tag + "_counts": res.counts.astype(np.int64),
                tag + "_bins": res.bins.astype(np.int16),
                tag + "_steps": np.int64(res.timing["steps"]),
                tag + "_onbin_b": np.array([c[0] for c in calls], dtype=np.int64),
                tag + "_onbin_t": np.array([c[1] for c in calls], dtype=np.float64),
                tag + "_onbin_counts": np.stack([c[2] for c in calls]).astype(np.int16),
            })
            print("%-8s %-4s %4d steps, %6d spikes, %d bins reported, %.1f s"
                  % (name, tag, int(res.timing["steps"]), int(res.counts.sum()), len(calls),
                     time.time() - t0))
    finally:
        sim.Engine._poisson = saved
    path = OUT / ("%s.npz" % name)
    np.savez_compressed(path, **out)
    print("-> %s (%d KB)" % (path.name, path.stat().st_size // 1024))


def run_reference(name):
    import torch

    sys.path.insert(0, str(REF_LAB))
    from flybrain import sim

    torch.set_num_threads(8)
    sc = S.SCENARIOS[name]
    conn = S.connectome(sc)
    n, B = sc["n"], sc["batch"]
    W = conn.to_torch_weights()
    sil = S.silenced(sc)
    if sil.size:
        W = sim._silence(W, sil, n)
    drv = S.driven(sc)
    eng = sim.Engine(W, n, params=sc["params"], device="cpu", batch=B,
                     seed=sc["seed"], no_refractory=drv, spmv=sim.SPMV_CSR)
    rates = S.rates_matrix(sc)
    seeds = np.full(B, sc["seed"], dtype=np.uint64)
    streams = np.arange(B, dtype=np.uint32)
    plan = dict(sc["plan"])
    idx = S.busy(sc)
    nbytes = (n + 7) // 8
    raster = np.zeros((sc["steps"], B, nbytes), dtype=np.uint8)
    marks = {}
    t0 = time.time()
    snap_at = S.SNAPSHOTS.get(name)
    snap = None
    for step in range(sc["steps"]):
        if step == snap_at:
            snap = eng.snapshot()
        what = plan.get(step)
        if what is not None:
            eng.set_masks(**S.mask_call(what, idx))
        gs = S.graded_spikes(sc, step)
        if gs is not None:
            eng.spikes[:, torch.from_numpy(gs[0])] = torch.from_numpy(gs[1])
        tape = O.drive_tape(rates, seeds, streams, np.full(B, step, np.int64),
                            sc["params"])
        sp = eng._core(torch.from_numpy(tape)).numpy()
        raster[step] = np.packbits(sp != 0, axis=1, bitorder="little")
        if step + 1 in S.MILESTONES or step + 1 == sc["steps"]:
            marks[step + 1] = {
                "v": fp(eng.v.numpy()), "g": fp(eng.conductance.numpy()),
                "refrac": fp(eng.refrac.numpy()), "spikes": fp(eng.spikes.numpy()),
                "ring": fp(eng.delay_buffer.numpy()), "ptr": int(eng.ptr),
            }
    wall = time.time() - t0
    out = {
        "raster_bits": raster,
        "marks_steps": np.array(sorted(marks), dtype=np.int64),
        "marks": np.array([[marks[k][f] for f in ("v", "g", "refrac", "spikes", "ring")]
                           for k in sorted(marks)]),
        "marks_ptr": np.array([marks[k]["ptr"] for k in sorted(marks)], dtype=np.int64),
        "total_spikes": np.int64(int(np.unpackbits(raster, bitorder="little").sum())),
        "ref_ms_per_step": np.float64(wall * 1000.0 / sc["steps"]),
    }
    if n <= 5000:
        out.update(v=eng.v.numpy(), g=eng.conductance.numpy(), refrac=eng.refrac.numpy(),
                   spikes=eng.spikes.numpy(), ring=eng.delay_buffer.numpy(),
                   ptr=np.int64(eng.ptr))
    else:
        # full size: the raster as (step, trial, neuron) triples (it is sparse),
        # the first 1,000 steps of it for long runs, plus per-neuron counts
        bits = np.unpackbits(raster, axis=2, bitorder="little")[:, :, :n]
        st, b, i = np.nonzero(bits[:1000])
        out.pop("raster_bits")
        out.update(spike_step=st.astype(np.int32), spike_trial=b.astype(np.int16),
                   spike_neuron=i.astype(np.int32),
                   counts=bits.sum(0).astype(np.int32))
    if snap is not None:
        # the reference's own snapshot, every key as it wrote it (gen is
        # its torch generator state, which this engine refuses by design)
        spath = OUT / ("%s_snap%d.npz" % (name, snap_at))
        np.savez_compressed(spath, **snap)
        print("%-14s snapshot at step %d -> %s" % (name, snap_at, spath.name))
    path = OUT / ("%s.npz" % name)
    np.savez_compressed(path, **out)
    print("%-14s %5d steps, %6d spikes, reference %.1f ms/step -> %s (%d KB)"
          % (name, sc["steps"], int(out["total_spikes"]), wall * 1000 / sc["steps"],
             path.name, path.stat().st_size // 1024))


def main(argv):
    names = argv or list(S.SCENARIOS) + list(S.RUN_SCENARIOS)
    O.build()
    for name in names:
        if name in S.RUN_SCENARIOS:
            run_sim_run(name)
        else:
            run_reference(name)


if __name__ == "__main__":
    main(sys.argv[1:])
