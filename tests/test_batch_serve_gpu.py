"""Batched trials and the serving loop, checked trial by trial against the oracle.

Each trial of a batch has its own seed, stimulus set, rate, silencing, masks
and duration; each must equal the same trial simulated alone by the oracle
(bit for bit), whatever else shares the GPU, whenever it starts.
"""

import copy

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

N, E = 3000, 3000 * 109


def conn():
    import fis.connectome as C

    return C.synthetic(n=N, e=E, seed=11)


def specs(seed, count, steps):
    from fis.batch import random_specs

    return random_specs(N, count, seed, steps, stim_range=(200, 600), silenced_range=(1, 40))


def oracle_trial(c, spec, steps=None):
    """The reference semantics of one trial: silencing removes rows and columns."""
    steps = spec.steps if steps is None else steps
    cc = c.without(spec.silenced)
    o = O.Oracle.from_connectome(cc, batch=1, no_refractory=spec.stim, seed=spec.seed,
                                 streams=[0])
    r = np.asarray(spec.rate_hz, dtype=np.float64)
    o.rates[0, np.asarray(spec.stim)] = r.astype(np.float32)
    o.set_masks(fire=spec.fire_off if spec.fire_off is not None else None,
                out=spec.out_off if spec.out_off is not None else None,
                inc=spec.in_off if spec.in_off is not None else None,
                hold=spec.hold if spec.hold is not None else None,
                v_clamp=spec.v_clamp)
    raster = o.run(steps, raster=True)
    counts = np.unpackbits(raster[:, 0], axis=1, bitorder="little")[:, :N].sum(0)
    return o, counts


def test_batch_trials_match_oracle():
    from fis.batch import Batch

    c = conn()
    sp = specs(3, 5, 260)
    sp[0].steps = 61             # uneven durations: retired in place mid-block,
    sp[1].steps = 137            # and the last trial group dropped once it ends
    sp[2].fire_off = sp[2].stim[:20]
    sp[3].hold, sp[3].v_clamp = np.arange(100, 160), -60.5
    sp[4].out_off, sp[4].in_off = sp[4].stim[20:60], np.arange(500, 700)
    b = Batch(c, 5, group=2)
    counts = b.run(sp)
    for j, s in enumerate(sp):
        o, want = oracle_trial(c, s)
        assert np.array_equal(counts[j], want), j
        core, slot = b.core, b.slots_of_run[j]
        assert np.array_equal(core.v[slot].cpu().numpy(), o.v[0]), j
        assert np.array_equal(core.g[slot].cpu().numpy(), o.conductance[0]), j
        assert np.array_equal(core.refrac[slot].cpu().numpy(), o.refrac[0]), j


def test_request_same_alone_and_in_mix():
    from fis.serve import Request, Server

    c = conn()
    target = Request(trials=specs(21, 3, 300), bin_steps=50)
    alone = Server(c, capacity=8, group=4).run([copy.deepcopy(target)], realtime=False)
    assert len(alone) == 1
    # In the mix it waits for slots, starts later, lands in other slots and
    # shares every launch with other requests of other lengths.
    mix = [Request(trials=specs(31, 6, 240), bin_steps=40),
           copy.deepcopy(target),
           Request(trials=specs(41, 2, 500), bin_steps=100),
           Request(trials=specs(51, 1, 77), bin_steps=7)]
    replies = Server(c, capacity=8, group=4).run(mix, realtime=False)
    got = {r.rid: r for r in replies}
    t_mix = got[1]
    assert t_mix.admitted >= got[0].released  # it waited for request 0's slots
    assert np.array_equal(t_mix.counts, alone[0].counts)
    assert np.array_equal(t_mix.bins, alone[0].bins)
    # and against the oracle, trial by trial summed
    want = sum(oracle_trial(c, s)[1] for s in target.trials)
    assert np.array_equal(t_mix.counts, want)


def test_server_latency_stats_and_budget():
    from fis.serve import Request, Server

    c = conn()
    srv = Server(c, capacity=4, group=4, memory_budget=4 * N * 4 * 10)
    big = Request(trials=specs(5, 1, 1000), bin_steps=1)   # 1000 bins > budget
    with pytest.raises(MemoryError):
        srv.submit(big)
    reps = srv.run([Request(trials=specs(6, 2, 120), bin_steps=60, arrival=0.0),
                    Request(trials=specs(7, 3, 100), bin_steps=50, arrival=0.01)],
                   realtime=True)
    st = Server.latency_stats(reps)
    assert st["n"] == 2 and st["p99_s"] >= st["p50_s"] > 0


@pytest.mark.parametrize("ring", ["int16", "int32"])
@pytest.mark.parametrize("scatter_mode", [0, 1])
@pytest.mark.parametrize("update_streams,group", [(1, 2), (2, 2), (2, 3)])
@pytest.mark.parametrize("update_tiles", [1, 2])
def test_overlapped_advance_equals_sequential(ring, scatter_mode, update_streams, group,
                                              update_tiles):
    """Scatter/update overlap on two rings (updates on one or two streams,
    an even and an odd number of trial groups) gives the one-ring result, bit
    for bit."""
    from fis.batch import Batch
    from fis.engine import Core

    c = conn()
    sp = specs(61, 7, (150, 300))   # uneven: trial groups drop out as they end
    got = []
    for overlap in (False, True):
        core = Core(c, 7, group=group, ring=ring, overlap=overlap, scatter_mode=scatter_mode,
                    update_streams=update_streams, update_tiles=update_tiles)
        counts = Batch(c, 7, core=core).run(sp)
        got.append((counts, core.v.cpu().numpy(), core.g.cpu().numpy(),
                    core.refrac.cpu().numpy(), core.step))
    for a, b in zip(got[0], got[1]):
        assert np.array_equal(a, b)
    s = sp[3]
    assert np.array_equal(got[1][0][3], oracle_trial(c, s)[1])


@pytest.mark.parametrize("tiles", [1, 2])
def test_bounded_wait_reports_error_and_context_survives(tiles):
    """A staging wait that runs out sets an error bit the host raises on; the
    CUDA context stays usable and a fresh batch is exact again (one tile per
    update CTA, and the streamed tiles)."""
    from fis.batch import Batch

    c = conn()
    sp = specs(71, 2, 40)
    b = Batch(c, 2, group=2, update_tiles=tiles)
    b.core.desc.wait_polls = 2000
    b.core.desc.inject_stall = 1    # no staging copy is issued: every wait runs out
    with pytest.raises(RuntimeError, match="error bits"):
        b.run(sp)
    torch.cuda.synchronize()
    fresh = Batch(c, 2, group=2).run(sp)
    for j, s in enumerate(sp):
        assert np.array_equal(fresh[j], oracle_trial(c, s)[1]), j
    # the batch that saw the error is usable again: raising refilled its
    # rings, which the CTAs that gave up had left as the scatter wrote them
    b.core.desc.inject_stall = 0
    b.core.desc.wait_polls = 0
    again = b.run(sp)
    for j, s in enumerate(sp):
        assert np.array_equal(again[j], oracle_trial(c, s)[1]), j


def test_last_step_raster_mode_keeps_state_and_last_spikes():
    """raster=False (only each block's last step kept) changes nothing else."""
    from fis.batch import Batch
    from fis.engine import Core

    c = conn()
    sp = specs(81, 4, (90, 140))
    got = []
    for raster in (True, False):
        core = Core(c, 4, group=2, raster=raster)
        counts = Batch(c, 4, core=core).run(sp)
        last = core.spikes_at().cpu().numpy()
        got.append((counts, core.v.cpu().numpy(), core.g.cpu().numpy(),
                    core.refrac.cpu().numpy(), last))
        if not raster:
            with pytest.raises(ValueError):
                core.spikes_at(core.step - 2)
    for a, b in zip(got[0], got[1]):
        assert np.array_equal(a, b)


def test_run_many_equals_run():
    """The pipelined run_many gives each batch exactly what run gives it."""
    from fis.batch import Batch

    c = conn()
    batches = [specs(91, 3, (40, 120)), specs(92, 4, 60), specs(93, 2, (20, 90))]
    want = [Batch(c, 4, group=2).run(sp) for sp in batches]
    got = list(Batch(c, 4, group=2).run_many(batches))
    assert len(got) == len(want)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


def test_run_many_on_a_side_stream():
    """run_many enqueues on the caller's stream from its worker thread."""
    import torch

    from fis.batch import Batch

    c = conn()
    batches = [specs(94, 3, (40, 120)), specs(95, 4, 60), specs(96, 4, (20, 90)),
               specs(97, 1, 80)]
    want = [Batch(c, 4, group=2).run(sp) for sp in batches]
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        b = Batch(c, 4, group=2)
        got = list(b.run_many(iter(batches)))
    torch.cuda.synchronize()
    assert len(got) == len(want)
    for a, w in zip(got, want):
        assert np.array_equal(a, w)


def test_run_many_raises_a_batch_error_when_its_counts_are_due():
    """run_many reads each batch's error bits with its counts (copied in stream
    order, no host wait): a batch whose staging waits ran out raises at its
    yield, with the next batch already enqueued; the context stays usable."""
    from fis.batch import Batch

    c = conn()
    sp = specs(72, 2, 40)
    b = Batch(c, 2, group=2)
    b.core.desc.wait_polls = 2000
    b.core.desc.inject_stall = 1    # no staging copy is issued: every wait runs out
    it = b.run_many([sp, sp])
    with pytest.raises(RuntimeError, match="error bits"):
        next(it)
    torch.cuda.synchronize()
    fresh = Batch(c, 2, group=2).run(sp)
    for j, s in enumerate(sp):
        assert np.array_equal(fresh[j], oracle_trial(c, s)[1]), j


@pytest.mark.parametrize("group", [3, 8])
def test_drive_lists_equal_the_full_scan(group):
    """Phase A's drive over each trial's list of stimulated neurons (what
    Batch gives it) draws exactly what the scan over every rate draws: the
    same counts and the same final state, trial for trial, in a mix of
    uneven durations whose trials are reloaded into freed slots."""
    from fis.batch import Batch

    c = conn()
    first = specs(91, 7, (60, 140))
    second = specs(92, 3, (50, 90))
    got = []
    for lists in (False, True):
        b = Batch(c, 7, group=group, drive_lists=lists)
        counts = [b.run(first), b.run(second)]
        core = b.core
        got.append((counts, core.v.cpu().numpy(), core.g.cpu().numpy(),
                    core.refrac.cpu().numpy()))
        if lists:
            # the lists hold the stimulated neurons of the last load
            for j, s in enumerate(second):
                slot = b.slots_of_run[j]
                k = int(core.drive_len[slot])
                assert sorted(core.drive_idx[slot, :k].tolist()) == sorted(set(int(x) for x in s.stim))
    (ca, va, ga, ra), (cb, vb, gb, rb) = got
    for x, y in zip(ca, cb):
        for u, w in zip(x, y):
            assert np.array_equal(u, w)
    assert np.array_equal(va, vb) and np.array_equal(ga, gb) and np.array_equal(ra, rb)
    for j, s in enumerate(second):
        assert np.array_equal(cb[1][j], oracle_trial(c, s)[1]), j


def test_tuner_runoff_and_tuned_launch_is_exact():
    """The autotuner on a small connectome: it times its candidates, runs the
    fastest three again (the runoff that picks the winner), and the launch it
    returns gives the same counts as the oracle, trial for trial."""
    from fis.batch import Batch
    from fis.tune import core_kwargs, tune

    c = conn()
    sp = specs(95, 8, 60)
    best = tune(c, 8, groups=[2, 4, 8], chunks=[256], grids=[(8, 8)], steps=40, reps=1,
                use_cache=False, specs=sp, tag="test")
    cands = best["candidates"]
    assert len(cands) >= 3
    ran = [r for r in cands if "runoff_ms_per_step" in r]
    assert len(ran) == 3
    assert best["runoff_ms_per_step"] == min(r["runoff_ms_per_step"] for r in ran)
    got = Batch(c, 8, **core_kwargs(best)).run(sp)
    for j, s in enumerate(sp):
        assert np.array_equal(got[j], oracle_trial(c, s)[1]), j
