"""The graded-spike mode (Engine(graded=True)) against the reference, bit for bit.

A caller that writes fractional values into ``Engine.spikes`` between steps
(visdyn.py:660-676) gets the reference's float path: the csrmv product of the
spikes as written (sim.py:910-913) and the refractory update with them
(sim.py:921).  The golden fixture ``graded_b2`` was made by the reference's
own engine with the same writes before every step.
"""

import numpy as np
import pytest
import torch

import scenarios as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def bits(a):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    return np.ascontiguousarray(a).view(np.uint32)


def graded_engine(name, **kw):
    from fis import sim

    sc = S.SCENARIOS[name]
    conn = S.connectome(sc)
    eng = sim.build_engine(weights=conn, silenced=S.silenced(sc), params=sc["params"],
                           batch=sc["batch"], seed=sc["seed"], no_refractory=S.driven(sc),
                           graded=True, **kw)
    return sc, eng


def write_graded(eng, sc, step):
    gs = S.graded_spikes(sc, step)
    if gs is not None:
        eng.spikes[:, torch.from_numpy(gs[0]).cuda()] = torch.from_numpy(gs[1]).cuda()


@pytest.mark.parametrize("drive", ["philox", "tape"])
def test_graded_mode_matches_reference(drive, golden):
    z = golden("graded_b2")
    sc, eng = graded_engine("graded_b2")
    assert eng.use_graphs() is False
    rates = S.rates_matrix(sc)
    rt = torch.from_numpy(rates).cuda()
    seeds = np.full(sc["batch"], sc["seed"], dtype=np.uint64)
    streams = np.arange(sc["batch"], dtype=np.uint32)
    plan = dict(sc["plan"])
    idx = S.busy(sc)
    rows = []
    for step in range(sc["steps"]):
        if step in plan:
            eng.set_masks(**S.mask_call(plan[step], idx))
        write_graded(eng, sc, step)
        if drive == "philox":
            sp = eng.step(rt)
        else:
            tape = O.drive_tape(rates, seeds, streams, np.full(sc["batch"], step), sc["params"])
            sp = eng._core(torch.from_numpy(tape).cuda())
        rows.append(np.packbits(sp.cpu().numpy() != 0, axis=1, bitorder="little"))
    assert np.array_equal(np.stack(rows), z["raster_bits"])
    for key, got in (("v", eng.v), ("g", eng.conductance), ("refrac", eng.refrac),
                     ("spikes", eng.spikes), ("ring", eng.delay_buffer)):
        assert np.array_equal(bits(got), bits(z[key])), key
    assert int(eng.ptr) == int(z["ptr"])


def test_graded_mode_equals_the_exact_engine_on_whole_spikes():
    """Without fractional writes both paths compute the same integer sums."""
    from fis import sim

    name = "batch3_masks"
    sc = S.SCENARIOS[name]
    conn = S.connectome(sc)
    kw = dict(params=sc["params"], batch=sc["batch"], seed=sc["seed"],
              no_refractory=S.driven(sc), graphs=False)
    a = sim.build_engine(weights=conn, graded=True, **kw)
    b = sim.build_engine(weights=conn, **kw)
    rates = torch.from_numpy(S.rates_matrix(sc)).cuda()
    plan = dict(sc["plan"])
    idx = S.busy(sc)
    for step in range(sc["steps"]):
        if step in plan:
            a.set_masks(**S.mask_call(plan[step], idx))
            b.set_masks(**S.mask_call(plan[step], idx))
        assert torch.equal(a.step(rates), b.step(rates)), step
    for x, y in ((a.v, b.v), (a.conductance, b.conductance), (a.refrac, b.refrac)):
        assert np.array_equal(bits(x), bits(y))
    assert np.array_equal(bits(a.delay_buffer), bits(b.delay_buffer))
    assert a.ptr == b.ptr


def test_graded_snapshot_restore_and_run_block():
    """Snapshot with fractional spikes pending, restore into a fresh graded
    engine, and continue (step by step and by run_block): the same bits."""
    sc, a = graded_engine("graded_b2", graphs=False)
    rt = torch.from_numpy(S.rates_matrix(sc)).cuda()
    for step in range(70):
        write_graded(a, sc, step)
        a.step(rt)
    write_graded(a, sc, 70)
    snap = a.snapshot()
    assert np.any((snap["spikes"] != 0) & (snap["spikes"] != 1))
    _, b = graded_engine("graded_b2", graphs=False)
    b.restore(snap)
    acc = torch.zeros_like(a.spikes)
    for _ in range(45):
        acc += a.step(rt)
    got = b.run_block(rt, 45)
    assert torch.equal(acc, got)
    for name in ("v", "conductance", "refrac", "spikes", "delay_buffer"):
        assert np.array_equal(bits(getattr(a, name)), bits(getattr(b, name))), name
    assert a.ptr == b.ptr


def test_exact_engine_still_refuses_graded_writes():
    from fis import sim

    sc = S.SCENARIOS["small_b1"]
    eng = sim.build_engine(weights=S.connectome(sc), batch=1, seed=1, graphs=False)
    rates = torch.from_numpy(S.rates_matrix(sc)).cuda()
    eng.step(rates)
    eng.spikes[0, :5] = 0.5
    with pytest.raises(RuntimeError, match="graded=True"):
        eng.step(rates)
