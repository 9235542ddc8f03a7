"""The CUDA engine against the reference's outputs and the oracle, bit for bit.

Every test here runs the engine through its C ABI (``libfis_b200.so`` via
``fis``) on the inputs the golden fixtures were made from, and compares
spike rasters and full state with the reference's own results.
"""

import numpy as np
import pytest
import torch

import scenarios as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SMALL = ["small_b1", "batch3_masks", "silenced_b2", "alt_params"]


def raster_rows(core, first, last):
    """Bit rows [step][B][nbytes] of global steps first..last-1 from the engine."""
    nbytes = (core.n + 7) // 8
    out = []
    bits = core.bits.cpu().numpy()  # [B][W][L]
    for s in range(first, last):
        row = np.ascontiguousarray(bits[:, :, s % core.lag]).view(np.uint8)[:, :nbytes]
        out.append(row.copy())
    return out


def make_engine(name, graphs=False, group=None, ring=None, scatter_mode=None, update_tiles=None):
    from fis import sim

    sc = S.SCENARIOS[name]
    conn = S.connectome(sc)
    eng = sim.build_engine(weights=conn, silenced=S.silenced(sc), params=sc["params"],
                           batch=sc["batch"], seed=sc["seed"], no_refractory=S.driven(sc),
                           graphs=graphs, group=group, ring=ring)
    if scatter_mode is not None or update_tiles is not None:
        eng.core.set_launch(scatter_mode, update_tiles=update_tiles)
    return sc, eng


def final_state_equal(eng, z):
    checks = {
        "v": eng.v.cpu().numpy(), "g": eng.conductance.cpu().numpy(),
        "refrac": eng.refrac.cpu().numpy(), "spikes": eng.spikes.cpu().numpy(),
        "ring": eng.delay_buffer.cpu().numpy(),
    }
    bad = [k for k, a in checks.items() if not np.array_equal(a, z[k])]
    if int(eng.ptr) != int(z["ptr"]):
        bad.append("ptr")
    return bad


@pytest.mark.parametrize("name", SMALL)
@pytest.mark.parametrize("graphs", [False, True])
def test_step_api_matches_reference(name, graphs, golden):
    """``Engine.step`` per step, masks between steps, as the reference's probes."""
    z = golden(name)
    sc, eng = make_engine(name, graphs=graphs)
    rates = torch.from_numpy(S.rates_matrix(sc)).cuda()
    plan = dict(sc["plan"])
    idx = S.busy(sc)
    rows = []
    for step in range(sc["steps"]):
        if step in plan:
            eng.set_masks(**S.mask_call(plan[step], idx))
        sp = eng.step(rates)
        rows.append(np.packbits(sp.cpu().numpy() != 0, axis=1, bitorder="little"))
    assert np.array_equal(np.stack(rows), z["raster_bits"])
    assert final_state_equal(eng, z) == []
    assert eng.calls == sc["steps"]


@pytest.mark.parametrize("name", SMALL)
def test_tape_driven_core_matches_reference(name, golden):
    """``Engine._core(voltage_stim)`` with the shared tape (the probes' form)."""
    z = golden(name)
    sc, eng = make_engine(name)
    rates = S.rates_matrix(sc)
    seeds = np.full(sc["batch"], sc["seed"], dtype=np.uint64)
    streams = np.arange(sc["batch"], dtype=np.uint32)
    plan = dict(sc["plan"])
    idx = S.busy(sc)
    rows = []
    for step in range(sc["steps"]):
        if step in plan:
            eng.set_masks(**S.mask_call(plan[step], idx))
        tape = O.drive_tape(rates, seeds, streams, np.full(sc["batch"], step), sc["params"])
        sp = eng._core(torch.from_numpy(tape).cuda())
        rows.append(np.packbits(sp.cpu().numpy() != 0, axis=1, bitorder="little"))
    assert np.array_equal(np.stack(rows), z["raster_bits"])
    assert final_state_equal(eng, z) == []


@pytest.mark.parametrize("name", SMALL)
@pytest.mark.parametrize("group", [None, 1, 2])
@pytest.mark.parametrize("ring", ["int16", "int32"])
@pytest.mark.parametrize("scatter_mode,update_tiles", [(0, 1), (1, 1), (1, 2)])
def test_blocked_stepping_matches_reference(name, group, ring, scatter_mode, update_tiles,
                                            golden):
    """Blocks of up to 20 fused steps, split only where the masks change; both
    scatter forms (a warp per work item, a warp per 32 items) and one or two
    tiles per update CTA."""
    z = golden(name)
    sc, eng = make_engine(name, group=group, ring=ring, scatter_mode=scatter_mode,
                          update_tiles=update_tiles)
    assert eng.core.ring16 == (ring == "int16")
    core = eng.core
    core.rates.copy_(torch.from_numpy(S.rates_matrix(sc)))
    plan = dict(sc["plan"])
    idx = S.busy(sc)
    cuts = sorted(set([s for s in plan] + [sc["steps"]]))
    rows = []
    step = 0
    for cut in cuts:
        if step in plan:
            eng.set_masks(**S.mask_call(plan[step], idx))
        while step < cut:
            k = min(core.max_block, cut - step)
            core.block(k, spikes_out=eng.spikes)
            rows += raster_rows(core, step, step + k)
            step += k
    eng._spikes_version = eng.spikes._version
    assert np.array_equal(np.stack(rows), z["raster_bits"])
    assert final_state_equal(eng, z) == []


@pytest.mark.parametrize("scatter_mode,update_tiles", [(0, 1), (1, 1), (1, 2)])
def test_full_size_config0_matches_reference(scatter_mode, update_tiles, golden):
    """138,639 neurons, 15.09 M edges, 1,000 steps in 20-step blocks."""
    z = golden("full_cfg0")
    sc, eng = make_engine("full_cfg0", scatter_mode=scatter_mode, update_tiles=update_tiles)
    core = eng.core
    core.rates.copy_(torch.from_numpy(S.rates_matrix(sc)))
    rows = []
    for step in range(0, sc["steps"], 20):
        core.block(20, spikes_out=eng.spikes)
        rows += raster_rows(core, step, step + 20)
    bits = np.unpackbits(np.stack(rows), axis=2, bitorder="little")[:, :, :sc["n"]]
    st, b, i = np.nonzero(bits)
    assert np.array_equal(st, z["spike_step"]) and np.array_equal(i, z["spike_neuron"])
    fps = [O.fingerprint(a) for a in (eng.v.cpu().numpy(), eng.conductance.cpu().numpy(),
                                      eng.refrac.cpu().numpy(), eng.spikes.cpu().numpy(),
                                      eng.delay_buffer.cpu().numpy())]
    assert fps == list(z["marks"][-1])


@pytest.mark.parametrize("ring", ["int16", "int32"])
def test_snapshot_restore_continues_bit_exactly(ring):
    """Continue-from-snapshot equals the uninterrupted run (probe/resume_state.py)."""
    name = "batch3_masks"
    sc, a = make_engine(name, ring=ring)
    rates = torch.from_numpy(S.rates_matrix(sc)).cuda()
    idx = S.busy(sc)
    a.set_masks(out=idx[:200], hold=idx[200:300], v_clamp=-60.0)
    for _ in range(137):
        a.step(rates)
    snap = a.snapshot()
    for _ in range(90):
        a.step(rates)
    _, b = make_engine(name, ring=ring)
    b.restore(snap)
    for _ in range(90):
        b.step(rates)
    for name_ in ("v", "conductance", "refrac", "spikes"):
        assert torch.equal(getattr(a, name_), getattr(b, name_)), name_
    assert torch.equal(a.delay_buffer, b.delay_buffer)
    assert a.ptr == b.ptr


def test_restore_drop_one_changes_the_future():
    """Completeness of the state: dropping any element changes what follows."""
    name = "small_b1"
    sc, a = make_engine(name)
    rates = torch.from_numpy(S.rates_matrix(sc)).cuda()
    for _ in range(120):
        a.step(rates)
    snap = a.snapshot()
    for _ in range(60):
        a.step(rates)
    ref = a.v.clone()
    for drop in ("v", "conductance", "refrac", "delay_buffer", "spikes", "ptr"):
        _, b = make_engine(name)
        for _ in range(7):
            b.step(rates)
        b.restore(snap, drop=(drop,))
        for _ in range(60):
            b.step(rates)
        assert not torch.equal(b.v, ref), drop


def test_ev_spmv_dropin_exact():
    """The reference-FFI drop-in equals an exact integer sum."""
    from fis import evspmv

    c = S.connectome(S.SCENARIOS["batch3_masks"])
    w = c.to_torch_weights("cuda").to_sparse_csr()
    B = 3
    ev = evspmv.Events(w, B, "cuda")
    g = torch.Generator(device="cpu").manual_seed(3)
    sp = (torch.rand(B, c.n, generator=g) < 0.05).float().cuda()
    mo = (torch.rand(B, c.n, generator=g) < 0.9).float().cuda()
    out = ev.mm(sp, mo).cpu().numpy()
    x = (sp * mo).cpu().numpy().astype(np.int64)
    pre = np.repeat(np.arange(c.n), c.out_degree())
    want = np.zeros((B, c.n), dtype=np.int64)
    for b in range(B):
        np.add.at(want[b], c.col, c.cnt.astype(np.int64) * x[b, pre])
    assert np.array_equal(out, want.astype(np.float32))


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("ring", ["int16", "int32"])
def test_injected_refractory_counts_match_oracle(ring):
    """Refractory counts written into the state continue as the oracle's, bit
    for bit and signed zeros included (sim.py:921, (r + 1) * (1 - spike)).

    A third of the neurons get counts from -7 to 40 -- including counts below
    -1, which the dynamics never produce, and for which the count after a
    spike is the reference's -0 -- and half of those a membrane above
    threshold, so they fire at once: first one step per launch, then in
    20-step blocks.
    """
    name = "batch3_masks"
    sc, eng = make_engine(name, ring=ring)
    conn = S.connectome(sc)
    o = O.Oracle.from_connectome(conn, batch=sc["batch"], params_dict=sc["params"],
                                 no_refractory=S.driven(sc), seed=sc["seed"])
    rates = S.rates_matrix(sc)
    o.rates[:] = rates
    rt = torch.from_numpy(rates).cuda()
    n, B = sc["n"], sc["batch"]
    rng = np.random.default_rng(11)
    vals = np.array([-7.0, -2.5, -1.5, -1.0, -0.5, -0.0, 0.0, 3.0, 40.0], np.float32)

    def inject():
        pick = np.sort(rng.choice(n, size=n // 3, replace=False))
        r = o.refrac.copy()
        r[:, pick] = rng.choice(vals, size=(B, pick.size))
        v = o.v.copy()
        v[:, pick[::2]] = np.float32(eng.v_th + 5.0)
        o.refrac[:] = r
        o.v[:] = v
        eng.refrac.copy_(torch.from_numpy(r))
        eng.v.copy_(torch.from_numpy(v))

    inject()
    neg_zero = 0
    for step in range(6):
        eng.step(rt)
        o.run(1)
        assert np.array_equal(_bits(eng.refrac.cpu().numpy()), _bits(o.refrac)), step
        assert np.array_equal(_bits(eng.v.cpu().numpy()), _bits(o.v)), step
        assert np.array_equal(_bits(eng.conductance.cpu().numpy()), _bits(o.conductance)), step
        neg_zero += int((_bits(o.refrac) == 0x80000000).sum())
    assert neg_zero > 0  # the case the plain form exists for did occur

    for block in range(3):
        inject()
        got = eng.run_block(rt, 40).cpu().numpy()
        raster = o.run(40, raster=True)
        bits = np.unpackbits(raster, axis=2, bitorder="little")[:, :, :n]
        assert np.array_equal(got, bits.sum(0).astype(np.float32)), block
        assert np.array_equal(_bits(eng.refrac.cpu().numpy()), _bits(o.refrac)), block
        assert np.array_equal(_bits(eng.v.cpu().numpy()), _bits(o.v)), block
        assert np.array_equal(_bits(eng.conductance.cpu().numpy()), _bits(o.conductance)), block


def test_run_block_equals_stepping():
    """The closed loop's 200-step brain block equals 200 single steps."""
    name = "batch3_masks"
    sc, a = make_engine(name)
    _, b = make_engine(name)
    rates = torch.from_numpy(S.rates_matrix(sc)).cuda()
    acc = torch.zeros_like(a.spikes)
    for block in range(3):
        acc.zero_()
        for _ in range(200):
            acc += a.step(rates)
        got = b.run_block(rates, 200)
        assert torch.equal(acc, got), block
        for x, y in ((a.v, b.v), (a.conductance, b.conductance), (a.spikes, b.spikes)):
            assert torch.equal(x, y), block
    assert a.calls == b.calls == 600


def test_full_size_one_second_rates_match_reference(golden):
    """1 s of the plain configuration: identical first 100 ms, rates corr >= 0.99."""
    from fis.metrics import compare_rates

    z = golden("full_cfg0_1s")
    sc, eng = make_engine("full_cfg0_1s")
    rates = torch.from_numpy(S.rates_matrix(sc)).cuda()
    first = []
    core = eng.core
    core.rates.copy_(rates)
    for step in range(0, 1000, 20):
        core.block(20, spikes_out=eng.spikes)
        first += raster_rows(core, step, step + 20)
    bits = np.unpackbits(np.stack(first), axis=2, bitorder="little")[:, :, :sc["n"]]
    st, b, i = np.nonzero(bits)
    assert np.array_equal(st, z["spike_step"]) and np.array_equal(i, z["spike_neuron"])
    counts = eng.run_block(rates, 9000)[0].cpu().numpy().astype(np.int64)
    counts += bits[:, 0].sum(0).astype(np.int64)
    m = compare_rates(counts / 1.0, z["counts"][0] / 1.0)
    assert m["corr"] >= 0.99
    assert np.array_equal(counts, z["counts"][0])  # bit-exact, so in fact identical


def test_build_engine_from_the_upstream_folder(tmp_path, monkeypatch):
    """build_engine(weights=None) reads FIS_FLYWIRE_DATA's upstream tables and
    steps exactly as the same matrix passed as weights=."""
    import pyarrow as pa
    import pyarrow.parquet as pq

    from fis import connectome as C
    from fis import sim

    sc = S.SCENARIOS["small_b1"]
    conn = S.connectome(sc)
    pre = np.repeat(np.arange(conn.n), np.diff(conn.row_ptr))
    pq.write_table(pa.table({C.UPSTREAM_PRE: pa.array(pre, pa.int64()),
                             C.UPSTREAM_POST: pa.array(conn.col.astype(np.int64)),
                             C.UPSTREAM_VALUE: pa.array(conn.cnt.astype(np.float32))}),
                   str(tmp_path / C.UPSTREAM_CONN_FILE))
    with open(tmp_path / C.UPSTREAM_COMP_FILE, "w") as fh:
        fh.write(",root_id\n" + "".join("%d,%d\n" % (i, i) for i in range(conn.n)))
    monkeypatch.setenv("FIS_CACHE", str(tmp_path / "cache"))
    monkeypatch.setenv("FIS_FLYWIRE_DATA", str(tmp_path))
    kw = dict(batch=sc["batch"], seed=sc["seed"], no_refractory=S.driven(sc), graphs=False)
    a = sim.build_engine(**kw)
    b = sim.build_engine(weights=conn, **kw)
    rates = torch.from_numpy(S.rates_matrix(sc)).cuda()
    for _ in range(60):
        assert torch.equal(a.step(rates), b.step(rates))
    assert torch.equal(a.v, b.v) and torch.equal(a.conductance, b.conductance)
