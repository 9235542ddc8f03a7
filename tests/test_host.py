"""Host-side logic that needs no GPU: connectome, packing, params, ABI exports."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import fis._lib as L
import fis.connectome as C
from fis.engine import lif_params
from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]


def test_synthetic_full_size_statistics():
    c = C.synthetic()
    d = c.out_degree()
    assert c.n == C.N_FLYWIRE and c.nnz == C.E_FLYWIRE
    assert abs(d.mean() - C.E_FLYWIRE / C.N_FLYWIRE) < 1e-9
    assert d.max() <= c.n - 1 and d.min() >= 1
    pre = np.repeat(np.arange(c.n), d)
    assert not np.any(pre == c.col)                      # no self-loops
    assert np.all(np.diff(pre.astype(np.int64) * c.n + c.col) > 0)  # unique, sorted
    assert c.cnt.min() >= -2400 and c.cnt.max() <= 2400 and not np.any(c.cnt == 0)
    sign = np.sign(c.cnt)
    assert np.all(sign[c.row_ptr[:-1][d > 0]] == sign[c.row_ptr[1:][d > 0] - 1])  # sign per pre
    frac_inh = np.mean(sign[c.row_ptr[:-1][d > 0]] < 0)
    assert 0.28 < frac_inh < 0.32
    assert c.exactness()["ok"]


def test_synthetic_is_deterministic():
    a = C.synthetic(n=3000, e=300000, seed=4, cache=False)
    b = C.synthetic(n=3000, e=300000, seed=4, cache=False)
    assert np.array_equal(a.col, b.col) and np.array_equal(a.cnt, b.cnt)
    c = C.synthetic(n=3000, e=300000, seed=5, cache=False)
    assert not np.array_equal(a.col, c.col)


def test_packed_roundtrip_and_limits():
    c = C.synthetic(n=2000, e=150000, seed=2, cache=False)
    w = c.packed()
    post = (w >> 14).astype(np.int64)
    cnt = ((w.astype(np.int64) & 0x3FFF) ^ 0x2000) - 0x2000
    assert np.array_equal(post, c.col) and np.array_equal(cnt, c.cnt)
    big = C.Connectome(4, np.array([0, 1, 1, 1, 1]), np.array([1], np.int32),
                       np.array([9000], np.int32))
    with pytest.raises(C.ConnectomeError):
        big.packed()


def test_from_weights_roundtrip():
    import torch

    c = C.synthetic(n=1500, e=90000, seed=9, cache=False)
    w = c.to_torch_weights()
    back = C.from_weights(w)
    assert np.array_equal(back.row_ptr, c.row_ptr)
    assert np.array_equal(back.col, c.col) and np.array_equal(back.cnt, c.cnt)
    bad = torch.sparse_coo_tensor(torch.tensor([[0], [1]]), torch.tensor([1.5]), (3, 3))
    with pytest.raises(C.ConnectomeError):
        C.from_weights(bad)


def test_without_matches_reference_silencing_semantics():
    c = C.synthetic(n=1200, e=60000, seed=3, cache=False)
    sil = np.array([5, 17, 400])
    s = c.without(sil)
    pre = np.repeat(np.arange(s.n), s.out_degree())
    assert not np.isin(pre, sil).any() and not np.isin(s.col, sil).any()
    kept = ~(np.isin(np.repeat(np.arange(c.n), c.out_degree()), sil) | np.isin(c.col, sil))
    assert s.nnz == int(kept.sum())


def test_bounds_check_refuses_bad_csr():
    c = C.Connectome(3, np.array([0, 1, 2, 2]), np.array([1, 3], np.int32),
                     np.array([1, 1], np.int32))
    with pytest.raises(C.ConnectomeError):
        c.check_bounds()


@pytest.mark.parametrize("p", [None, {"tauSyn": 4.0, "tDelay": 1.0, "v0": -55.0, "vReset": -58.0,
                                      "vRest": -52.5, "vThreshold": -46.3, "tauMem": 17.0,
                                      "tRefrac": 1.3, "scalePoisson": 200, "wScale": 0.31}])
def test_params_match_oracle(p):
    a, b = lif_params(p), O.params(p)
    for name, _ in b._fields_:
        assert getattr(a, name) == getattr(b, name), name


def test_library_exports_every_declared_symbol():
    """The C-ABI library loads on a CPU-only host and exports fis.h's symbols."""
    import fis.build

    fis.build.build()
    header = (ROOT / "include" / "fis.h").read_text()
    declared = set(re.findall(r"^int\s+(\w+)\(", header, flags=re.M))
    assert declared == set(L.EXPORTS)
    lib = ctypes.CDLL(str(L.LIB_PATH))
    for name in declared:
        assert hasattr(lib, name), name
    L.load()  # ABI and struct-layout checks (no device call)
    assert lib.ev_spmv_abi() == 3


def test_check_rejects_bad_descriptor():
    lib = L.load()
    d = L.EngineDesc()
    assert lib.fis_check(ctypes.byref(d)) == -1  # null pointers
    assert lib.fis_block(ctypes.byref(d), 0, 1, 1, None, None, 1, None) == -1


def test_rate_guard():
    from fis import sim

    sim.check_rates_hz([0.0, 150.0, 10000.0], "test")
    for bad in ([10001.0], [-1.0], [float("nan")]):
        with pytest.raises(sim.RateTooHigh):
            sim.check_rates_hz(bad, "test")


def test_stim_schedule_matches_reference_order():
    from fis import sim

    s1 = sim.Stimulus(np.array([1, 2]), 100.0, t_on_ms=5.0, t_off_ms=20.0)
    s2 = sim.Stimulus(np.array([3]), 50.0)
    ev = sim.stim_schedule([s1, s2], steps=1000)
    assert [(e[0], e[2]) for e in ev] == [(0, 50.0), (50, 100.0), (200, 0.0)]


def test_engine_refuses_cpu_loudly():
    from fis import evspmv, sim

    c = C.synthetic(n=500, e=20000, seed=1, cache=False)
    with pytest.raises(evspmv.EventKernelUnavailable):
        sim.Engine(c, c.n, device="cpu")


def test_sparse_rows_equal_dense_rows():
    """The sparse upload of Batch.load lays out exactly host_rows' rows."""
    from fis.batch import host_rows, random_specs, sparse_rows

    n = 5000
    specs = random_specs(n, 6, 3, 100, stim_range=(50, 300), silenced_range=(1, 40))
    specs[2].fire_off = specs[2].stim[:10]
    specs[3].hold, specs[3].in_off = np.arange(10, 60), np.arange(30, 90)
    specs[4].stim = np.concatenate([specs[4].stim, specs[4].stim[:5]])   # repeats
    specs[4].rate_hz = np.arange(len(specs[4].stim), dtype=np.float64) + 1.0
    specs[5].out_off = specs[5].stim[:7]
    slots = [3, 0, 5, 1, 4, 2]
    flags, rates = host_rows(specs, n)
    fa, fb, ra, rv = sparse_rows(specs, n, slots)
    assert np.all(np.diff(fa) > 0) and np.all(np.diff(ra) > 0)
    F = np.zeros((6, n), np.uint8)
    R = np.zeros((6, n), np.float32)
    F.reshape(-1)[fa] = fb
    R.reshape(-1)[ra] = rv
    for j, b in enumerate(slots):
        assert np.array_equal(F[b], flags[j]) and np.array_equal(R[b], rates[j]), j


def test_sparse_rows_fast_and_sorting_paths_agree():
    """sparse_rows skips its sort when positions already ascend; the same
    trials in descending slots (the sorting path) give the same rows, and
    empty inputs give empty arrays."""
    from fis.batch import TrialSpec, host_rows, random_specs, sparse_rows

    n = 3000
    specs = random_specs(n, 5, 11, 50, stim_range=(20, 200), silenced_range=(1, 30))
    specs.append(TrialSpec(seed=1, steps=10))  # no stimulus, no flags
    k = len(specs)
    up = list(range(k))
    down = list(reversed(range(k)))
    fa, fb, ra, rv = sparse_rows(specs, n, up)
    assert np.all(np.diff(fa) > 0) and np.all(np.diff(ra) > 0)
    flags, rates = host_rows(specs, n)
    for slots, (a1, b1, a2, v2) in ((up, (fa, fb, ra, rv)), (down, sparse_rows(specs, n, down))):
        F = np.zeros((k, n), np.uint8)
        R = np.zeros((k, n), np.float32)
        F.reshape(-1)[a1] = b1
        R.reshape(-1)[a2] = v2
        for j, b in enumerate(slots):
            assert np.array_equal(F[b], flags[j]) and np.array_equal(R[b], rates[j]), (slots, j)
    e = sparse_rows([], n, [])
    assert all(x.size == 0 for x in e)
    e = sparse_rows([TrialSpec(seed=0, steps=5)], n, [0])
    assert all(x.size == 0 for x in e)


def test_exactness_record_and_transpose():
    """evspmv.exactness: the reference's record (keys and verdict) computed
    from the CSR arrays; Events' transposition lists each presynaptic row with
    its postsynaptic indices ascending."""
    import torch

    from fis import evspmv

    c = C.synthetic(n=700, e=700 * 40, seed=4, cache=False)
    w = c.to_torch_weights().to_sparse_csr()
    rec = evspmv.exactness(w)
    want = float(c.in_abs_sum().max())
    assert rec["макс сумма модулей по строке"] == want
    assert rec["значения целые"] and rec["годится"]
    assert rec["мин значение"] == float(c.cnt.min()) and rec["макс значение"] == float(c.cnt.max())
    assert rec["запас"] == round((1 << 24) / want, 1)
    frac = torch.sparse_csr_tensor(w.crow_indices(), w.col_indices(), w.values() + 0.25,
                                   size=w.shape)
    bad = evspmv.exactness(frac)
    assert not bad["значения целые"] and not bad["годится"] and bad["макс нецелая часть"] == 0.25
    n, _, rp, col, val = evspmv._csr_arrays(w)
    t_ptr, t_post, t_val = evspmv._by_pre(n, rp, col, val)
    assert t_ptr.dtype == rp.dtype and t_post.dtype == col.dtype
    assert np.array_equal(t_ptr, c.row_ptr) and np.array_equal(t_post, c.col)
    assert np.array_equal(t_val, c.cnt.astype(np.float32))


def test_csr_faults_name_each_fault():
    rp = np.array([0, 2, 3], dtype=np.int64)
    assert C.csr_faults(2, rp, np.array([1, 0, 1]), 3) == []
    assert any("outside" in f for f in C.csr_faults(2, rp, np.array([1, 0, 2]), 3))
    assert any("n+1" in f for f in C.csr_faults(2, np.array([0, 3, 2, 3]), np.zeros(3), 3))
    assert any("decreases" in f for f in C.csr_faults(2, np.array([0, 4, 3]), np.zeros(3), 3))
    assert any("values" in f for f in C.csr_faults(2, rp, np.array([1, 0, 1]), 4))


def test_result_save_load_round_trip(tmp_path):
    """save() writes the reference's three files; load() rebuilds the same
    counts, bins, config, stimuli and silencing."""
    import pandas as pd

    from fis import sim

    rng = np.random.default_rng(5)
    n = 400
    bins = rng.integers(0, 3, size=(7, n)).astype(np.int16)
    bins[:, ::3] = 0
    neurons = pd.DataFrame({"root_id": np.arange(n) + 10 ** 9,
                            "region": np.array(["AL", "MB"])[np.arange(n) % 2]})
    cfg = sim.RunConfig(t_run_s=0.07, bin_ms=10.0, n_trials=2, seed=3)
    stims = [sim.Stimulus(np.array([5, 9, 11]), 150.0, 1.0, None, "s1"),
             sim.Stimulus(np.array([2]), 90.0, 0.0, 30.0, "s2")]
    res = sim.Result(bins.sum(0).astype(np.int64), bins, cfg, stims, np.array([4, 8]), neurons,
                     {"steps": 700, "sim_s": 0.1})
    meta = res.meta(with_indices=True)
    assert meta["stimuli"][0] == {"name": "s1", "n": 3, "rate_hz": 150.0, "t_on_ms": 1.0,
                                  "t_off_ms": None, "indices": [5, 9, 11]}
    assert meta["silenced"] == [4, 8] and res.meta()["silenced"] is None
    assert meta["n_active"] == int((res.counts / (0.07 * 2) >= 0.5).sum())
    out = sim.save(res, tmp_path / "run")
    assert sorted(p.name for p in out.iterdir()) == ["bins.npz", "meta.json", "rates.parquet"]
    back = sim.load(out, neurons=neurons)
    assert np.array_equal(back.counts, res.counts)
    assert np.array_equal(back.bins, res.bins)
    assert back.config == cfg
    assert [s.to_dict(True) for s in back.stimuli] == [s.to_dict(True) for s in stims]
    assert list(back.silenced) == [4, 8] and back.timing == res.timing
    table = res.rate_table()
    assert list(table.columns) == ["root_id", "region", "rate_hz", "n_spikes"]
    assert table["rate_hz"].is_monotonic_decreasing
    tl = res.region_timeline()
    want = bins[:, ::2].mean(1) / (0.01 * 2)
    assert np.allclose(tl.loc["AL"].to_numpy(), want)


def test_drive_lists_from_rates_and_from_sparse_positions():
    """The driven-neuron lists phase A reads (Core.use_drive_lists): rebuilt
    from the rates, or set from the sparse positions a batch load writes,
    each trial's first drive_len entries are its neurons with a positive
    rate (ascending) and other trials' lists are untouched."""
    import types

    import torch

    from fis.engine import Core

    rng = np.random.default_rng(3)
    B, n = 5, 97
    rates = torch.zeros((B, n), dtype=torch.float32)
    for b in range(B):
        idx = rng.choice(n, size=int(rng.integers(0, 20)), replace=False)
        rates[b, torch.as_tensor(idx)] = torch.as_tensor(rng.uniform(50, 300, idx.size),
                                                         dtype=torch.float32)
    fake = types.SimpleNamespace(n=n, batch=B, rates=rates,
                                 drive_idx=torch.full((B, n), -1, dtype=torch.int32),
                                 drive_len=torch.full((B,), -1, dtype=torch.int32))
    Core.rebuild_drive_lists(fake)
    for b in range(B):
        want = torch.nonzero(rates[b] > 0).flatten().tolist()
        k = int(fake.drive_len[b])
        assert fake.drive_idx[b, :k].tolist() == want
    # a load of rows 1 and 3 (positions unsorted, as packed per trial)
    before = fake.drive_idx.clone(), fake.drive_len.clone()
    pos = []
    for b in (3, 1):
        pos += [b * n + int(i) for i in rng.permutation(rng.choice(n, size=7, replace=False))]
    rows = torch.as_tensor([1, 3])
    Core.set_drive_lists_sparse(fake, rows, torch.as_tensor(pos, dtype=torch.int64))
    for b in range(B):
        k = int(fake.drive_len[b])
        if b in (1, 3):
            want = sorted(p - b * n for p in pos if p // n == b)
            assert fake.drive_idx[b, :k].tolist() == want
        else:
            assert k == int(before[1][b])
            assert torch.equal(fake.drive_idx[b], before[0][b])
    Core.set_drive_lists_sparse(fake, slice(0, 2), torch.zeros(0, dtype=torch.int64))
    assert fake.drive_len[:2].tolist() == [0, 0]
