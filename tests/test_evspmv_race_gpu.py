"""The reference's own event kernel raced against this library on one B200.

``oracle/_ref/libev_spmv_ref.so`` is the reference's ``ev_spmv.cu``
(``lab/flybrain/ev_spmv.cu:60-132``) compiled from its source for sm_100a by
``oracle/Makefile`` (the recipe that needs the reference tree; the test is
skipped where the library was not built).  On the full 138,639-neuron
connectome, one trial, with 28, 103, 50,000 and 138,639 spiking presynaptic
neurons (the activity levels the reference measured its kernel at,
``LIF_PERF.md:405-414``), three ways to the same product ``W @ spikes``:

* the reference's ``ev_spmv_i32`` (one 128-thread block per presynaptic neuron);
* this library's ``ev_spmv_i32`` drop-in (same C signature);
* this library's block scatter ``fis_scatter`` (the phase-A grid of the fused
  engine) pushing the same spikes, loaded as the spike list of one step, into
  an int32 ring of one slot, in both of its forms (a warp per work item, and
  a warp per 32 work items).

All three must give the same integer sums (the weights are integer synapse
counts, so float atomics are exact in any order).  Each is timed with CUDA
events on the launching stream, alone, after warm-up, median of the repeats;
the table is printed (run with ``-s``) and written to ``$FIS_RACE_OUT`` when
that names a file.
"""

import ctypes
import json
import os
import statistics
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
REF_LIB = ROOT / "oracle" / "_ref" / "libev_spmv_ref.so"
LEVELS = (28, 103, 50_000, 138_639)
REPS = 50


def _bind(path):
    lib = ctypes.CDLL(str(path))
    P = ctypes.c_void_p
    lib.ev_spmv_i32.argtypes = [P, P, P, P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
    lib.ev_spmv_i32.restype = ctypes.c_int
    lib.ev_spmv_abi.restype = ctypes.c_int
    return lib


def _timed(fn, before=None, reps=REPS):
    ms = []
    for r in range(reps + 3):
        if before is not None:
            before()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        if r >= 3:
            ms.append(s.elapsed_time(e))
    return statistics.median(ms)


@pytest.mark.skipif(not REF_LIB.exists(), reason="reference kernel not built (oracle/Makefile ref)")
def test_reference_kernel_race():
    import fis._lib as L
    import fis.connectome as C
    from fis.engine import Core

    conn = C.synthetic(seed=0)
    n = conn.n
    ref, ours = _bind(REF_LIB), L.load()
    assert ref.ev_spmv_abi() == ours.ev_spmv_abi() == 3
    dev = torch.device("cuda")
    crow = torch.from_numpy(conn.row_ptr.astype(np.int32)).to(dev)
    col = torch.from_numpy(conn.col.astype(np.int32)).to(dev)
    val = torch.from_numpy(conn.cnt.astype(np.float32)).to(dev)
    mo = torch.ones((1, n), device=dev)
    out = torch.zeros((1, n), device=dev)
    core = Core(conn, 1, group=1, ring="int32")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    deg = conn.out_degree()
    pre_of_edge = np.repeat(np.arange(n), deg)
    rows = []
    for k in LEVELS:
        rng = np.random.default_rng(k)
        spiking = np.sort(rng.choice(n, size=k, replace=False))
        sp = torch.zeros((1, n), device=dev)
        sp[0, torch.as_tensor(spiking, device=dev)] = 1.0
        fires = np.zeros(n, dtype=bool)
        fires[spiking] = True
        sel = fires[pre_of_edge]
        want = np.rint(np.bincount(conn.col[sel], weights=conn.cnt[sel].astype(np.float64),
                                   minlength=n)).astype(np.int64)

        def call(lib):
            rc = lib.ev_spmv_i32(P(crow), P(col), P(val), P(sp), P(mo), P(out), n, 1, 128,
                                 stream)
            assert rc == 0

        got = {}
        for name, lib in (("reference ev_spmv_i32", ref), ("fis ev_spmv_i32", ours)):
            out.zero_()
            call(lib)
            torch.cuda.synchronize()
            assert np.array_equal(out[0].cpu().numpy(), want.astype(np.float32)), (name, k)
            got[name] = _timed(lambda lib=lib: call(lib), before=out.zero_)

        # the fused engine's scatter: the spikes as the list of step t-1, then
        # the clock moved so that a one-step block reads exactly that list
        t = 2 * core.lag
        core.list_len.zero_()
        core.set_clock(t)
        assert ours.fis_load_spikes(ctypes.byref(core.desc), 0, 1, P(sp), stream) == 0
        core.set_clock(t + core.lag - 1)

        def scatter():
            rc = ours.fis_scatter(ctypes.byref(core.desc), 0, 1, 1, P(core.ring), stream)
            assert rc == 0

        for mode in (0, 1):
            core.set_launch(mode)
            core.ring.zero_()
            scatter()
            torch.cuda.synchronize()
            assert np.array_equal(core.ring[0, 0, :n].cpu().numpy(), want.astype(np.int32)), k
            got["fis block scatter mode %d" % mode] = _timed(scatter, before=core.ring.zero_)
        edges = int(deg[spiking].sum())
        rows.append({"spiking": k, "edges": edges, **{key + " ms": v for key, v in got.items()},
                     "fis ev_spmv speedup": got["reference ev_spmv_i32"] / got["fis ev_spmv_i32"],
                     "fis scatter speedup": got["reference ev_spmv_i32"]
                     / min(got["fis block scatter mode 0"], got["fis block scatter mode 1"])})
    print()
    for r in rows:
        print(json.dumps(r))
    dest = os.environ.get("FIS_RACE_OUT")
    if dest:
        Path(dest).write_text("\n".join(json.dumps(r) for r in rows) + "\n")
