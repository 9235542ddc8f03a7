"""The allocation-free block step, checked against the regular one.

``fis_block`` takes a scratch ring from its caller.  Some callers cannot
allocate one: a closed-loop controller that steps the brain inside a hard
real-time budget (a device allocation may synchronize the GPU and stall for
milliseconds), or a host binding only the C ABI with no device allocator of
its own.  ``fis_block_noalloc`` keeps the ring in a fixed 12 MiB array inside
the library.  This file is collected last on purpose: it runs after every
other GPU test, and also passes alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _engine(conn, drive, ring=None):
    import fis._lib as L
    from fis.engine import Core

    core = Core(conn, 1, group=1, ring=ring)
    idx = torch.as_tensor(drive, device=core.device)
    core.rates[0, idx] = 150.0
    core.flags[0, idx] |= L.FIS_FL_NOREFRAC
    core.reset_slots(slice(None))
    core.trials[0].seed = 11
    core.mark_trials()
    return core


@pytest.mark.parametrize("ring", ["int16", "int32"])
def test_noalloc_block_matches_block_on_two_calls(ring):
    import fis._lib as L
    import fis.connectome as C

    conn = C.synthetic()  # the full 138,639-neuron connectome
    drive = np.sort(np.random.default_rng(7).choice(conn.n, 2249, replace=False))
    a, b = _engine(conn, drive, ring), _engine(conn, drive, ring)
    a.advance(200)  # spikes in flight through the delay
    b.advance(200)
    lib = L.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    sa = torch.zeros((1, conn.n), device=a.device)
    sb = torch.zeros((1, conn.n), device=b.device)
    for call in range(2):
        a._sync_trials()
        b._sync_trials()
        rc = lib.fis_block(ctypes.byref(a.desc), 0, 1, 20, ctypes.c_void_p(a.ring.data_ptr()),
                           ctypes.c_void_p(sa.data_ptr()), 1, stream)
        assert rc == 0
        rc = lib.fis_block_noalloc(ctypes.byref(b.desc), 0, 1, 20,
                                   ctypes.c_void_p(sb.data_ptr()), 1, stream)
        assert rc == 0
        a.step += 20
        b.step += 20
        torch.cuda.synchronize()
        for x, y in ((a.v, b.v), (a.g, b.g), (a.refrac, b.refrac), (sa, sb),
                     (a.bits, b.bits), (a.list_len, b.list_len), (a.clock, b.clock)):
            assert torch.equal(x, y), call
        assert int(sa.sum()) > 0 or call == 0 or int(a.bits.ne(0).sum()) > 0


@pytest.mark.parametrize("ring,trials", [("int32", 2), ("int16", 3)])
def test_noalloc_refuses_blocks_larger_than_its_array(ring, trials):
    import fis._lib as L
    import fis.connectome as C
    from fis.engine import Core

    conn = C.synthetic()
    lib = L.load()
    nr = lib.fis_ring_row(conn.n)
    def words(t):  # ring words of a 20-step block: rows of trials, or of trial pairs
        return 20 * nr * ((t + 1) // 2 if ring == "int16" else t)

    assert words(trials - 1) <= L.FIS_NOALLOC_RING_INTS < words(trials)
    core = Core(conn, trials, group=trials, ring=ring)
    rc = lib.fis_block_noalloc(ctypes.byref(core.desc), 0, trials, 20, None, 1,
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == -2  # FIS_E_BOUNDS, nothing launched


def test_noalloc_checks_arguments_before_touching_its_array():
    """A refused call returns fis_block's status for the same arguments (block
    longer than the delay allows, trial range outside the batch, an external
    drive over a multi-step block), checked before the array is cleared."""
    import fis._lib as L
    import fis.connectome as C
    from fis.engine import Core

    conn = C.synthetic(n=3000, e=3000 * 100, seed=2)
    core = Core(conn, 2, group=2)
    lib = L.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for b0, nb, k in ((0, 1, L.FIS_MAX_BLOCK + 1), (0, 1, 0), (1, 2, 20), (-1, 1, 20),
                      (0, 0, 20)):
        rc = lib.fis_block_noalloc(ctypes.byref(core.desc), b0, nb, k, None, 1, stream)
        assert rc == -2, (b0, nb, k)
    vs = torch.zeros((2, conn.n), device=core.device)
    core.desc.vstim = vs.data_ptr()
    assert lib.fis_block_noalloc(ctypes.byref(core.desc), 0, 1, 2, None, 1, stream) == -2
    core.desc.vstim = None
    torch.cuda.synchronize()
