"""Device-resident engine core: B trial slots over one connectome.

``Core`` owns every device buffer of ``include/fis.h``'s ``fis_engine``
descriptor (allocated once, through torch's caching allocator) and drives the
two-phase block of ``libfis_b200.so``.  It is the layer under both the
reference-compatible :class:`fis.sim.Engine` and the batched/serving layers.

Layout in HBM (B slots, N neurons, L = lag = buf_len + 1 = 20 by default):

* connectome: ``row_ptr`` int64 [N+1], packed ``edges`` uint32 [E rounded up
  to 4] (60.4 MB at E = 15.09 M), ``nchunks`` uint16 [N];
* state, trial-major [B][N]: ``v, g, refrac`` float32, ``flags`` uint8,
  ``rates`` float32 -- read once and written once per block of up to 20 steps;
* spike history: ``lists`` uint32 [L][B][cap], ``list_len`` int32 [2L][B],
  ``bits`` uint32 [B][ceil(N/32)][L];
* scratch ring [K][G][NR] (int32, or biased int16 pairs) for one trial group
  of G slots, reused by every group: sized to stay resident in the 126 MB L2
  between the scatter that fills it and the update that drains it.  Two such
  rings when the scatter of one group overlaps the update of the previous one.
"""

from __future__ import annotations

import ctypes
import math
import os

import numpy as np
import torch

from . import _lib
from .connectome import Connectome

MODEL_PARAMS = {
    "tauSyn": 5.0, "tDelay": 1.8, "v0": -52.0, "vReset": -52.0, "vRest": -52.0,
    "vThreshold": -45.0, "tauMem": 20.0, "tRefrac": 2.2, "scalePoisson": 250,
    "wScale": 0.275,
}
DT = 0.1

# Bytes of scratch ring per trial group that are meant to stay in L2.
RING_L2_BYTES = 48 << 20


def lif_params(p=None) -> _lib.LifParams:
    """The step's constants, derived as ``Engine.__init__`` derives them.

    ``sim.py:356-366``: each Python double (``DT / tauSyn`` ...) meets a float32
    tensor, so it is rounded to float32 once; ``1 - DT/tauSyn`` is formed in
    double first (``sim.py:929``).  The Poisson kick is the float32 product
    ``w_scale * (1.0 * scalePoisson)`` (``sim.py:859-861``).
    """
    p = dict(MODEL_PARAMS if p is None else p)
    f = np.float32
    buf_len = int(p["tDelay"] / DT) + 1
    w = f(p["wScale"])
    kick = f(w * f(f(1.0) * f(p["scalePoisson"])))
    return _lib.LifParams(
        a_syn=float(f(1.0 - DT / p["tauSyn"])), a_mem=float(f(DT / p["tauMem"])),
        w_scale=float(w), kick=float(kick), prob_scale=float(f(DT / 1000.0)),
        v_rest=float(f(p["vRest"])), v_reset=float(f(p["vReset"])),
        v_th=float(f(p["vThreshold"])),
        refrac_steps=float(f(float(round(p["tRefrac"] / DT)))),
        buf_len=buf_len, lag=buf_len + 1, pad_=0)


def require_cuda(device):
    dev = torch.device(device)
    if dev.type != "cuda":
        raise _lib.KernelUnavailable(
            "this engine runs on CUDA only (asked for %r); there is no CPU path" % device)
    if not torch.cuda.is_available():
        raise _lib.KernelUnavailable("CUDA is not available in this process")
    return torch.device("cuda", torch.cuda.current_device() if dev.index is None else dev.index)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class Core:
    """B trial slots, their state on the device, and the block launcher."""

    # an empty word of the paired int16 ring: the biased zero 0x8000 in both
    # halves (0x80008000 as int32); the int32 ring's empty value is 0
    RING_EMPTY16 = -0x7FFF8000

    def __init__(self, conn: Connectome, batch: int, params=None, device="cuda",
                 group=None, chunk=None, max_block=_lib.FIS_MAX_BLOCK, ring=None,
                 overlap=True, raster=True, scatter_mode=None, scat_ctas=0, drive_ctas=0,
                 update_streams=1, update_tiles=None):
        self.device = require_cuda(device)
        self.lib = _lib.load()
        conn.check_bounds()
        ex = conn.exactness()
        if not ex["ok"]:
            raise _lib.KernelUnavailable(
                "max |row sum| %.0f >= 2**24: integer accumulation would not be "
                "exact for this matrix" % ex["max_abs_row_sum"])
        self.conn = conn
        self.overlap = bool(overlap)
        # raster=False keeps only each block's last step in `bits` (enough for
        # the next block); spikes of other steps are then not available
        self.raster = bool(raster)
        # Scratch-ring element: biased int16 when no neuron's incoming
        # |count| sum reaches 2**15 (exact, half the ring traffic), else int32.
        ring = ring or os.environ.get("FIS_RING", "auto")
        if ring not in ("auto", "int16", "int32"):
            raise ValueError("ring must be auto, int16 or int32")
        fits16 = ex["max_abs_row_sum"] < (1 << 15)
        if ring == "int16" and not fits16:
            raise _lib.KernelUnavailable(
                "an int16 ring is not exact here: max |row sum| %.0f >= 2**15"
                % ex["max_abs_row_sum"])
        self.ring16 = fits16 if ring == "auto" else ring == "int16"
        self.n = n = int(conn.n)
        self.batch = B = int(batch)
        if B < 1:
            raise ValueError("batch must be >= 1")
        self.pdict = dict(MODEL_PARAMS if params is None else params)
        self.P = lif_params(self.pdict)
        self.v0 = float(np.float32(self.pdict["v0"]))
        L = self.lag = int(self.P.lag)
        self.buf_len = int(self.P.buf_len)
        self.max_block = max(1, min(int(max_block), _lib.FIS_MAX_BLOCK, L))
        dev = self.device

        deg = conn.out_degree()
        maxdeg = int(deg.max()) if n else 0
        if chunk is None:
            chunk = max(256, 128 * math.ceil(maxdeg / (255 * 128)))
        if chunk % 128 or chunk < 128 or math.ceil(maxdeg / chunk) > 256:
            raise ValueError("chunk %d does not cover rows of %d edges in 256 pieces"
                             % (chunk, maxdeg))
        self.chunk = int(chunk)
        nch = np.where(deg > 0, -(-deg // self.chunk), 0).astype(np.int64)
        self.list_cap = max(1, int(nch.sum()))

        packed = conn.packed()
        nnz = packed.shape[0]
        nnz4 = max(4, (nnz + 3) // 4 * 4)
        edges = np.zeros(nnz4, dtype=np.uint32)
        edges[:nnz] = packed
        with torch.cuda.device(dev):
            self.row_ptr = torch.from_numpy(conn.row_ptr.astype(np.int64)).to(dev)
            self.edges = torch.from_numpy(edges.view(np.int32)).to(dev)
            self.nchunks = torch.from_numpy(nch.astype(np.int16)).to(dev)
            self.v = torch.full((B, n), self.v0, dtype=torch.float32, device=dev)
            self.g = torch.zeros((B, n), dtype=torch.float32, device=dev)
            self.refrac = torch.full((B, n), self.P.refrac_steps, dtype=torch.float32, device=dev)
            self.flags = torch.zeros((B, n), dtype=torch.uint8, device=dev)
            self.rates = torch.zeros((B, n), dtype=torch.float32, device=dev)
            self.trials_dev = torch.zeros(B * ctypes.sizeof(_lib.Trial), dtype=torch.uint8,
                                          device=dev)
            self.lists = torch.zeros((L, B, self.list_cap), dtype=torch.int32, device=dev)
            self.list_len = torch.zeros((2 * L, B), dtype=torch.int32, device=dev)
            self.words = (n + 31) // 32
            self.bits = torch.zeros((B, self.words, L), dtype=torch.int32, device=dev)
            # fis_clock: step, then (step mod lag) | (step mod 2*lag) << 32
            self.clock = torch.zeros(2, dtype=torch.int64, device=dev)
            # [0] block-completion counter, [1] error bits (FIS_ERR_*)
            self.done = torch.zeros(2, dtype=torch.int32, device=dev)
            # kick steps of the current block per driven (trial, neuron)
            self.kicks = torch.zeros((B, n), dtype=torch.int32, device=dev)
        # per-trial lists of driven neurons for phase A (use_drive_lists)
        self.drive_idx = None
        self.drive_len = None
        self.trials = (_lib.Trial * B)()
        for b in range(B):
            self.trials[b].start = 0
            self.trials[b].end = 2 ** 62
            self.trials[b].v_clamp = float(np.float32(self.pdict["vReset"]))
            self.trials[b].stream = b
            self.trials[b].rec = -1
        self._trials_dirty = True
        self.recs = []          # recording buffers (int32 [n_bins][N])
        self._recs_ptrs = None  # device array of their addresses
        self.step = 0           # host mirror of the device clock
        self.pending = None     # (first step, int32 [buf_len][B][N]) after restore
        self.set_group(group)

        self.desc = _lib.EngineDesc()
        d = self.desc
        d.row_ptr = self.row_ptr.data_ptr()
        d.edges = self.edges.data_ptr()
        d.nchunks = self.nchunks.data_ptr()
        d.v, d.g, d.refrac = self.v.data_ptr(), self.g.data_ptr(), self.refrac.data_ptr()
        d.flags = self.flags.data_ptr()
        d.rates = self.rates.data_ptr()
        d.vstim = None
        d.trials = self.trials_dev.data_ptr()
        d.lists = self.lists.data_ptr()
        d.list_len = self.list_len.data_ptr()
        d.bits = self.bits.data_ptr()
        d.clock = self.clock.data_ptr()
        d.done = self.done.data_ptr()
        d.kicks = self.kicks.data_ptr()
        d.drive_idx = None
        d.drive_len = None
        d.recs = None
        d.nnz = nnz
        d.list_cap = self.list_cap
        d.n, d.batch, d.chunk, d.n_recs = n, B, self.chunk, 0
        d.ring16 = 1 if self.ring16 else 0
        d.raster = 1 if self.raster else 0
        d.p = self.P
        self.set_launch(scatter_mode, scat_ctas, drive_ctas, update_streams, update_tiles)

    def use_drive_lists(self):
        """Give phase A per-trial lists of the driven neurons, so that its
        Poisson drive reads the rates of those neurons only instead of every
        rate (the draws and the results are the same).

        From then on every write of ``rates`` must keep the lists in step:
        each trial's first ``drive_len[b]`` entries of ``drive_idx[b]`` are a
        superset of its neurons with a positive rate.  ``fis.batch.Batch``
        does this as it loads trials; a caller that writes ``rates`` itself
        calls ``rebuild_drive_lists`` afterwards.  The lists are built now
        from the current rates.
        """
        if self.drive_idx is None:
            self.drive_idx = torch.zeros((self.batch, self.n), dtype=torch.int32,
                                         device=self.device)
            self.drive_len = torch.zeros(self.batch, dtype=torch.int32, device=self.device)
            self.desc.drive_idx = self.drive_idx.data_ptr()
            self.desc.drive_len = self.drive_len.data_ptr()
        self.rebuild_drive_lists()

    def rebuild_drive_lists(self, rows=None):
        """Rebuild the driven-neuron lists of ``rows`` (all trials by
        default) from ``rates``: the neurons with a positive rate, ascending."""
        if self.drive_idx is None:
            return
        rows = slice(None) if rows is None else rows
        driven = self.rates[rows] > 0
        # a stable sort of "not driven" puts each row's driven neurons first,
        # in ascending order
        order = torch.sort((~driven).to(torch.int8), dim=1, stable=True).indices
        self.drive_idx[rows] = order.to(torch.int32)
        self.drive_len[rows] = driven.sum(dim=1, dtype=torch.int32)

    def set_drive_lists_sparse(self, rows, positions):
        """Set the lists of the trials in ``rows`` (a slice or an index
        tensor) from ``positions``: the flat positions slot * N + neuron
        (int64, on the device, unique) of every neuron of those trials that
        may have a positive rate."""
        if self.drive_idx is None:
            return
        n = self.n
        self.drive_len[rows] = 0
        if positions.numel() == 0:
            return
        p = torch.sort(positions).values
        slot = p // n
        cnt = torch.bincount(slot, minlength=self.batch)
        first = torch.cumsum(cnt, 0) - cnt
        rank = torch.arange(p.numel(), device=p.device) - first[slot]
        self.drive_idx[slot, rank] = (p - slot * n).to(torch.int32)
        self.drive_len[rows] = cnt.to(torch.int32)[rows]

    def set_launch(self, scatter_mode=None, scat_ctas=0, drive_ctas=0, update_streams=1,
                   update_tiles=None):
        """Phase A's launch shape (exact: it changes scheduling, never sums).

        ``scatter_mode`` 0: a warp walks one work item (spike, row chunk) at a
        time; 1: a warp resolves 32 items together and walks their edges as
        one stream (None: ``FIS_SCATTER_MODE``, else 1).  ``scat_ctas`` and
        ``drive_ctas``: scattering and drive CTAs per 8 SMs (0: the library's
        default for the mode).  ``update_streams`` 2: in the overlapped native
        loop, consecutive updates (of different trial groups) alternate
        between two streams.  ``update_tiles`` 2: streamed tiles -- up to 4
        update CTAs per SM, each pipelining a run of (trial pair, tile) items
        whose input arrives by bulk copies while the previous item's steps
        run (None: ``FIS_UPDATE_TILES``, else 1; measured ~24 % slower than
        one tile per CTA on the bench, which stays the default).
        """
        if scatter_mode is None:
            scatter_mode = int(os.environ.get("FIS_SCATTER_MODE", "1"))
        if update_tiles is None:
            update_tiles = int(os.environ.get("FIS_UPDATE_TILES", "1"))
        d = self.desc
        d.scatter_mode, d.scat_ctas, d.drive_ctas = (int(scatter_mode), int(scat_ctas),
                                                     int(drive_ctas))
        d.update_streams = int(update_streams)
        d.update_tiles = int(update_tiles)
        _lib.check(self.lib.fis_check(ctypes.byref(d)), "fis_check")
        self.update_tiles = int(update_tiles)
        self.scatter_mode, self.scat_ctas, self.drive_ctas = (int(scatter_mode), int(scat_ctas),
                                                               int(drive_ctas))
        self.update_streams = int(update_streams)

    def check_errors(self):
        """Raise if a kernel flagged an error since the last check (synchronises).

        A CTA whose staged input did not arrive within its bounded wait skipped
        its update and set FIS_ERR_STAGE: the state is then not the model's.
        """
        self.raise_errors(int(self.done[1].item()))

    def errors_async(self):
        """The error bits as of this point of the stream, copied into a pinned
        host word without waiting; pass it to ``raise_errors`` once the stream
        has passed this point (an event recorded after this call)."""
        host = torch.empty(1, dtype=torch.int32, pin_memory=True)
        host.copy_(self.done[1:2], non_blocking=True)
        return host

    def raise_errors(self, err):
        """Raise for error bits ``err`` (an int, or a word from ``errors_async``).

        A CTA that gave up waiting for its staged input left its lines of the
        scratch ring as the scatter wrote them, so the rings are refilled with
        their empty value before the error is raised: the core stays usable
        for a fresh run.  If a CTA also gave up on the copies still in flight
        (FIS_ERR_STAGE_LOST), the CUDA context cannot be trusted any more.
        """
        err = int(err[0]) if torch.is_tensor(err) else int(err)
        if not err:
            return
        self.done[1].zero_()
        self._empty_rings()
        if err & _lib.FIS_ERR_STAGE_LOST:
            raise RuntimeError("the device reported error bits 0x%x: copies into a CTA's "
                               "shared memory outlived it (FIS_ERR_STAGE_LOST); this CUDA "
                               "context is not safe to use further" % err)
        raise RuntimeError("the device reported error bits 0x%x (FIS_ERR_STAGE = 1: "
                           "a block's staged input did not arrive)" % err)

    def _empty_rings(self):
        self.ring2.fill_(self.RING_EMPTY16 if self.ring16 else 0)

    def set_clock(self, step):
        """Set the device step counter (and its slot indices) and the host mirror."""
        step = int(step)
        L = self.lag
        packed = (step % L) | ((step % (2 * L)) << 32)
        self.clock.copy_(torch.tensor([step, packed], dtype=torch.int64))
        self.step = step

    # --- configuration ---------------------------------------------------

    def ring_rows(self, nb):
        """Rows of NR 32-bit words per ring slot for ``nb`` trials.

        int32 ring: one row per trial; paired int16 ring: one row per pair of
        trials (trial 2p in the low half of each word, 2p + 1 in the high).
        """
        return (nb + 1) // 2 if self.ring16 else nb

    def set_group(self, group=None):
        """Trial-group size G of the scratch ring (None: fit in L2)."""
        if group is None:
            group = max(1, RING_L2_BYTES // (self.max_block * self.n * 4))
        self.group = int(max(1, min(int(group), self.batch)))
        self.ring_row = int(self.lib.fis_ring_row(self.n))
        shape = (2 if self.overlap else 1, self.max_block, self.ring_rows(self.group),
                 self.ring_row)
        with torch.cuda.device(self.device):
            self.ring2 = torch.full(shape, self.RING_EMPTY16 if self.ring16 else 0,
                                    dtype=torch.int32, device=self.device)
        self.ring = self.ring2[0]

    def set_recordings(self, bufs):
        """Recording buffers, each int32 [n_bins][N]; trials point at them by index."""
        self.recs = list(bufs)
        if self.recs:
            ptrs = torch.tensor([b.data_ptr() for b in self.recs], dtype=torch.int64)
            self._recs_ptrs = ptrs.to(self.device)
            self.desc.recs = self._recs_ptrs.data_ptr()
        else:
            self._recs_ptrs = None
            self.desc.recs = None
        self.desc.n_recs = len(self.recs)

    def _sync_trials(self):
        if self._trials_dirty:
            # a fresh pinned buffer from torch's caching host allocator, which
            # holds it until the asynchronous copy has run: the host does not
            # wait for the stream
            host = torch.empty(ctypes.sizeof(self.trials), dtype=torch.uint8, pin_memory=True)
            ctypes.memmove(host.data_ptr(), ctypes.addressof(self.trials), ctypes.sizeof(self.trials))
            self.trials_dev.copy_(host, non_blocking=True)
            self._trials_dirty = False

    def mark_trials(self):
        self._trials_dirty = True

    # --- slots -------------------------------------------------------------

    def reset_slots(self, rows):
        """Initial state for slots ``rows`` (a slice or index tensor).

        ``v = v0``, ``g = 0``, ``refrac = refrac_steps`` of each neuron (0 under
        FIS_FL_NOREFRAC), as ``Engine.__init__`` (sim.py:383-388); the slot's
        spike history is emptied so nothing of a previous occupant is delivered.
        """
        self.v[rows] = self.v0
        self.g[rows] = 0.0
        nore = (self.flags[rows] & _lib.FIS_FL_NOREFRAC) != 0
        self.refrac[rows] = torch.where(nore, torch.zeros((), device=self.device),
                                        torch.full((), self.P.refrac_steps, device=self.device))
        self.list_len[:, rows] = 0

    # --- stepping ------------------------------------------------------------

    def block(self, k, spikes_out=None, stream=None, timer=None, rows=None,
              scatter_timer=None):
        """Advance every slot by ``k`` steps (1 <= k <= max_block).

        ``rows``: launch only the trial groups covering slots [0, rows); the
        caller guarantees that no slot at or above it is running (a slot that
        is launched again later is re-initialised first, see reset_slots).
        ``timer`` (optional) is called as ``timer(stream, True)`` right before
        and ``timer(stream, False)`` right after each update launch, so a caller
        can bracket the dominant kernel with CUDA events; ``scatter_timer`` the
        same around each phase-A launch (scatter and Poisson drive).
        """
        k = int(k)
        if not 1 <= k <= self.max_block:
            raise ValueError("block of %d steps; 1..%d allowed" % (k, self.max_block))
        self._sync_trials()
        st = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        sp = ctypes.c_void_p(spikes_out.data_ptr()) if spikes_out is not None else None
        G = self.group
        B = self.batch if rows is None else max(1, min(int(rows), self.batch))
        for g0 in range(0, B, G):
            nb = min(G, B - g0)
            if self.pending is not None:
                self._apply_pending(g0, nb, k, st)
            ring = ctypes.c_void_p(self.ring.data_ptr())
            if scatter_timer is not None:
                scatter_timer(st, True)
            rc = self.lib.fis_scatter(ctypes.byref(self.desc), g0, nb, k, ring,
                                      ctypes.c_void_p(st))
            _lib.check(rc, "fis_scatter")
            if scatter_timer is not None:
                scatter_timer(st, False)
            if timer is not None:
                timer(st, True)
            rc = self.lib.fis_update(ctypes.byref(self.desc), g0, nb, k, ring, sp,
                                     1 if g0 + nb == B else 0, ctypes.c_void_p(st))
            _lib.check(rc, "fis_update")
            if timer is not None:
                timer(st, False)
        self.step += k
        if self.pending is not None and self.step >= self.pending[0] + self.buf_len:
            self.pending = None

    def _apply_pending(self, g0, nb, k, st):
        p0, rows = self.pending
        t0 = self.step
        lo, hi = max(t0, p0), min(t0 + k, p0 + self.buf_len)
        if lo >= hi:
            return
        n, NR = self.n, self.ring_row
        src = rows[lo - p0, g0]  # [nb][N] starts here; row stride B*N
        # the kernel's ring for this group: k slots of ring_rows(nb) rows of NR words
        slot = self.ring_rows(nb) * NR
        rc = self.lib.fis_add_rows(ctypes.byref(self.desc), nb, hi - lo,
                                   ctypes.c_void_p(src.data_ptr()), self.batch * n, n,
                                   ctypes.c_void_p(self.ring.data_ptr() + (lo - t0) * slot * 4),
                                   slot, NR, ctypes.c_void_p(st))
        _lib.check(rc, "fis_add_rows")

    def advance(self, steps, spikes_out=None, timer=None, events=None, every=1, rows=None):
        """``steps`` steps in blocks of at most ``max_block``.

        Runs the native block loop (``fis_advance_overlap`` when there are two
        or more trial groups and two rings, else ``fis_advance``) unless
        restored pending input or a Python ``timer`` needs the per-block path.
        ``events``: a list of ``torch.cuda.Event`` pairs (flattened) recorded
        around every ``every``-th update launch.  ``rows``: advance only slots
        [0, rows), as in :meth:`block`.
        """
        steps = int(steps)
        if steps <= 0:
            return
        nrows = self.batch if rows is None else max(1, min(int(rows), self.batch))
        if self.pending is not None or timer is not None or self.max_block != min(
                _lib.FIS_MAX_BLOCK, self.lag):
            if events and timer is None:
                # the native loop's event pairs, around every `every`-th update
                # launch, recorded on the current stream that block() uses
                n_pairs, every, seen = len(events) // 2, max(1, int(every)), [0]
                for e in events:  # pairs never reached read as zero, as natively
                    e.record(torch.cuda.current_stream(self.device))

                def timer(_stream, start):
                    j, r = divmod(seen[0], every)
                    if r == 0 and j < n_pairs:
                        events[2 * j + (0 if start else 1)].record(
                            torch.cuda.current_stream(self.device))
                    if not start:
                        seen[0] += 1
            left = steps
            while left > 0:
                k = min(left, self.max_block)
                self.block(k, spikes_out=spikes_out if k == left else None, timer=timer,
                           rows=nrows)
                left -= k
            return
        self._sync_trials()
        st = torch.cuda.current_stream(self.device)
        ev_arr, n_pairs = None, 0
        if events:
            for e in events:  # materialize the event handles on this stream
                e.record(st)
            n_pairs = len(events) // 2
            ev_arr = (ctypes.c_void_p * (2 * n_pairs))(*[e.cuda_event for e in events[:2 * n_pairs]])
        fn, name = self.lib.fis_advance, "fis_advance"
        if self.overlap and nrows > self.group:
            fn, name = self.lib.fis_advance_overlap, "fis_advance_overlap"
        rc = fn(ctypes.byref(self.desc), self.step, steps, self.group, nrows,
                ctypes.c_void_p(self.ring2.data_ptr()),
                ctypes.c_void_p(spikes_out.data_ptr()) if spikes_out is not None else None,
                ev_arr, n_pairs, max(1, int(every)), ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, name)
        self.step += steps

    def launches_per_block(self, rows=None):
        """Kernel launches of one block: per trial group the phase-A grid
        (scatter and Poisson drive) and the update."""
        nrows = self.batch if rows is None else max(1, min(int(rows), self.batch))
        return 2 * (-(-nrows // self.group))

    # --- readouts -------------------------------------------------------------

    def spikes_at(self, step=None, out=None):
        """Spikes of global step ``step`` (default: the last one) as float [B][N]."""
        step = self.step - 1 if step is None else int(step)
        if not (self.step - self.lag <= step < self.step) or step < 0:
            raise ValueError("step %d is not among the last %d" % (step, self.lag))
        if not self.raster and step != self.step - 1:
            raise ValueError("this core keeps the raster of its last step only (raster=False)")
        if out is None:
            out = torch.empty((self.batch, self.n), dtype=torch.float32, device=self.device)
        rc = self.lib.fis_spikes_f32(ctypes.byref(self.desc), 0, self.batch, step,
                                     ctypes.c_void_p(out.data_ptr()),
                                     ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream))
        _lib.check(rc, "fis_spikes_f32")
        return out

    def delay_buffer(self):
        """The reference's ``delay_buffer`` [B][buf_len][N] float32 (sim.py:385)."""
        self._sync_trials()
        R, n, B = self.buf_len, self.n, self.batch
        out = torch.empty((B, R, n), dtype=torch.float32, device=self.device)
        per = max(1, min(B, (256 << 20) // (R * n * 4)))
        st = torch.cuda.current_stream(self.device).cuda_stream
        for b0 in range(0, B, per):
            nb = min(per, B - b0)
            scratch = torch.zeros((R, nb, n), dtype=torch.int32, device=self.device)
            if self.pending is not None:
                p0, rows = self.pending
                for j in range(R):
                    s = p0 + j
                    if s >= self.step:
                        scratch[s % R] += rows[j, b0:b0 + nb]
            rc = self.lib.fis_delay_buffer(ctypes.byref(self.desc), b0, nb,
                                           ctypes.c_void_p(scratch.data_ptr()),
                                           ctypes.c_void_p(out[b0].data_ptr()),
                                           ctypes.c_void_p(st))
            _lib.check(rc, "fis_delay_buffer")
        return out

    # --- restore path -----------------------------------------------------------

    def load_state(self, step, v=None, g=None, refrac=None, spikes=None, ring_counts=None):
        """Put a state in place at global step ``step`` (restore path).

        ``ring_counts`` int32 [B][buf_len][N] in the reference's slot order:
        slot ``s % buf_len`` holds the input of step ``s``.  ``spikes`` are the
        spikes of step ``step - 1`` and are queued for delivery.
        """
        step = int(step)
        self.set_clock(step)
        for dst, src in ((self.v, v), (self.g, g), (self.refrac, refrac)):
            if src is not None:
                dst.copy_(src)
        self.list_len.zero_()
        self.bits.zero_()
        if ring_counts is not None:
            R = self.buf_len
            order = [(step + j) % R for j in range(R)]
            rows = ring_counts.permute(1, 0, 2)[order].contiguous()
            self.pending = (step, rows) if bool(rows.any()) else None
        else:
            self.pending = None
        if spikes is not None and step >= 1:
            rc = self.lib.fis_load_spikes(ctypes.byref(self.desc), 0, self.batch,
                                          ctypes.c_void_p(spikes.contiguous().data_ptr()),
                                          ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream))
            _lib.check(rc, "fis_load_spikes")
