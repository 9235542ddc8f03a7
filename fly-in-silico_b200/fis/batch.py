"""Many independent trials on one connectome: the batched form of the step.

The reference runs one engine per job and its trials share one stimulus set
(``lab/flybrain/sim.py:990-1117``, ``worker.py:454-505``).  Here every trial
slot carries its own Philox seed, stimulus set and rates, silencing, masks and
duration, and all slots advance together: each block reads the CSR rows of
the spikes that arrive in it once, and each neuron's state once per 20 steps.

A trial's result does not depend on the other slots: its drive is keyed by
its own seed and own step, its input comes only from its own spikes, and
integer accumulation makes the order of contributions irrelevant.  Per-trial
silencing is the flag FIS_FL_SILENCED, which has the effect of the reference's
``_silence`` (``sim.py:324-336``) on that trial alone.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .connectome import Connectome
from .engine import Core
from .sim import check_rates_hz


@dataclass
class TrialSpec:
    """One trial: drive, interventions, duration and seed."""

    seed: int
    steps: int
    stim: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))
    rate_hz: float | np.ndarray = 0.0
    silenced: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))
    no_refractory: np.ndarray | None = None  # None: the stimulated neurons (sim.run)
    fire_off: np.ndarray | None = None
    out_off: np.ndarray | None = None
    in_off: np.ndarray | None = None
    hold: np.ndarray | None = None
    v_clamp: float | None = None
    bin_steps: int | None = None             # None: one bin over the whole trial

    def n_bins(self):
        bs = self.bin_steps or max(1, self.steps)
        return max(1, -(-self.steps // bs))


def host_rows(specs, n):
    """Flags (uint8) and rates (float32) rows [len(specs)][n] built on the host."""
    k = len(specs)
    flags = np.zeros((k, n), dtype=np.uint8)
    rates = np.zeros((k, n), dtype=np.float32)
    for j, s in enumerate(specs):
        stim = np.asarray(s.stim, dtype=np.int64)
        r = np.asarray(s.rate_hz, dtype=np.float64)
        check_rates_hz(r, "trial %d rate" % j)
        rates[j, stim] = r.astype(np.float32)
        nore = stim if s.no_refractory is None else np.asarray(s.no_refractory, np.int64)
        flags[j, nore] |= _lib.FIS_FL_NOREFRAC
        flags[j, np.asarray(s.silenced, np.int64)] |= _lib.FIS_FL_SILENCED
        for idx, bit in ((s.fire_off, _lib.FIS_FL_FIRE_OFF), (s.out_off, _lib.FIS_FL_OUT_OFF),
                         (s.in_off, _lib.FIS_FL_IN_OFF), (s.hold, _lib.FIS_FL_HOLD)):
            if idx is not None and len(idx):
                flags[j, np.asarray(idx, np.int64)] |= bit
    return flags, rates


def sparse_rows(specs, n, slots):
    """The non-zero flags and rates of ``specs`` placed in ``slots``, sparse.

    Returns (flag_at, flag_bits, rate_at, rate_val): flat positions
    slot * n + neuron (int64, unique, ascending) with the OR of their flag bits
    (uint8), and the positions with a rate (int64, unique) with the rate as
    float32 (a repeated stimulated neuron keeps its last rate, as an indexed
    assignment does).  Together they equal ``host_rows`` laid into the slots.
    """
    f_at, f_bits, r_at, r_val = [], [], [], []
    for j, (b, s) in enumerate(zip(slots, specs)):
        base = int(b) * n
        stim = np.asarray(s.stim, dtype=np.int64)
        r = np.asarray(s.rate_hz, dtype=np.float64)
        check_rates_hz(r, "trial %d rate" % j)
        r_at.append(base + stim)
        r_val.append(np.broadcast_to(r.astype(np.float32), stim.shape))
        nore = stim if s.no_refractory is None else np.asarray(s.no_refractory, np.int64)
        for idx, bit in ((nore, _lib.FIS_FL_NOREFRAC), (s.silenced, _lib.FIS_FL_SILENCED),
                         (s.fire_off, _lib.FIS_FL_FIRE_OFF), (s.out_off, _lib.FIS_FL_OUT_OFF),
                         (s.in_off, _lib.FIS_FL_IN_OFF), (s.hold, _lib.FIS_FL_HOLD)):
            if idx is not None and len(idx):
                idx = np.asarray(idx, np.int64)
                f_at.append(base + idx)
                f_bits.append(np.full(idx.shape, bit, dtype=np.uint8))
    i64, u8, f32 = np.zeros(0, np.int64), np.zeros(0, np.uint8), np.zeros(0, np.float32)
    fa = np.concatenate(f_at) if f_at else i64
    fb = np.concatenate(f_bits) if f_bits else u8
    ra = np.concatenate(r_at) if r_at else i64
    rv = np.concatenate(r_val) if r_val else f32
    # One stable sort per array (skipped when the positions already ascend,
    # as a trial's sorted stimulus set in ascending slots does); runs of a
    # repeated position then merge: flag bits OR together, and a rate keeps
    # its last value, as an indexed assignment does.
    if fa.size and not np.all(fa[1:] > fa[:-1]):
        order = np.argsort(fa, kind="stable")
        fa, fb = fa[order], fb[order]
        first = np.flatnonzero(np.concatenate(([True], fa[1:] != fa[:-1])))
        fa = fa[first]
        fb = np.bitwise_or.reduceat(fb, first)
    if ra.size and not np.all(ra[1:] > ra[:-1]):
        order = np.argsort(ra, kind="stable")
        ra, rv = ra[order], rv[order]
        last = np.flatnonzero(np.concatenate((ra[1:] != ra[:-1], [True])))
        ra, rv = ra[last], rv[last]
    return fa, fb, ra, np.ascontiguousarray(rv)


class Batch:
    """Trial slots on one GPU; load specs, advance, read per-trial results.

    Recording buffers (int32 [n_bins][N], one atomic add per spike inside the
    update kernel) live in a registry: a trial records either into a buffer of
    its own or into one shared by the trials of a request (their spikes then
    sum, as the reference's bins sum over trials, ``sim.py:1068-1076``).
    """

    def __init__(self, conn: Connectome, capacity: int, params=None, device="cuda",
                 group=None, chunk=None, core: Core | None = None, drive_lists=None, **launch):
        # results come from recordings: no per-step raster needed.  `launch`:
        # the remaining Core arguments of a tuning result (ring,
        # scatter_mode, scat_ctas, drive_ctas).  `drive_lists`: phase A's
        # drive visits each trial's stimulated neurons only (the batch knows
        # them as it loads the trial) instead of scanning every rate.  By
        # default from 8 slots up: with phase A overlapped by other groups'
        # updates its shorter drive measured faster (64 trials: -1.8 % per
        # step); one trial alone, with nothing to overlap, waits for the
        # list's extra round trip instead (+4 % per step).
        self.core = core or Core(conn, capacity, params=params, device=device, group=group,
                                 chunk=chunk, raster=False, **launch)
        if drive_lists is None:
            drive_lists = self.core.batch >= 8
        if drive_lists:
            self.core.use_drive_lists()
        self.n = self.core.n
        self.capacity = self.core.batch
        self._copy_stream = None  # the side stream of the counts' copy to the host
        self._recs = {}                          # index -> int32 [n_bins][N]
        self._rec_refs = {}                      # index -> trials recording into it
        self._slot_rec = [None] * self.capacity  # slot -> index
        self._dummy_rec = None

    # --- recording registry ---------------------------------------------------

    def _rec_add(self, tensor, refs):
        idx = 0
        while idx in self._recs:
            idx += 1
        self._recs[idx] = tensor
        self._rec_refs[idx] = refs
        return idx

    def _rec_upload(self):
        if self._dummy_rec is None:
            self._dummy_rec = torch.zeros((1, self.n), dtype=torch.int32, device=self.core.device)
        top = max(self._recs) + 1 if self._recs else 0
        self.core.set_recordings([self._recs.get(i, self._dummy_rec) for i in range(top)])

    def release(self, slot):
        """Detach ``slot`` from its recording (freed with its last trial)."""
        idx = self._slot_rec[slot]
        self._slot_rec[slot] = None
        if idx is None:
            return
        self._rec_refs[idx] -= 1
        if self._rec_refs[idx] <= 0:
            del self._recs[idx]
            del self._rec_refs[idx]

    def recording(self, slot):
        """The recording buffer of ``slot`` (device int32 [n_bins][N])."""
        return self._recs[self._slot_rec[slot]]

    def recordings(self):
        return list(self._recs.values())

    # --- trials -------------------------------------------------------------------

    def _rows_host(self, specs, slots):
        """The sparse rows of ``specs`` in ``slots``, packed into one pinned buffer.

        Layout: int64 flag positions, int64 rate positions (8-byte aligned),
        float32 rates, uint8 flag bits.  The buffer comes from torch's caching
        host allocator, which keeps it until the copy that reads it has run.
        """
        fa, fb, ra, rv = sparse_rows(specs, self.n, slots)
        nbytes = 8 * (fa.size + ra.size) + 4 * rv.size + fb.size
        pin = torch.empty(max(8, -(-nbytes // 8) * 8), dtype=torch.uint8, pin_memory=True)
        host = pin.numpy()
        o1, o2 = 8 * fa.size, 8 * (fa.size + ra.size)
        o3 = o2 + 4 * rv.size
        host[:o1].view(np.int64)[:] = fa
        host[o1:o2].view(np.int64)[:] = ra
        host[o2:o3].view(np.float32)[:] = rv
        host[o3:o3 + fb.size] = fb
        return pin, nbytes, (o1, o2, o3, fa.size, ra.size, fb.size)

    def load(self, slots, specs, start=None, rec=None, staged=None):
        """Place ``specs`` into ``slots`` starting at global step ``start``.

        The trials' non-zero flags and rates travel sparse (positions and
        values, one pinned copy) and are laid into the zeroed rows on the
        device; state is reset to the reference's initial values.  ``rec``: a
        shared recording buffer for all these trials; by default each trial
        gets one of its own (views of one buffer when their bin counts agree).
        ``staged``: the rows already packed by ``_rows_host`` for these slots.
        """
        c = self.core
        slots = list(slots)
        k = len(slots)
        start = c.step if start is None else int(start)
        pin, nbytes, (o1, o2, o3, nfa, nra, nfb) = staged or self._rows_host(specs, slots)
        dev = pin[:nbytes].to(c.device, non_blocking=True)
        self.last_h2d_bytes = nbytes
        idx = torch.as_tensor(slots, dtype=torch.long, device=c.device)
        contiguous = slots == list(range(slots[0], slots[0] + k))
        rows = slice(slots[0], slots[0] + k) if contiguous else idx
        c.flags[rows] = 0
        c.rates[rows] = 0.0
        if nfa:
            c.flags.view(-1)[dev[:o1].view(torch.int64)] = dev[o3:o3 + nfb]
        if nra:
            c.rates.view(-1)[dev[o1:o2].view(torch.int64)] = dev[o2:o3].view(torch.float32)
        # the loaded trials' driven-neuron lists: the positions just written
        c.set_drive_lists_sparse(rows, dev[o1:o2].view(torch.int64))
        for b in slots:
            if self._slot_rec[b] is not None:
                self.release(b)
        shared = None
        if rec is not None:
            shared = self._rec_add(rec, k)
        bins = [s.n_bins() for s in specs]
        own = None
        if shared is None and len(set(bins)) == 1:
            own = torch.zeros((k, bins[0], self.n), dtype=torch.int32, device=c.device)
        self.last_recording = own  # [k][n_bins][N] in the order of `specs`, or None
        for j, (b, s) in enumerate(zip(slots, specs)):
            t = c.trials[b]
            t.seed = int(s.seed) & (2 ** 64 - 1)
            t.stream = 0
            t.start = start
            t.end = start + int(s.steps)
            t.history = 0
            t.v_clamp = float(np.float32(c.pdict["vReset"] if s.v_clamp is None else s.v_clamp))
            if shared is not None:
                ri, nb = shared, int(rec.shape[0])
            else:
                r = own[j] if own is not None else torch.zeros(
                    (bins[j], self.n), dtype=torch.int32, device=c.device)
                ri, nb = self._rec_add(r, 1), bins[j]
            self._slot_rec[b] = ri
            t.rec = ri
            t.bin_steps = int(s.bin_steps or max(1, s.steps))
            t.n_bins = nb
        self._rec_upload()
        c.mark_trials()
        c.reset_slots(rows)

    def _plan(self, specs):
        """Host side of a run: placement (longest first) and the packed rows."""
        k = len(specs)
        if k > self.capacity:
            raise ValueError("%d trials for %d slots" % (k, self.capacity))
        order = sorted(range(k), key=lambda j: -int(specs[j].steps))
        slots_of_run = [0] * k
        for slot, j in enumerate(order):
            slots_of_run[j] = slot
        placed = [specs[j] for j in order]
        return {"specs": placed, "slots_of_run": slots_of_run,
                "staged": self._rows_host(placed, list(range(k)))}

    def _launch(self, plan, timer=None):
        """Device side of a run, all enqueued: load, advance, per-trial counts
        into a pinned host buffer.  Returns the handle ``_finish`` waits on."""
        c = self.core
        placed = plan["specs"]
        k = len(placed)
        self.slots_of_run = plan["slots_of_run"]
        for b in range(k, self.capacity):   # idle slots do nothing
            c.trials[b].start = c.trials[b].end = 0
        self.load(range(k), placed, staged=plan["staged"])
        dur = [int(s.steps) for s in placed]
        G, K = c.group, c.max_block
        t, total = 0, dur[0] if dur else 0
        while t < total:
            active = sum(1 for d in dur if d > t)
            rows = min(self.capacity, -(-active // G) * G)
            nxt = dur[(rows - 1) // G * G]   # longest trial of the last group
            nxt = min(total, t + -(-(nxt - t) // K) * K)  # whole blocks
            c.advance(nxt - t, timer=timer, rows=rows)
            t = nxt
        out = torch.empty((k, self.n), dtype=torch.int32, pin_memory=True)
        if self.last_recording is not None:  # [k][n_bins][N], trials in slot order
            sums = self.last_recording.sum(1, dtype=torch.int32)
            pos = torch.as_tensor(self.slots_of_run, dtype=torch.long, device=c.device)
            dev = sums.index_select(0, pos)
        else:
            dev = torch.stack([self.recording(self.slots_of_run[j]).sum(0, dtype=torch.int32)
                               for j in range(k)])
        # The copy to the host (and of the error bits) runs on a side stream,
        # after the run, so that the next run's kernels do not queue behind it.
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream(c.device))
        if self._copy_stream is None:
            self._copy_stream = torch.cuda.Stream(c.device)
        cs = self._copy_stream
        cs.wait_event(ready)
        with torch.cuda.stream(cs):
            out.copy_(dev, non_blocking=True)
            errs = c.errors_async()
            done = torch.cuda.Event()
            done.record(cs)
        dev.record_stream(cs)
        self.last_d2h_bytes = out.numel() * out.element_size()
        return out, done, errs

    def _finish(self, handle):
        out, done, errs = handle
        done.synchronize()
        self.core.raise_errors(errs)
        # the pinned buffer itself, kept alive by the array: no second copy
        return out.numpy()

    def run(self, specs, timer=None):
        """Run ``specs`` (at most ``capacity``) to completion; host counts per trial.

        Trials are placed longest first, so the running ones always fill the
        lowest slots: once every trial of the last trial group has ended, that
        group is no longer launched.  ``slots_of_run[j]`` is the slot that ran
        ``specs[j]``.  Returns int32 [len(specs)][N] spike counts summed over
        each trial's bins, in the order of ``specs``, copied to the host.
        """
        return self._finish(self._launch(self._plan(specs), timer=timer))

    def run_many(self, spec_lists):
        """``run`` over several batches, one after another on the device.

        The device goes from one batch to the next without waiting for the
        host.  Enqueueing a batch blocks the host until the device's launch
        queue has room, i.e. until the batch is nearly done, so each batch is
        enqueued by a worker thread (bound to the caller's device and stream)
        while this thread packs the next batch's rows; this thread issues no
        device work until the worker has returned.  A batch's counts (and its
        error bits) are reduced and copied out in stream order before the next
        batch's load resets the slots.  Yields each batch's counts (as ``run``
        returns them) as it completes; ``slots_of_run`` then already
        describes the batch after it.
        """
        from concurrent.futures import ThreadPoolExecutor

        dev = self.core.device
        stream = torch.cuda.current_stream(dev)

        def launch(plan):
            with torch.cuda.device(dev), torch.cuda.stream(stream):
                return self._launch(plan)

        it = iter(spec_lists)
        specs = next(it, None)
        plan = self._plan(specs) if specs is not None else None
        pending = None
        with ThreadPoolExecutor(max_workers=1) as pool:
            while plan is not None:
                job = pool.submit(launch, plan)
                specs = next(it, None)
                plan = self._plan(specs) if specs is not None else None  # host only
                launched = job.result()
                if pending is not None:
                    yield self._finish(pending)
                pending = launched
        if pending is not None:
            yield self._finish(pending)


def random_specs(n, count, seed, steps, stim_range=(500, 5000), rate_range=(50.0, 300.0),
                 silenced_range=(1, 100)):
    """Seeded trial mix: own seed, stimulus set, rate and silencing per trial."""
    rng = np.random.default_rng(seed)
    specs = []
    for j in range(count):
        k = int(rng.integers(stim_range[0], stim_range[1] + 1))
        stim = np.sort(rng.choice(n, size=k, replace=False))
        rate = float(rng.uniform(*rate_range))
        ns = int(rng.integers(silenced_range[0], silenced_range[1] + 1))
        sil = np.sort(rng.choice(n, size=ns, replace=False))
        dur = steps if np.isscalar(steps) else int(rng.integers(steps[0], steps[1] + 1))
        specs.append(TrialSpec(seed=int(rng.integers(0, 2 ** 63)), steps=int(dur), stim=stim,
                               rate_hz=rate, silenced=sil))
    return specs
