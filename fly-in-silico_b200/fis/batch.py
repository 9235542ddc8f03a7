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


class Batch:
    """Trial slots on one GPU; load specs, advance, read per-trial results."""

    def __init__(self, conn: Connectome, capacity: int, params=None, device="cuda",
                 group=None, core: Core | None = None):
        self.core = core or Core(conn, capacity, params=params, device=device, group=group)
        self.n = self.core.n
        self.capacity = self.core.batch
        self._recs = [None] * self.capacity
        self._pinned = {}

    def _staging(self, name, shape, dtype):
        buf = self._pinned.get(name)
        if buf is None or buf.shape != shape:
            buf = torch.empty(shape, dtype=dtype, pin_memory=True)
            self._pinned[name] = buf
        return buf

    def load(self, slots, specs, start=None):
        """Place ``specs`` into ``slots`` starting at global step ``start``.

        Rows are built on the host and copied once (pinned, asynchronous);
        state is reset to the reference's initial values; each trial gets a
        recording buffer int32 [n_bins][N] of its own.
        """
        c = self.core
        slots = list(slots)
        start = c.step if start is None else int(start)
        flags, rates = host_rows(specs, self.n)
        fpin = self._staging("flags", flags.shape, torch.uint8)
        rpin = self._staging("rates", rates.shape, torch.float32)
        fpin.numpy()[:] = flags
        rpin.numpy()[:] = rates
        idx = torch.as_tensor(slots, dtype=torch.long, device=c.device)
        contiguous = slots == list(range(slots[0], slots[0] + len(slots)))
        if contiguous:
            c.flags[slots[0]:slots[0] + len(slots)].copy_(fpin, non_blocking=True)
            c.rates[slots[0]:slots[0] + len(slots)].copy_(rpin, non_blocking=True)
        else:
            c.flags[idx] = fpin.to(c.device, non_blocking=True)
            c.rates[idx] = rpin.to(c.device, non_blocking=True)
        for j, (b, s) in enumerate(zip(slots, specs)):
            t = c.trials[b]
            t.seed = int(s.seed) & (2 ** 64 - 1)
            t.stream = 0
            t.start = start
            t.end = start + int(s.steps)
            t.v_clamp = float(np.float32(c.pdict["vReset"] if s.v_clamp is None else s.v_clamp))
            nb = s.n_bins()
            rec = self._recs[b]
            if rec is None or rec.shape[0] != nb:
                rec = torch.zeros((nb, self.n), dtype=torch.int32, device=c.device)
                self._recs[b] = rec
            else:
                rec.zero_()
            t.rec = b
            t.bin_steps = int(s.bin_steps or max(1, s.steps))
            t.n_bins = nb
        c.set_recordings([r if r is not None else self._dummy() for r in self._recs])
        c.mark_trials()
        c.reset_slots(idx if not contiguous else slice(slots[0], slots[0] + len(slots)))

    def _dummy(self):
        d = getattr(self, "_dummy_rec", None)
        if d is None:
            d = self._dummy_rec = torch.zeros((1, self.n), dtype=torch.int32,
                                              device=self.core.device)
        return d

    def results(self, slots, out=None):
        """Per-slot recordings (device tensors int32 [n_bins][N])."""
        return [self._recs[b] for b in slots]

    def run(self, specs, timer=None):
        """Run ``specs`` (at most ``capacity``) to completion; host counts per trial.

        Returns int32 [len(specs)][N] spike counts summed over each trial's
        bins, copied to the host.
        """
        c = self.core
        if len(specs) > self.capacity:
            raise ValueError("%d trials for %d slots" % (len(specs), self.capacity))
        slots = list(range(len(specs)))
        for b in range(len(specs), self.capacity):   # idle slots do nothing
            c.trials[b].start = c.trials[b].end = 0
        self.load(slots, specs)
        c.advance(max(int(s.steps) for s in specs), timer=timer)
        out = self._staging("counts", (len(specs), self.n), torch.int32)
        dev = torch.stack([self._recs[b].sum(0, dtype=torch.int32) for b in slots])
        out.copy_(dev, non_blocking=True)
        torch.cuda.current_stream(c.device).synchronize()
        return out.numpy().copy()


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
