"""The reference's ``flybrain.sim`` surface, backed by the B200 engine.

Same names, arguments, attributes and error behaviour as
``lab/flybrain/sim.py`` for the hot path: ``MODEL_PARAMS``, ``DT``,
``Stimulus``, ``RunConfig``, ``Result``, ``Engine`` (``step``, ``set_masks``,
``snapshot``, ``restore``, ``use_graphs``, ``fan``, ``mask_counts``,
``masks_clear``, ``spmv_info``), ``build_engine``, ``run``, ``save``,
``load``, ``check_rates_hz`` / ``RateTooHigh``.  Callers of the reference
(the worker, the closed loop, the probes) switch by importing this module
instead.

What is different, and why:

* there is no CPU path: ``device`` must be CUDA, and a missing library raises
  :class:`fis.evspmv.EventKernelUnavailable` (the reference's loud failure);
* the Poisson drive is a counter-based Philox stream keyed by (seed, trial,
  own step, neuron) instead of torch's generator, so ``gen`` holds that key;
  the draws of one trial do not depend on what else runs in the batch;
* ``delay_buffer``, ``ptr`` and the float masks are read-only views
  materialized from the engine's own state (an int32 spike history and one
  flag byte per neuron); ``restore`` is the way to change them;
* ``use_graphs`` captures one CUDA graph (the device keeps its own step
  counter, so one graph serves every ring position, where the reference
  needs 19);
* writing into ``spikes`` between steps (graded values, visdyn.py:660-676)
  raises unless the engine was built with ``graded=True``, which selects the
  reference's float path (its csrmv summation order, a float and writable
  ``delay_buffer``, no CUDA graphs) instead of the exact integer engine.
"""

from __future__ import annotations

import ctypes
import json
import os
import time
from dataclasses import asdict, dataclass, field
from pathlib import Path

import numpy as np
import torch

from . import _lib
from . import connectome as C
from . import evspmv
from .engine import DT, MODEL_PARAMS, Core, lif_params, require_cuda

FAST = "быстрый"
REFERENCE = "эталонный"
SPMV_CSR = "эталонный"
SPMV_EVENT = "событийный"
SPMV_CHOICES = (SPMV_CSR, SPMV_EVENT)
SPMV_DEFAULT = SPMV_EVENT

# Rate guard (reference sim.py:131-161).  The engine itself never asserts on
# the device, but the limit and its check are kept so callers see the same
# refusal at the same place: at the writer of the rates, on the host.
MAX_RATE_HZ = 1000.0 / DT


class RateTooHigh(ValueError):
    """A drive rate outside [0, 10 kHz] (reference sim.py:127-128)."""


def check_rates_hz(values, where):
    """Check rates before they are written; loud, names the place.

    Same contract as the reference (sim.py:131-161); NaN is refused too.
    """
    a = np.asarray(values, dtype=np.float64)
    if a.size == 0:
        return values
    if np.isnan(a).any():
        raise RateTooHigh("%s: drive rate is NaN" % where)
    worst, least = float(a.max()), float(a.min())
    if not (least >= 0.0) or worst > MAX_RATE_HZ:
        raise RateTooHigh(
            "%s: drive rate %.4g Hz (lowest %.4g) outside [0, %.0f]; p = rate * DT/1000 "
            "must stay a probability" % (where, worst, least, MAX_RATE_HZ))
    return values


@dataclass
class Stimulus:
    """Poisson drive into a set of neurons, optionally time-windowed."""

    indices: np.ndarray
    rate_hz: float = 200.0
    t_on_ms: float = 0.0
    t_off_ms: float | None = None
    name: str = "stim"

    def to_dict(self, with_indices=False):
        """The stimulus as a JSON-ready record (the reference's keys)."""
        idx = np.asarray(self.indices).ravel()
        rec = {"name": self.name, "n": int(idx.size)}
        rec.update((k, getattr(self, k)) for k in ("rate_hz", "t_on_ms", "t_off_ms"))
        if with_indices:
            rec["indices"] = idx.astype(np.int64).tolist()
        return rec


@dataclass
class RunConfig:
    t_run_s: float = 1.0
    bin_ms: float = 10.0
    n_trials: int = 1
    seed: int = 0
    device: str | None = None
    params: dict = field(default_factory=lambda: dict(MODEL_PARAMS))
    speed: str = FAST
    spmv: str | None = None


# Neuron annotation columns a rate table carries when they are present.
ANNOTATION_COLUMNS = ("root_id", "label", "cell_class", "super_class", "region",
                      "super_region", "side", "top_nt")


@dataclass
class Result:
    """Outcome of one run: per-neuron rates plus a neuron x time-bin raster.

    ``counts`` int64 [N] spikes per neuron summed over trials; ``bins`` int16
    [n_bins, N] spikes per bin summed over trials (the reference's fields,
    sim.py:255-321).
    """

    counts: np.ndarray
    bins: np.ndarray
    config: RunConfig
    stimuli: list
    silenced: np.ndarray
    neurons: object
    timing: dict

    @property
    def n_bins(self):
        return int(np.shape(self.bins)[0])

    @property
    def rates(self):
        """Firing rate in Hz per neuron, averaged over trials."""
        trial_seconds = self.config.t_run_s * self.config.n_trials
        return np.asarray(self.counts) / trial_seconds

    def active(self, min_rate=0.5):
        """Indices of the neurons firing at ``min_rate`` Hz or more."""
        return np.flatnonzero(self.rates >= min_rate)

    def rate_table(self, min_rate=0.5):
        """Active neurons with their annotations, fastest first."""
        import pandas as pd

        idx = self.active(min_rate)
        table = pd.DataFrame(index=pd.Index(idx))
        if self.neurons is not None:
            keep = [c for c in ANNOTATION_COLUMNS if c in self.neurons.columns]
            table = self.neurons.loc[idx, keep].copy()
        table["rate_hz"] = self.rates[idx]
        table["n_spikes"] = np.asarray(self.counts)[idx]
        return table.sort_values("rate_hz", ascending=False)

    def region_timeline(self):
        """DataFrame region x bin of the mean firing rate in Hz."""
        import pandas as pd

        per_neuron = pd.DataFrame(np.asarray(self.bins, dtype=np.float64).T,
                                  index=self.neurons["region"].to_numpy())
        mean_count = per_neuron.groupby(level=0, sort=False).mean()
        seconds = self.config.bin_ms / 1000.0 * self.config.n_trials
        return mean_count / seconds

    def meta(self, with_indices=False):
        """The run record written to meta.json (the reference's keys)."""
        cfg = asdict(self.config)
        params = cfg.pop("params")
        sil = np.asarray(self.silenced).astype(np.int64)
        rates = self.rates
        return {
            "config": cfg,
            "params": params,
            "stimuli": [s.to_dict(with_indices) for s in self.stimuli],
            "silenced": sil.tolist() if with_indices else None,
            "n_silenced": int(sil.size),
            "timing": self.timing,
            "n_neurons": int(np.size(self.counts)),
            "n_active": int(np.count_nonzero(rates >= 0.5)),
            "total_spikes": int(np.sum(self.counts)),
        }


class PhiloxState:
    """The drive's generator: a Philox key and counter base per trial.

    Stands where the reference keeps a ``torch.Generator`` (sim.py:354-355).
    ``get_state``/``set_state`` exchange a uint8 tensor, as torch's do.
    """

    MAGIC = b"FISPHLX1"

    def __init__(self, core: Core):
        self._core = core

    def manual_seed(self, seed):
        for b in range(self._core.batch):
            self._core.trials[b].seed = int(seed) & (2 ** 64 - 1)
        self._core.mark_trials()
        return self

    def get_state(self):
        c = self._core
        B = c.batch
        rec = np.zeros(B, dtype=[("seed", "<u8"), ("stream", "<u4"), ("own", "<i8")])
        for b in range(B):
            rec[b] = (c.trials[b].seed, c.trials[b].stream, c.step - c.trials[b].start)
        raw = self.MAGIC + np.int32(B).tobytes() + rec.tobytes()
        return torch.frombuffer(bytearray(raw), dtype=torch.uint8).clone()

    @classmethod
    def parse(cls, state):
        raw = bytes(np.asarray(state, dtype=np.uint8).tobytes())
        if not raw.startswith(cls.MAGIC):
            raise ValueError(
                "generator state is not this engine's (a torch generator state cannot "
                "seed the Philox drive); restore with drop=('gen',) to keep the current one")
        B = int(np.frombuffer(raw[8:12], dtype=np.int32)[0])
        rec = np.frombuffer(raw[12:], dtype=[("seed", "<u8"), ("stream", "<u4"), ("own", "<i8")])
        if rec.shape[0] != B:
            raise ValueError("corrupt generator state")
        return rec


def _warm(device):
    """Load the kernels once per device before a graph capture."""
    key = str(device)
    if key in _warm.done:
        return
    n = 64
    rp = np.zeros(n + 1, dtype=np.int64)
    rp[1:] = 1
    conn = C.Connectome(n, rp, np.array([1], dtype=np.int32), np.array([1], dtype=np.int32))
    core = Core(conn, 1, device=device, group=1)
    out = torch.zeros((1, n), device=core.device)
    core.block(2, spikes_out=out)
    core.spikes_at()
    torch.cuda.synchronize(core.device)
    _warm.done.add(key)


_warm.done = set()


def _index(idx, device):
    return torch.as_tensor(np.asarray(idx, dtype=np.int64), device=device)


class Engine:
    """One brain (B trials), held in a state you can step forward.

    Reference: ``sim.Engine`` (sim.py:338-953).  By default the step is the
    exact integer engine, which carries whole spikes and refuses a caller's
    write into ``spikes``.  ``graded=True`` opts into the reference's float
    path for callers that write fractional spikes between steps
    (visdyn.py:660-676): the csrmv product of the spikes as written, in the
    reference's summation order, and a float delay ring; one step per call,
    no CUDA graphs.
    """

    STATE_TENSORS = ("v", "conductance", "spikes", "refrac", "delay_buffer")
    MASK_TENSORS = ("m_fire", "m_out", "m_in", "m_hold", "v_hold")

    def __init__(self, weights, n, params=None, device="cuda", batch=1, seed=0,
                 no_refractory=None, spmv=None, allow_inexact=False, group=None, ring=None,
                 graded=False):
        p = dict(params or MODEL_PARAMS)
        self.p = p
        self.n = int(n)
        self.batch = int(batch)
        name = SPMV_DEFAULT if spmv is None else str(spmv)
        if name not in SPMV_CHOICES:
            raise ValueError("spmv %r not in %s" % (name, SPMV_CHOICES))
        try:
            dev = require_cuda(device)
        except _lib.KernelUnavailable as exc:
            raise evspmv.EventKernelUnavailable(str(exc)) from exc
        self.device = "cuda" if dev.index == torch.cuda.current_device() else str(dev)
        if isinstance(weights, C.Connectome):
            conn = weights
            if conn.n != self.n:
                raise ValueError("n = %d but the connectome has %d neurons" % (n, conn.n))
        else:
            try:
                conn = C.from_weights(weights, self.n)
            except C.ConnectomeError as exc:
                raise evspmv.EventKernelUnavailable(
                    "%s; this engine is exact integer accumulation only%s"
                    % (exc, " (allow_inexact is not offered)" if allow_inexact else "")) from exc
        self._conn = conn
        self._exact = conn.exactness()
        try:
            self.core = Core(conn, self.batch, params=p, device=dev, group=group, ring=ring)
        except _lib.KernelUnavailable as exc:
            raise evspmv.EventKernelUnavailable(str(exc)) from exc
        c = self.core
        self.gen = PhiloxState(c).manual_seed(seed)
        self.tau_syn_f = DT / p["tauSyn"]
        self.tau_mem_f = DT / p["tauMem"]
        self.prob_scale = DT / 1000.0
        self.poisson_gain = p["scalePoisson"]
        self.w_scale = p["wScale"]
        self.v_rest, self.v_reset = p["vRest"], p["vReset"]
        self.v_th = p["vThreshold"]
        self.buf_len = c.buf_len
        self.refrac_steps = torch.full((self.n,), float(round(p["tRefrac"] / DT)),
                                       dtype=torch.float32, device=c.device)
        if no_refractory is not None and len(no_refractory):
            free = (no_refractory.to(device=c.device, dtype=torch.long)
                    if torch.is_tensor(no_refractory) else _index(no_refractory, c.device))
            self.refrac_steps[free] = 0.0
            c.flags[:, free] |= _lib.FIS_FL_NOREFRAC
        c.reset_slots(slice(None))
        self.v = c.v
        self.conductance = c.g
        self.refrac = c.refrac
        self.spikes = torch.zeros((self.batch, self.n), dtype=torch.float32, device=c.device)
        self._spikes_version = self.spikes._version
        self._graphs = None
        self._vstim = None
        self._pool = None
        self._ev = None
        self.spmv = name
        self.calls = 0
        # Graded-spike mode (an explicit opt-in): the reference's float path,
        # for callers that write fractional values into `spikes` between
        # steps (visdyn.py:660-676).  The weights as CSR by postsynaptic
        # neuron (presynaptic indices ascending in a row), the reference's
        # float delay ring [B][buf_len][N], and the product's scratch.
        self.graded = bool(graded)
        if self.graded:
            dev = c.device
            self._t_csr = tuple(torch.from_numpy(a).to(dev) for a in conn.by_post())
            self._fring = torch.zeros((self.batch, self.buf_len, self.n), dtype=torch.float32,
                                      device=dev)
            # the product [B][N], then the nonzero mask [B][ceil(N/32)] words
            self._rec = torch.empty(self.batch * (self.n + (self.n + 31) // 32),
                                    dtype=torch.float32, device=dev)

    # --- views of the engine's own state ---------------------------------

    @property
    def ptr(self):
        return self.core.step % self.buf_len

    @ptr.setter
    def ptr(self, value):
        raise AttributeError("ptr follows the engine's step counter; set it through restore()")

    @property
    def delay_buffer(self):
        if self.graded:
            return self._fring
        return self.core.delay_buffer()

    def _mask(self, bit):
        return ((self.core.flags & bit) == 0).to(torch.float32)

    @property
    def m_fire(self):
        return self._mask(_lib.FIS_FL_FIRE_OFF)

    @property
    def m_out(self):
        return self._mask(_lib.FIS_FL_OUT_OFF)

    @property
    def m_in(self):
        return self._mask(_lib.FIS_FL_IN_OFF)

    @property
    def m_hold(self):
        return self._mask(_lib.FIS_FL_HOLD)

    @property
    def v_hold(self):
        c = self.core
        clamp = torch.tensor([c.trials[b].v_clamp for b in range(c.batch)],
                             dtype=torch.float32, device=c.device)[:, None]
        held = (c.flags & _lib.FIS_FL_HOLD) != 0
        return torch.where(held, clamp.expand_as(c.v), torch.zeros((), device=c.device))

    @property
    def w_csr(self):
        got = getattr(self, "_w_csr", None)
        if got is None:
            import warnings
            with warnings.catch_warnings():
                warnings.filterwarnings("ignore", message=".*[Ss]parse.*")
                got = self._w_csr = self._conn.to_torch_weights(self.core.device).to_sparse_csr()
        return got

    # --- the event product ----------------------------------------------

    def spmv_info(self):
        """How the recurrent product was computed, for the run record."""
        return {
            "умножение связей": self.spmv,
            "побитовое равенство обеспечено": bool(self._exact["ok"]),
            "условия равенства": evspmv.exactness_from(self._exact),
            "сборка ядра": {"библиотека": str(_lib.LIB_PATH.name), "abi": _lib.FIS_ABI_VERSION,
                            "цель": "sm_100a",
                            "кольцо": ("int16 со смещением" if self.core.ring16 else "int32")
                            + ", блок до 20 шагов",
                            "группа проб": self.core.group},
        }

    # --- interventions ----------------------------------------------------

    def set_masks(self, fire=None, out=None, inc=None, hold=None, v_clamp=None):
        """Set the intervention masks by neuron index lists (sim.py:510-593).

        ``fire``: no spike is emitted; ``out``: the spike reaches no synapse;
        ``inc``: delayed input is discarded; ``hold``: the membrane is replaced
        by ``v_clamp`` (default ``vReset``) before the threshold.  An empty list
        lifts the intervention, ``None`` leaves it as it is.  Delay tails are the
        reference's: ``out`` 19 steps, ``fire`` 20, ``inc`` and ``hold`` none.
        """
        c = self.core
        for bit, idx in ((_lib.FIS_FL_FIRE_OFF, fire), (_lib.FIS_FL_OUT_OFF, out),
                         (_lib.FIS_FL_IN_OFF, inc), (_lib.FIS_FL_HOLD, hold)):
            if idx is None:
                continue
            c.flags &= (~bit) & 0xFF
            if len(idx):
                c.flags[:, _index(idx, c.device)] |= bit
        if hold is not None:
            self._v_clamp = self.v_reset if v_clamp is None else float(v_clamp)
            for b in range(c.batch):
                c.trials[b].v_clamp = float(np.float32(self._v_clamp))
            c.mark_trials()

    def fan(self):
        """In- and out-degree of every neuron (sim.py:595-615)."""
        got = getattr(self, "_fan", None)
        if got is None:
            dev = self.core.device
            n_out = torch.from_numpy(self._conn.out_degree().astype(np.int64)).to(dev)
            n_in = torch.from_numpy(np.bincount(self._conn.col, minlength=self.n)
                                    .astype(np.int64)).to(dev)
            got = self._fan = (n_in, n_out)
        return got

    def mask_counts(self):
        f = self.core.flags[0]
        return {
            "не выдают спайк": int(((f & _lib.FIS_FL_FIRE_OFF) != 0).sum()),
            "исходящие отключены": int(((f & _lib.FIS_FL_OUT_OFF) != 0).sum()),
            "входящие отключены": int(((f & _lib.FIS_FL_IN_OFF) != 0).sum()),
            "мембрана удержана": int(((f & _lib.FIS_FL_HOLD) != 0).sum()),
        }

    def masks_clear(self):
        bits = (_lib.FIS_FL_FIRE_OFF | _lib.FIS_FL_OUT_OFF | _lib.FIS_FL_IN_OFF
                | _lib.FIS_FL_HOLD)
        return not bool(((self.core.flags & bits) != 0).any())

    def advance_ptr(self):
        raise AttributeError("the ring position advances with step(); it cannot be moved alone")

    # --- stepping ------------------------------------------------------------

    def _check_spikes_untouched(self):
        if self.spikes._version != self._spikes_version:
            raise RuntimeError(
                "Engine.spikes was written by the caller; graded or edited spikes are not "
                "supported by the exact integer engine (restore() sets a 0/1 spike state; "
                "build the engine with graded=True for the reference's float path)")

    def _graded_step(self, rates=None, vstim=None):
        """One step of the graded-spike mode (fis_graded_step): the product of
        the spikes as they are now, fractional values included."""
        c = self.core
        c._sync_trials()
        t_ptr, t_pre, t_val = self._t_csr
        saved = c.desc.rates
        if rates is not None:
            c.desc.rates = rates.data_ptr()
        try:
            rc = c.lib.fis_graded_step(
                ctypes.byref(c.desc), c.step, ctypes.c_void_p(t_ptr.data_ptr()),
                ctypes.c_void_p(t_pre.data_ptr()), ctypes.c_void_p(t_val.data_ptr()),
                ctypes.c_void_p(self.spikes.data_ptr()), ctypes.c_void_p(self._fring.data_ptr()),
                self.ptr, ctypes.c_void_p(self._rec.data_ptr()),
                ctypes.c_void_p(vstim.data_ptr()) if vstim is not None else None,
                ctypes.c_void_p(torch.cuda.current_stream(c.device).cuda_stream))
        finally:
            c.desc.rates = saved
        _lib.check(rc, "fis_graded_step")
        c.step += 1
        self.calls += 1

    def _rates_arg(self, rates):
        c = self.core
        if rates.shape != (self.batch, self.n):
            raise ValueError("rates must be [%d, %d], got %s"
                             % (self.batch, self.n, tuple(rates.shape)))
        if rates.device != c.device or rates.dtype != torch.float32 or not rates.is_contiguous():
            rates = rates.to(device=c.device, dtype=torch.float32).contiguous()
        return rates

    def step(self, rates):
        """Advance one 0.1 ms tick; ``rates`` [batch, n] in Hz (sim.py:745-771)."""
        if self.graded:
            self._graded_step(rates=self._rates_arg(rates))
            return self.spikes
        self._check_spikes_untouched()
        self.calls += 1
        c = self.core
        r = self._rates_arg(rates)
        if self._graphs is not None and c.pending is None:
            c._sync_trials()
            self._vstim.copy_(r)
            self._graphs[0].replay()
            c.step += 1
        else:
            c.desc.rates = r.data_ptr()
            try:
                c.block(1, spikes_out=self.spikes)
            finally:
                c.desc.rates = c.rates.data_ptr()
        self._spikes_version = self.spikes._version
        return self.spikes

    def _core(self, voltage_stim):
        """One step with an explicit drive tape instead of the Philox draw.

        The reference's deterministic half of the step (sim.py:863-953): the
        caller supplies ``voltage_stim`` [batch, n] (``w * (bern * gain)``).
        """
        if self.graded:
            self._graded_step(vstim=self._rates_arg(voltage_stim))
            return self.spikes
        self._check_spikes_untouched()
        c = self.core
        vs = self._rates_arg(voltage_stim)
        c.desc.vstim = vs.data_ptr()
        try:
            c.block(1, spikes_out=self.spikes)
        finally:
            c.desc.vstim = None
        self._spikes_version = self.spikes._version
        return self.spikes

    def run_block(self, rates, steps):
        """``steps`` ticks at constant ``rates``; returns the summed spikes [B, N].

        The closed loop's brain step (``body.py:1908-1912``: ``acc +=
        engine.step(rates)[0]`` 200 times per 20 ms control step) as one call:
        the steps run in 20-step fused blocks and the spikes are summed on the
        device by the update kernel, with no host work between steps.  Equal to
        stepping one by one; ``spikes`` holds the last step afterwards.  In
        graded-spike mode the steps run one by one.
        """
        if self.graded:
            r = self._rates_arg(rates)
            acc = torch.zeros((self.batch, self.n), dtype=torch.float32, device=self.core.device)
            for _ in range(int(steps)):
                self._graded_step(rates=r)
                acc += self.spikes
            return acc
        self._check_spikes_untouched()
        c = self.core
        r = self._rates_arg(rates)
        steps = int(steps)
        acc = torch.zeros((self.batch, self.n), dtype=torch.int32, device=c.device)
        saved = [(c.trials[b].rec, c.trials[b].bin_steps, c.trials[b].n_bins)
                 for b in range(self.batch)]
        recs, n_recs = c.recs, c.desc.n_recs
        c.set_recordings([acc[b:b + 1] for b in range(self.batch)])
        for b in range(self.batch):
            c.trials[b].rec, c.trials[b].bin_steps, c.trials[b].n_bins = b, 0x7FFFFFFF, 1
        c.mark_trials()
        c.desc.rates = r.data_ptr()
        try:
            c.advance(steps, spikes_out=self.spikes)
        finally:
            c.desc.rates = c.rates.data_ptr()
            for b, (rec, bs, nb) in enumerate(saved):
                c.trials[b].rec, c.trials[b].bin_steps, c.trials[b].n_bins = rec, bs, nb
            c.mark_trials()
            c.set_recordings(recs)
        self.calls += steps
        self._spikes_version = self.spikes._version
        return acc.to(torch.float32)

    def use_graphs(self, enable=True):
        """Capture the step into a CUDA graph (sim.py:634-743).  Returns
        whether graphs are in use; the graded-spike mode steps without them."""
        if self.graded:
            return False
        if not enable:
            self._graphs = self._vstim = self._pool = None
            return False
        if self._graphs is not None:
            return True
        c = self.core
        _warm(c.device)
        c._sync_trials()
        self._vstim = torch.zeros((self.batch, self.n), dtype=torch.float32, device=c.device)
        g = torch.cuda.CUDAGraph()
        saved = c.desc.rates
        c.desc.rates = self._vstim.data_ptr()
        step0 = c.step
        try:
            torch.cuda.synchronize(c.device)
            with torch.cuda.graph(g):
                c.block(1, spikes_out=self.spikes)
        except BaseException:
            self._vstim = None
            c.step = step0
            raise
        finally:
            c.desc.rates = saved
        c.step = step0  # the capture did not run anything
        self._graphs = [g]
        return True

    # --- whole state ----------------------------------------------------------

    def snapshot(self):
        """State as host arrays (sim.py:780-814): the reference's names and layouts."""
        out = {name: getattr(self, name).detach().cpu().numpy().copy()
               for name in self.STATE_TENSORS}
        for name in self.MASK_TENSORS:
            out[name] = getattr(self, name).detach().cpu().numpy().copy()
        out["ptr"] = np.int64(self.ptr)
        out["gen"] = self.gen.get_state().cpu().numpy().copy()
        out["calls"] = np.int64(self.calls)
        return out

    def restore(self, state, drop=()):
        """Put a state in place; returns the names restored (sim.py:816-846)."""
        c = self.core
        cur = None
        done = []

        def want(name):
            return name not in drop and name in state

        def cur_state():
            nonlocal cur
            if cur is None:
                cur = self.snapshot()
            return cur

        def arr(name):
            src = state[name] if want(name) else cur_state()[name]
            return torch.as_tensor(np.asarray(src), dtype=torch.float32, device=c.device)

        # masks first: they are flag bits here, and must be exact 0/1 floats
        masks = {}
        for name in self.MASK_TENSORS:
            if want(name):
                masks[name] = np.asarray(state[name], dtype=np.float32)
        for name, bit in (("m_fire", _lib.FIS_FL_FIRE_OFF), ("m_out", _lib.FIS_FL_OUT_OFF),
                          ("m_in", _lib.FIS_FL_IN_OFF), ("m_hold", _lib.FIS_FL_HOLD)):
            if name in masks:
                m = masks[name]
                if not np.all((m == 0.0) | (m == 1.0)):
                    raise ValueError("%s holds values other than 0 and 1" % name)
        v_hold = masks.get("v_hold")
        m_hold = masks.get("m_hold")
        if v_hold is not None:
            held = (m_hold == 0.0) if m_hold is not None else (
                (c.flags & _lib.FIS_FL_HOLD) != 0).cpu().numpy()
            for b in range(c.batch):
                vals = np.unique(v_hold[b][held[b]])
                if np.any(v_hold[b][~held[b]] != 0.0) or vals.size > 1:
                    raise ValueError("v_hold must be one clamp value per trial on held neurons")
                if vals.size:
                    c.trials[b].v_clamp = float(vals[0])
            c.mark_trials()
        for name, bit in (("m_fire", _lib.FIS_FL_FIRE_OFF), ("m_out", _lib.FIS_FL_OUT_OFF),
                          ("m_in", _lib.FIS_FL_IN_OFF), ("m_hold", _lib.FIS_FL_HOLD)):
            if name in masks:
                off = torch.as_tensor(masks[name] == 0.0, device=c.device)
                c.flags &= (~bit) & 0xFF
                c.flags |= off.to(torch.uint8) * bit
                done.append(name)
        if v_hold is not None:
            done.append("v_hold")

        v, g, refrac = arr("v"), arr("conductance"), arr("refrac")
        spikes = arr("spikes")
        ring = arr("delay_buffer")
        counts = None
        if not self.graded:
            if not bool(((spikes == 0) | (spikes == 1)).all()):
                raise ValueError("spikes must be 0/1: the integer ring carries whole spikes "
                                 "only (the graded-spike mode takes any values)")
            w = np.float32(self.w_scale)
            counts = torch.round(ring / float(w)).to(torch.int32)
            back = (counts.to(torch.float32) * float(w))
            if not bool((back == ring).all()):
                raise ValueError("delay_buffer holds values that are not w_scale * integer "
                                 "counts (the graded-spike mode takes any values)")
        ptr = int(state["ptr"]) % self.buf_len if want("ptr") else self.ptr
        if want("gen"):
            rec = PhiloxState.parse(state["gen"])
            if rec.shape[0] != c.batch:
                raise ValueError("generator state is for %d trials" % rec.shape[0])
            own = rec["own"].astype(np.int64)
        else:
            rec = None
            own = np.array([c.step - c.trials[b].start for b in range(c.batch)], dtype=np.int64)
        # the new clock: at least the current one, in the restored ring position
        t = c.step + ((ptr - c.step) % self.buf_len)
        t = max(t, int(own.max()) if own.size else 0)
        t += (ptr - t) % self.buf_len
        for b in range(c.batch):
            if rec is not None:
                c.trials[b].seed = int(rec["seed"][b])
                c.trials[b].stream = int(rec["stream"][b])
            c.trials[b].start = t - int(own[b])
            # the spikes of step t-1 loaded below are this trial's, also when
            # its own step restarts at t (generator state dropped)
            c.trials[b].history = 1
        c.mark_trials()
        c._sync_trials()
        if self.graded:
            c.set_clock(t)
            c.v.copy_(v)
            c.g.copy_(g)
            c.refrac.copy_(refrac)
            self._fring.copy_(ring)
        else:
            c.load_state(t, v=v, g=g, refrac=refrac, spikes=spikes, ring_counts=counts)
        self.spikes.copy_(spikes)
        self._spikes_version = self.spikes._version
        for name in self.STATE_TENSORS:
            if want(name):
                done.append(name)
        if want("ptr"):
            done.append("ptr")
        if want("gen"):
            done.append("gen")
        return done


def connectome_of(weights=None):
    """The connectome a run or an engine is built on.

    ``weights`` is the reference's sparse ``W[post, pre]`` or a
    :class:`fis.connectome.Connectome`.  The reference loads FlyWire from its
    data directory when ``weights`` is None (sim.py:981-982, data.py:229-259);
    here that directory is named by the environment variable
    ``FIS_FLYWIRE_DATA`` (the upstream ``data`` folder with its connectivity
    parquet and completeness CSV), and without it ``weights`` is required.
    """
    if weights is None:
        data = os.environ.get("FIS_FLYWIRE_DATA")
        if not data:
            raise FileNotFoundError(
                "no connectome given: pass weights= (torch sparse W[post, pre] of synapse "
                "counts, or fis.connectome.Connectome), or set FIS_FLYWIRE_DATA to the "
                "upstream data folder")
        return C.from_upstream(data)
    return weights if isinstance(weights, C.Connectome) else C.from_weights(weights)


def build_engine(weights=None, neurons=None, silenced=None, params=None, device=None,
                 batch=1, seed=0, no_refractory=None, graphs=True, spmv=None,
                 allow_inexact=False, group=None, ring=None, graded=False):
    """Return a ready :class:`Engine` (sim.py:956-987).

    ``weights`` as :func:`connectome_of` takes it (None: the FlyWire folder
    named by ``FIS_FLYWIRE_DATA``).  ``graded=True`` builds the graded-spike
    mode of :class:`Engine`.
    """
    conn = connectome_of(weights)
    n = len(neurons) if neurons is not None else conn.n
    sil = np.asarray(silenced if silenced is not None else [], dtype=np.int64)
    conn = conn.without(sil)
    eng = Engine(conn, n, params=params, device=device or "cuda", batch=batch, seed=seed,
                 no_refractory=no_refractory, spmv=spmv, allow_inexact=allow_inexact,
                 group=group, ring=ring, graded=graded)
    if graphs:
        eng.use_graphs()
    return eng


def stim_schedule(stimuli, steps):
    """``(step, indices, rate)`` events sorted by step (sim.py:1021-1031)."""
    ev = []
    for s in stimuli:
        idx = np.asarray(s.indices, dtype=np.int64)
        on = int(round(s.t_on_ms / DT))
        off = steps if s.t_off_ms is None else int(round(s.t_off_ms / DT))
        ev.append((on, idx, float(s.rate_hz)))
        if off < steps:
            ev.append((off, idx, 0.0))
    ev.sort(key=lambda e: e[0])
    return ev


def run(stimuli, silenced=None, config: RunConfig | None = None, neurons=None, weights=None,
        progress=True, on_bin=None, should_stop=None):
    """Simulate and return a :class:`Result` (sim.py:990-1117).

    Binning happens on the device: each spike adds one to its (bin, neuron)
    counter inside the update kernel, so the host reads back only at bin
    boundaries where ``on_bin`` or ``should_stop`` ask for it.  ``weights``
    as :func:`connectome_of` takes it.  The steps run in fused blocks of up
    to 20 without CUDA graphs whatever ``config.speed`` says, so the
    timing record states ``"graphs": False``.
    """
    config = config or RunConfig()
    silenced = np.asarray([] if silenced is None else silenced, dtype=np.int64)
    conn = connectome_of(weights)
    n = len(neurons) if neurons is not None else conn.n
    device = config.device or "cuda"
    t0 = time.perf_counter()
    B = config.n_trials
    steps = int(round(config.t_run_s * 1000.0 / DT))
    bin_steps = max(1, int(round(config.bin_ms / DT)))
    n_bins = int(np.ceil(steps / bin_steps))
    events = stim_schedule(stimuli, steps)
    for _, _, rate in events:
        check_rates_hz(rate, "run: stimulus rate")
    stim_all = (np.concatenate([e[1] for e in events]) if events
                else np.zeros(0, dtype=np.int64))
    eng = build_engine(weights=conn, neurons=neurons, silenced=silenced,
                       params=config.params, device=device, batch=B, seed=config.seed,
                       no_refractory=stim_all, graphs=False, spmv=config.spmv)
    c = eng.core
    rec = torch.zeros((max(n_bins, 1), n), dtype=torch.int32, device=c.device)
    c.set_recordings([rec])
    for b in range(B):
        c.trials[b].rec = 0
        c.trials[b].bin_steps = bin_steps
        c.trials[b].n_bins = n_bins
    c.mark_trials()
    t_setup = time.perf_counter() - t0

    bar = None
    if progress:
        try:
            from tqdm import tqdm

            bar = tqdm(total=steps, unit="step", ncols=78, desc="sim")
        except ImportError:
            bar = None
    t1 = time.perf_counter()
    ev = 0
    step = 0
    stopped = steps
    while step < steps:
        while ev < len(events) and events[ev][0] == step:
            _, idx, rate = events[ev]
            if idx.size:
                c.rates[:, _index(idx, c.device)] = rate
            ev += 1
        nxt = steps
        if ev < len(events):
            nxt = min(nxt, events[ev][0])
        if on_bin is not None or should_stop is not None:
            nxt = min(nxt, (step // bin_steps + 1) * bin_steps)
        k = min(c.max_block, nxt - step)
        c.block(k, spikes_out=eng.spikes)
        step += k
        eng.calls += k
        if bar is not None:
            bar.update(k)
        if (on_bin is not None or should_stop is not None) and (
                step % bin_steps == 0 or step == steps):
            b = min((step - 1) // bin_steps, n_bins - 1)
            if on_bin is not None:
                on_bin(b, step * DT, rec[b].to(torch.int16).cpu().numpy())
            if should_stop is not None and should_stop():
                stopped = step
                break
    torch.cuda.synchronize(c.device)
    t_sim = time.perf_counter() - t1
    c.check_errors()
    if bar is not None:
        bar.close()
    eng._spikes_version = eng.spikes._version
    binned = rec[:n_bins].to(torch.int16)
    counts = rec[:n_bins].to(torch.int64).sum(0)
    timing = {
        "setup_s": round(t_setup, 3), "sim_s": round(t_sim, 3), "steps": stopped,
        "device": device,
        "realtime_ratio": round(config.t_run_s / t_sim, 4) if t_sim else None,
        "speed": getattr(config, "speed", FAST), "graphs": False,
        **eng.spmv_info(),
    }
    return Result(counts.cpu().numpy(), binned.cpu().numpy(), config, list(stimuli),
                  silenced, neurons, timing)


# The saved-run format (sim.py:1120-1174): meta.json (Result.meta with the
# indices), rates.parquet (the rate table of active neurons, indexed by
# neuron) and bins.npz (the active neurons' columns of the raster).
META_FILE, RATES_FILE, BINS_FILE = "meta.json", "rates.parquet", "bins.npz"


def save(result: Result, out_dir: Path, min_rate=0.5):
    """Write a run directory (meta.json, rates.parquet, bins.npz); returns it."""
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    record = json.dumps(result.meta(with_indices=True), ensure_ascii=False, indent=2)
    (out / META_FILE).write_text(record, encoding="utf-8")
    result.rate_table(min_rate).to_parquet(out / RATES_FILE)
    cols = result.active(min_rate)
    # t0_ms: model time of the first raster row (a windowed recording
    # states it in its timing record; an ordinary run starts at 0)
    t0 = (result.timing or {}).get("запись с, мс", 0.0)
    raster = np.asarray(result.bins)[:, cols].astype(np.int16)
    np.savez_compressed(out / BINS_FILE, neuron_idx=cols.astype(np.int32), bins=raster,
                        bin_ms=np.float32(result.config.bin_ms), t0_ms=np.float32(t0))
    return out


def load(out_dir, neurons=None, n=None) -> Result:
    """Rebuild a :class:`Result` from a run directory written by :func:`save`.

    The neuron count comes from ``neurons``, else ``n``, else the record's
    ``n_neurons``; neurons absent from the saved tables read as silent.
    """
    import pandas as pd

    where = Path(out_dir)
    meta = json.loads((where / META_FILE).read_text(encoding="utf-8"))
    size = len(neurons) if neurons is not None else int(n or meta["n_neurons"])
    table = pd.read_parquet(where / RATES_FILE)
    counts = np.zeros(size, dtype=np.int64)
    np.put(counts, table.index.to_numpy(), table["n_spikes"].to_numpy())
    with np.load(where / BINS_FILE) as z:
        cols, part = z["neuron_idx"], z["bins"]
    bins = np.zeros((part.shape[0], size), dtype=np.int16)
    bins[:, cols] = part
    config = RunConfig(params=meta["params"], **meta["config"])

    def stimulus(rec):
        idx = np.asarray(rec.get("indices", []), dtype=np.int64)
        return Stimulus(idx, **{k: rec[k] for k in ("rate_hz", "t_on_ms", "t_off_ms", "name")})

    silenced = np.asarray(meta.get("silenced") or [], dtype=np.int64)
    return Result(counts, bins, config, [stimulus(r) for r in meta["stimuli"]], silenced,
                  neurons, meta["timing"])


__all__ = ["MODEL_PARAMS", "DT", "FAST", "REFERENCE", "SPMV_CSR", "SPMV_EVENT",
           "SPMV_CHOICES", "SPMV_DEFAULT", "MAX_RATE_HZ", "RateTooHigh", "check_rates_hz",
           "Stimulus", "RunConfig", "Result", "Engine", "build_engine", "run", "save", "load",
           "lif_params"]
