"""TEST INFRASTRUCTURE ONLY: Python face of the C oracle (lif_oracle.c).

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline use
this module, and only as the checker or the timed CPU reference; the product
(``fis``) never imports it.

It holds the reference's engine state in the reference's own layout
(``lab/flybrain/sim.py:383-411``): float32 ``v, conductance, spikes, refrac``
[B, N], ``delay_buffer`` [B, buf_len, N], integer ``ptr``, float masks
``m_fire, m_out, m_in, m_hold, v_hold`` [B, N] and per-(trial, neuron)
``refrac_steps``.  The model constants are derived here independently of the
product, the way ``Engine.__init__`` derives them (``sim.py:356-366``).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liblif_oracle.so"

MODEL_PARAMS = {
    "tauSyn": 5.0, "tDelay": 1.8, "v0": -52.0, "vReset": -52.0, "vRest": -52.0,
    "vThreshold": -45.0, "tauMem": 20.0, "tRefrac": 2.2, "scalePoisson": 250,
    "wScale": 0.275,
}
DT = 0.1


class OracleParams(ctypes.Structure):
    _fields_ = [("a_syn", ctypes.c_float), ("a_mem", ctypes.c_float),
                ("w_scale", ctypes.c_float), ("kick", ctypes.c_float),
                ("prob_scale", ctypes.c_float), ("v_rest", ctypes.c_float),
                ("v_reset", ctypes.c_float), ("v_th", ctypes.c_float),
                ("refrac_steps", ctypes.c_float), ("buf_len", ctypes.c_int32),
                ("lag", ctypes.c_int32), ("pad_", ctypes.c_int32)]


def params(p=None) -> OracleParams:
    """Constants as ``Engine.__init__`` computes them (sim.py:356-366, 383)."""
    p = dict(MODEL_PARAMS if p is None else p)
    f = np.float32
    buf_len = int(p["tDelay"] / DT) + 1
    w = f(p["wScale"])
    kick = f(w * f(f(1.0) * f(p["scalePoisson"])))
    return OracleParams(
        a_syn=float(f(1.0 - DT / p["tauSyn"])), a_mem=float(f(DT / p["tauMem"])),
        w_scale=float(w), kick=float(kick), prob_scale=float(f(DT / 1000.0)),
        v_rest=float(f(p["vRest"])), v_reset=float(f(p["vReset"])),
        v_th=float(f(p["vThreshold"])),
        refrac_steps=float(f(float(round(p["tRefrac"] / DT)))),
        buf_len=buf_len, lag=buf_len + 1, pad_=0)


class OracleParams64(ctypes.Structure):
    _fields_ = [("a_syn", ctypes.c_double), ("a_mem", ctypes.c_double),
                ("w_scale", ctypes.c_double), ("kick", ctypes.c_double),
                ("v_rest", ctypes.c_double), ("v_reset", ctypes.c_double),
                ("v_th", ctypes.c_double), ("prob_scale", ctypes.c_float),
                ("buf_len", ctypes.c_int32)]


def params64(p=None) -> OracleParams64:
    """The same constants in float64, before the reference's float32 cast."""
    p = dict(MODEL_PARAMS if p is None else p)
    return OracleParams64(
        a_syn=1.0 - DT / p["tauSyn"], a_mem=DT / p["tauMem"], w_scale=float(p["wScale"]),
        kick=float(p["wScale"]) * float(p["scalePoisson"]), v_rest=float(p["vRest"]),
        v_reset=float(p["vReset"]), v_th=float(p["vThreshold"]),
        prob_scale=float(np.float32(DT / 1000.0)), buf_len=int(p["tDelay"] / DT) + 1)


def build(force=False):
    """Compile the oracle with its Makefile (gcc, seconds)."""
    if LIB.exists() and not force and LIB.stat().st_mtime >= (HERE / "lif_oracle.c").stat().st_mtime:
        return LIB
    subprocess.run(["make", "-s", "-C", str(HERE), "liblif_oracle.so"], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        P = ctypes.c_void_p
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [ctypes.c_int, ctypes.c_int64, P, P, P]
        L.oracle_destroy.argtypes = [P]
        L.oracle_philox4x32_10.argtypes = [P, P, P]
        L.oracle_drive.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P,
                                   ctypes.c_float, ctypes.c_float, P]
        L.oracle_core.argtypes = [P, P, ctypes.c_int, ctypes.c_int] + [P] * 14 + [ctypes.c_int]
        L.oracle_run.argtypes = ([P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
                                 + [P] * 17 + [ctypes.c_int])
        L.oracle_run_f64.argtypes = [P, P, ctypes.c_int, ctypes.c_int] + [P] * 17
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def philox4x32_10(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().oracle_philox4x32_10(_p(c), _p(k), _p(out))
    return out


def drive_tape(rates, seeds, streams, own_t, p=None):
    """The Poisson input ``w * (bern * gain)`` [B, N] of one step (the tape)."""
    rates = np.ascontiguousarray(rates, dtype=np.float32)
    B, n = rates.shape
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    streams = np.ascontiguousarray(streams, dtype=np.uint32)
    own = np.ascontiguousarray(own_t, dtype=np.int64)
    P = params(p)
    out = np.zeros((B, n), dtype=np.float32)
    lib().oracle_drive(n, B, _p(rates), _p(seeds), _p(streams), _p(own),
                       P.prob_scale, P.kick, _p(out))
    return out


class Oracle:
    """The reference engine's state and step, on the host, in plain C."""

    CSRMV = 1
    EVENT = 0

    def __init__(self, row_ptr, col, cnt, n, batch=1, params_dict=None,
                 no_refractory=None, seed=0, streams=None):
        self.n, self.batch = int(n), int(batch)
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.cnt = np.ascontiguousarray(cnt, dtype=np.int32)
        self.P = params(params_dict)
        self.pdict = dict(MODEL_PARAMS if params_dict is None else params_dict)
        self.buf_len = self.P.buf_len
        B, N = self.batch, self.n
        f = np.float32
        self.v = np.full((B, N), f(self.pdict["v0"]), dtype=np.float32)
        self.conductance = np.zeros((B, N), dtype=np.float32)
        self.spikes = np.zeros((B, N), dtype=np.float32)
        self.refrac_steps = np.full((B, N), self.P.refrac_steps, dtype=np.float32)
        if no_refractory is not None and len(no_refractory):
            nr = np.asarray(no_refractory)
            if nr.ndim == 2:
                self.refrac_steps[nr.astype(bool)] = 0.0
            else:
                self.refrac_steps[:, nr.astype(np.int64)] = 0.0
        self.refrac = self.refrac_steps.copy()
        self.delay_buffer = np.zeros((B, self.buf_len, N), dtype=np.float32)
        self.ptr = np.zeros(1, dtype=np.int32)
        self.m_fire = np.ones((B, N), dtype=np.float32)
        self.m_out = np.ones((B, N), dtype=np.float32)
        self.m_in = np.ones((B, N), dtype=np.float32)
        self.m_hold = np.ones((B, N), dtype=np.float32)
        self.v_hold = np.zeros((B, N), dtype=np.float32)
        self.rates = np.zeros((B, N), dtype=np.float32)
        self.seeds = np.full(B, seed, dtype=np.uint64)
        self.streams = (np.arange(B, dtype=np.uint32) if streams is None
                        else np.ascontiguousarray(streams, dtype=np.uint32))
        self.own_t = np.zeros(B, dtype=np.int64)
        self._rec = np.zeros((B, N), dtype=np.float32)
        self._h = lib().oracle_create(N, int(self.col.shape[0]), _p(self.row_ptr),
                                      _p(self.col), _p(self.cnt))
        if not self._h:
            raise MemoryError("oracle_create failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # module globals may be gone at interpreter exit
            try:
                lib().oracle_destroy(h)
            except TypeError:
                pass
            self._h = None

    def set_masks(self, fire=None, out=None, inc=None, hold=None, v_clamp=None,
                  trial=None):
        """``Engine.set_masks`` semantics (sim.py:510-593), optionally one trial."""
        rows = slice(None) if trial is None else slice(trial, trial + 1)
        for vec, idx in ((self.m_fire, fire), (self.m_out, out),
                         (self.m_in, inc), (self.m_hold, hold)):
            if idx is None:
                continue
            vec[rows] = 1.0
            if len(idx):
                vec[rows, np.asarray(idx, dtype=np.int64)] = 0.0
        if hold is not None:
            clamp = np.float32(self.pdict["vReset"] if v_clamp is None else v_clamp)
            self.v_hold[rows] = 0.0
            if len(hold):
                self.v_hold[rows, np.asarray(hold, dtype=np.int64)] = clamp

    def _args(self):
        return [_p(self.v), _p(self.conductance), _p(self.spikes), _p(self.refrac),
                _p(self.delay_buffer), _p(self.ptr), _p(self.refrac_steps),
                _p(self.m_fire), _p(self.m_out), _p(self.m_in), _p(self.m_hold),
                _p(self.v_hold)]

    def _threads(self, threads):
        """Explicit count, else one thread below a million neuron-trials (the
        per-step parallel regions cost more than they save there)."""
        if threads:
            return int(threads)
        return 1 if self.batch * self.n < (1 << 20) else nthreads_default()

    def core(self, vstim, mode=EVENT, threads=0):
        """One ``Engine._core(voltage_stim)`` call with an explicit tape."""
        threads = self._threads(threads)
        vstim = np.ascontiguousarray(vstim, dtype=np.float32)
        rc = lib().oracle_core(self._h, ctypes.byref(self.P), self.batch, mode,
                               *self._args(), _p(vstim), _p(self._rec), threads)
        if rc:
            raise RuntimeError("oracle_core returned %d" % rc)
        return self.spikes

    def run(self, steps, mode=EVENT, raster=False, threads=0):
        """``steps`` calls of ``Engine.step`` with the Philox drive.

        Returns the raster as uint8 bits [steps, B, ceil(N/8)] (little bit
        order) when ``raster`` is true.
        """
        threads = self._threads(threads)
        nbytes = (self.n + 7) // 8
        out = np.zeros((steps, self.batch, nbytes), dtype=np.uint8) if raster else None
        rc = lib().oracle_run(
            self._h, ctypes.byref(self.P), self.batch, int(steps), mode, *self._args(),
            _p(self.rates), _p(self.seeds), _p(self.streams), _p(self.own_t),
            _p(out) if raster else None, threads)
        if rc:
            raise RuntimeError("oracle_run returned %d" % rc)
        return out

    def run_f64(self, steps, raster=False):
        """``steps`` steps of the same equations in float64 from the current state.

        Works on float64 copies (``v64``, ``g64`` ... created on first use from
        the float32 state) and leaves the float32 state alone; the drive uses
        the same draws, so both runs see the same kicks.
        """
        if not hasattr(self, "v64"):
            self.v64 = self.v.astype(np.float64)
            self.g64 = self.conductance.astype(np.float64)
            self.spikes64 = self.spikes.astype(np.float64)
            self.refrac64 = self.refrac.astype(np.float64)
            self.ring64 = self.delay_buffer.astype(np.float64)
            self.ptr64 = self.ptr.copy()
            self.own64 = self.own_t.copy()
        nbytes = (self.n + 7) // 8
        out = np.zeros((steps, self.batch, nbytes), dtype=np.uint8) if raster else None
        P64 = params64(self.pdict)
        rc = lib().oracle_run_f64(
            self._h, ctypes.byref(P64), self.batch, int(steps), _p(self.v64), _p(self.g64),
            _p(self.spikes64), _p(self.refrac64), _p(self.ring64), _p(self.ptr64),
            _p(self.refrac_steps), _p(self.m_fire), _p(self.m_out), _p(self.m_in),
            _p(self.m_hold), _p(self.v_hold), _p(self.rates), _p(self.seeds), _p(self.streams),
            _p(self.own64), _p(out) if raster else None)
        if rc:
            raise RuntimeError("oracle_run_f64 returned %d" % rc)
        return out

    @classmethod
    def from_connectome(cls, conn, **kw):
        return cls(conn.row_ptr, conn.col, conn.cnt, conn.n, **kw)


def fingerprint(a) -> str:
    """sha256 of the raw bytes, first 16 hex digits (as the reference's probes)."""
    import hashlib

    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.tobytes()).hexdigest()[:16]


def nthreads_default():
    return os.cpu_count() or 1
