"""The reference's ``flybrain.evspmv`` surface over this library's kernels.

``exactness``, ``Events`` (transposed CSR + persistent output + host bounds
check + ``mm``), ``EventKernelUnavailable``, ``F32_EXACT_INT``, ``THREADS``
and ``ABI`` keep the names and meaning of ``lab/flybrain/evspmv.py``; the
kernel behind ``Events.mm`` is this library's ``ev_spmv_i32``/``ev_spmv_i64``
(``include/fis.h``), compiled for sm_100a, instead of the reference's
compute_52 PTX.
"""

from __future__ import annotations

import ctypes
import os

from . import _lib

F32_EXACT_INT = 1 << 24
THREADS = int(os.environ.get("FLYBRAIN_EV_THREADS", "128"))
ABI = _lib.REF_EV_ABI


class EventKernelUnavailable(_lib.KernelUnavailable):
    """The event kernel is unavailable, said loudly (evspmv.py:173-178)."""


def build(verbose=False, load=None, force=False):
    """Load the library; returns ``(library, build info)`` (evspmv.py:930-954)."""
    try:
        L = _lib.load()
    except _lib.KernelUnavailable as exc:
        raise EventKernelUnavailable(str(exc)) from exc
    info = {"дорога": "libfis_b200", "путь": str(_lib.LIB_PATH), "abi": L.ev_spmv_abi(),
            "цель": "sm_100a"}
    return L, info


def exactness_from(ex):
    """The reference's exactness record from ``Connectome.exactness()``."""
    worst = ex["max_abs_row_sum"]
    return {
        "значения целые": bool(ex["integral"]),
        "макс нецелая часть": 0.0,
        "макс сумма модулей по строке": worst,
        "предел точности float32": F32_EXACT_INT,
        "запас": round(F32_EXACT_INT / worst, 1) if worst else None,
        "годится": bool(ex["ok"] and worst > 0),
    }


def exactness(w_csr):
    """Conditions of bitwise equality with ``csrmv`` (evspmv.py:957-994).

    Integral values and a maximum absolute row sum of ``W[post, :]`` below
    2**24: then any summation order of the int-valued terms is exact.
    """
    import torch

    val = w_csr.values()
    crow = w_csr.crow_indices()
    frac = (val - torch.round(val)).abs().max() if val.numel() else torch.zeros(())
    integral = bool(float(frac) == 0.0)
    cum = torch.cumsum(val.abs().to(torch.float64), 0)
    cum = torch.cat([torch.zeros(1, dtype=cum.dtype, device=cum.device), cum])
    rows = cum[crow.to(torch.int64)]
    worst = float((rows[1:] - rows[:-1]).max()) if rows.numel() > 1 else 0.0
    return {
        "значения целые": integral,
        "макс нецелая часть": float(frac),
        "мин значение": float(val.min()) if val.numel() else 0.0,
        "макс значение": float(val.max()) if val.numel() else 0.0,
        "макс сумма модулей по строке": worst,
        "предел точности float32": F32_EXACT_INT,
        "запас": round(F32_EXACT_INT / worst, 1) if worst else None,
        "годится": bool(integral and 0.0 < worst < F32_EXACT_INT),
    }


class Events:
    """W by presynaptic neuron plus the kernel call (evspmv.py:997-1138)."""

    def __init__(self, w_csr, batch, device, threads=None, verbose=False, load=None):
        import torch

        self.kern, self.build_info = build(verbose=verbose, load=load)
        self.threads = int(threads or THREADS)
        self.batch = int(batch)
        if w_csr.shape[0] != w_csr.shape[1]:
            raise EventKernelUnavailable("weight matrix is not square: %s"
                                         % (tuple(w_csr.shape),))
        self.n = int(w_csr.shape[0])
        import warnings
        with warnings.catch_warnings():
            warnings.filterwarnings("ignore", message=".*[Ss]parse.*")
            wt = w_csr.t().to_sparse_csr()
        self.crow = wt.crow_indices().contiguous()
        self.col = wt.col_indices().contiguous()
        self.val = wt.values().contiguous().to(torch.float32)
        if self.crow.dtype != self.col.dtype:
            raise EventKernelUnavailable("index dtypes differ: crow %s, col %s"
                                         % (self.crow.dtype, self.col.dtype))
        if self.col.dtype not in (torch.int32, torch.int64):
            raise EventKernelUnavailable("index dtype %s; int32 or int64 only" % self.col.dtype)
        self._fn = self.kern.ev_spmv_i32 if self.col.dtype == torch.int32 else self.kern.ev_spmv_i64
        self.out = torch.zeros(self.batch, self.n, device=device)
        deg = (self.crow[1:] - self.crow[:-1]).to(torch.int64)
        self._check_bounds(deg)

    def _check_bounds(self, deg):
        """Once per build: everything the kernel addresses lies inside its buffers."""
        bad = []
        if self.crow.numel() != self.n + 1:
            bad.append("crow has %d entries, expected n+1 = %d" % (self.crow.numel(), self.n + 1))
        nnz = int(self.val.numel())
        if self.col.numel() != nnz:
            bad.append("%d column indices but %d values" % (self.col.numel(), nnz))
        if int(self.crow[-1]) != nnz:
            bad.append("crow[n] = %d but nnz = %d" % (int(self.crow[-1]), nnz))
        if bool((deg < 0).any()):
            bad.append("crow decreases")
        if nnz:
            lo, hi = int(self.col.min()), int(self.col.max())
            if lo < 0 or hi >= self.n:
                bad.append("column indices in [%d, %d], outside [0, %d)" % (lo, hi, self.n))
        if self.out.numel() != self.batch * self.n:
            bad.append("output buffer has %d elements, expected batch*n" % self.out.numel())
        if bad:
            raise EventKernelUnavailable("event kernel would address memory outside its "
                                         "buffers:\n  " + "\n  ".join(bad))

    def mm(self, sp, mo):
        """``out = W @ (sp * mo)`` per trial; returns the persistent buffer."""
        import torch

        if sp.shape != (self.batch, self.n) or mo.shape != sp.shape:
            raise ValueError("expected [%d, %d], got %s and %s"
                             % (self.batch, self.n, tuple(sp.shape), tuple(mo.shape)))
        if not (sp.is_contiguous() and mo.is_contiguous()):
            raise ValueError("spikes and mask must be contiguous")
        self.out.zero_()
        P = ctypes.c_void_p
        rc = self._fn(P(self.crow.data_ptr()), P(self.col.data_ptr()), P(self.val.data_ptr()),
                      P(sp.data_ptr()), P(mo.data_ptr()), P(self.out.data_ptr()),
                      self.n, self.batch, self.threads,
                      P(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise RuntimeError("event kernel launch returned %d" % rc)
        return self.out
