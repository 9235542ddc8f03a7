"""The reference's ``flybrain.evspmv`` surface over this library's kernels.

``exactness``, ``Events`` (CSR by presynaptic neuron + persistent output +
host bounds check + ``mm``), ``EventKernelUnavailable``, ``F32_EXACT_INT``,
``THREADS`` and ``ABI`` keep the names, arguments, record keys and failure
behaviour of ``lab/flybrain/evspmv.py:957-1138``; the kernel behind
``Events.mm`` is this library's ``ev_spmv_i32``/``ev_spmv_i64``
(``include/fis.h``), compiled for sm_100a, instead of the reference's
compute_52 PTX.

The bodies are this package's own: the weight matrix is taken apart into
numpy CSR arrays once (:func:`_csr_arrays`), its row sums come from one
``bincount`` over the row index of every value, and the bounds check is
:func:`fis.connectome.csr_faults`, the one the engine's own connectome uses.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from .connectome import csr_faults

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


def _record(integral, frac, lo, hi, worst):
    """The reference's exactness record (its keys are read by run reports)."""
    margin = round(F32_EXACT_INT / worst, 1) if worst else None
    return {
        "значения целые": bool(integral),
        "макс нецелая часть": float(frac),
        "мин значение": float(lo),
        "макс значение": float(hi),
        "макс сумма модулей по строке": float(worst),
        "предел точности float32": F32_EXACT_INT,
        "запас": margin,
        "годится": bool(integral) and 0.0 < worst < F32_EXACT_INT,
    }


def exactness_from(ex):
    """The exactness record from ``Connectome.exactness()`` (integral by
    construction: the connectome holds integer synapse counts)."""
    worst = float(ex["max_abs_row_sum"])
    rec = _record(ex["integral"], 0.0, 0.0, 0.0, worst)
    for key in ("мин значение", "макс значение"):
        del rec[key]
    rec["годится"] = bool(ex["ok"]) and rec["годится"]
    return rec


def _csr_arrays(w):
    """``(n_rows, n_cols, row_ptr, col, val)`` numpy arrays of a torch CSR (or
    any sparse) matrix, without changing its index dtype."""
    import torch

    if w.layout != torch.sparse_csr:
        w = w.to_sparse_csr()
    return (int(w.shape[0]), int(w.shape[1]), w.crow_indices().cpu().numpy(),
            w.col_indices().cpu().numpy(), w.values().detach().cpu().numpy())


def exactness(w_csr):
    """Conditions of bitwise equality with ``csrmv`` (evspmv.py:957-994).

    The product is exact in any summation order when every value is an
    integer and no row of ``W[post, :]`` has an absolute sum of 2**24 or
    more: every partial float32 sum is then an exact integer.  Returns the
    reference's record; raises nothing (the caller decides).
    """
    n_rows, _, row_ptr, _, val = _csr_arrays(w_csr)
    val = val.astype(np.float64)
    if val.size == 0:
        return _record(True, 0.0, 0.0, 0.0, 0.0)
    frac = float(np.abs(val - np.rint(val)).max())
    row_of = np.repeat(np.arange(n_rows), np.diff(row_ptr.astype(np.int64)))
    sums = np.bincount(row_of, weights=np.abs(val), minlength=n_rows)
    return _record(frac == 0.0, frac, val.min(), val.max(), float(sums.max()))


def _by_pre(n, row_ptr, col, val):
    """Transpose CSR ``W[post, pre]`` into CSR by presynaptic neuron, keeping
    the index dtype: row ``pre`` lists its ``(post, value)`` with ``post``
    ascending (a stable sort of the values by their column)."""
    itype = row_ptr.dtype
    post = np.repeat(np.arange(n, dtype=np.int64), np.diff(row_ptr.astype(np.int64)))
    order = np.argsort(col, kind="stable")
    t_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(col.astype(np.int64), minlength=n), out=t_ptr[1:])
    return (t_ptr.astype(itype), post[order].astype(itype),
            np.ascontiguousarray(val[order], dtype=np.float32))


class Events:
    """W by presynaptic neuron plus the kernel call (evspmv.py:997-1138).

    The output buffer is persistent (a captured graph writes into the same
    memory on every replay); ``mm`` zeroes it and launches the library's
    ``ev_spmv`` on the current stream.
    """

    def __init__(self, w_csr, batch, device, threads=None, verbose=False, load=None):
        import torch

        self.kern, self.build_info = build(verbose=verbose, load=load)
        self.threads = int(threads or THREADS)
        self.batch = int(batch)
        n_rows, n_cols, row_ptr, col, val = _csr_arrays(w_csr)
        if n_rows != n_cols:
            raise EventKernelUnavailable("weight matrix is not square: %s"
                                         % ((n_rows, n_cols),))
        self.n = n_rows
        if row_ptr.dtype != col.dtype:
            raise EventKernelUnavailable("index dtypes differ: crow %s, col %s"
                                         % (row_ptr.dtype, col.dtype))
        kernels = {np.dtype(np.int32): "ev_spmv_i32", np.dtype(np.int64): "ev_spmv_i64"}
        name = kernels.get(np.dtype(col.dtype))
        if name is None:
            raise EventKernelUnavailable("index dtype %s; int32 or int64 only" % col.dtype)
        self._fn = getattr(self.kern, name)
        faults = csr_faults(self.n, row_ptr, col, val.shape[0])
        if faults:
            raise EventKernelUnavailable("event kernel would address memory outside its "
                                         "buffers:\n  " + "\n  ".join(faults))
        t_ptr, t_post, t_val = _by_pre(self.n, row_ptr, col, val)
        self.crow = torch.from_numpy(t_ptr).to(device)
        self.col = torch.from_numpy(t_post).to(device)
        self.val = torch.from_numpy(t_val).to(device)
        self.out = torch.zeros(self.batch, self.n, device=device)

    def mm(self, sp, mo):
        """``out = W @ (sp * mo)`` per trial; returns the persistent buffer."""
        import torch

        want = (self.batch, self.n)
        if tuple(sp.shape) != want or tuple(mo.shape) != want:
            raise ValueError("expected [%d, %d], got %s and %s"
                             % (self.batch, self.n, tuple(sp.shape), tuple(mo.shape)))
        if not (sp.is_contiguous() and mo.is_contiguous()):
            raise ValueError("spikes and mask must be contiguous")
        self.out.zero_()
        args = [ctypes.c_void_p(t.data_ptr())
                for t in (self.crow, self.col, self.val, sp, mo, self.out)]
        rc = self._fn(*args, self.n, self.batch, self.threads,
                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise RuntimeError("event kernel launch returned %d" % rc)
        return self.out
