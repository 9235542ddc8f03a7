"""ctypes binding of ``include/fis.h`` (the library ``libfis_b200.so``).

The library is built in-tree (``fis.build``) and loaded from this package's
directory.  If it is missing, or was built against another ABI, every entry
point refuses loudly with :class:`KernelUnavailable`; there is no CPU path to
fall back to.  This mirrors the reference's loud failure
(``lab/flybrain/evspmv.py:173-189``).
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_NAME = "libfis_b200.so"
LIB_PATH = PKG / LIB_NAME

FIS_ABI_VERSION = 9
FIS_MAX_BLOCK = 20
FIS_NOALLOC_RING_INTS = 3 << 20
REF_EV_ABI = 3

FIS_FL_FIRE_OFF = 1 << 0
FIS_FL_OUT_OFF = 1 << 1
FIS_FL_IN_OFF = 1 << 2
FIS_FL_HOLD = 1 << 3
FIS_FL_NOREFRAC = 1 << 4
FIS_FL_SILENCED = 1 << 5

# device error bits in done[1] (FIS_ERR_*)
FIS_ERR_STAGE = 1 << 0
FIS_ERR_STAGE_LOST = 1 << 1

STATUS = {0: "ok", -1: "FIS_E_ARG (null pointer or size out of range)",
          -2: "FIS_E_BOUNDS (trial range, block length or slot out of range)",
          -3: "FIS_E_ALIGN (array not 16-byte aligned)"}

# Every symbol include/fis.h declares, checked at load time and by the tests.
EXPORTS = ("ev_spmv_i32", "ev_spmv_i64", "ev_spmv_abi", "fis_abi",
           "fis_sizeof_engine", "fis_sizeof_trial", "fis_check", "fis_block",
           "fis_scatter", "fis_update", "fis_advance", "fis_advance_overlap",
           "fis_delay_buffer", "fis_spikes_f32", "fis_load_spikes", "fis_add_rows",
           "fis_graded_step",
           "fis_ring_row", "fis_block_noalloc", "fis_red_rate")


class KernelUnavailable(RuntimeError):
    """The CUDA library is missing or unusable; said loudly, never bypassed."""


class LifParams(ctypes.Structure):
    _fields_ = [("a_syn", ctypes.c_float), ("a_mem", ctypes.c_float),
                ("w_scale", ctypes.c_float), ("kick", ctypes.c_float),
                ("prob_scale", ctypes.c_float), ("v_rest", ctypes.c_float),
                ("v_reset", ctypes.c_float), ("v_th", ctypes.c_float),
                ("refrac_steps", ctypes.c_float), ("buf_len", ctypes.c_int32),
                ("lag", ctypes.c_int32), ("pad_", ctypes.c_int32)]


class Trial(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("start", ctypes.c_int64),
                ("end", ctypes.c_int64), ("v_clamp", ctypes.c_float),
                ("stream", ctypes.c_uint32), ("rec", ctypes.c_int32),
                ("bin_steps", ctypes.c_int32), ("n_bins", ctypes.c_int32),
                ("history", ctypes.c_int32)]


class EngineDesc(ctypes.Structure):
    _fields_ = [("row_ptr", ctypes.c_void_p), ("edges", ctypes.c_void_p),
                ("nchunks", ctypes.c_void_p), ("v", ctypes.c_void_p),
                ("g", ctypes.c_void_p), ("refrac", ctypes.c_void_p),
                ("flags", ctypes.c_void_p), ("rates", ctypes.c_void_p),
                ("vstim", ctypes.c_void_p), ("trials", ctypes.c_void_p), ("lists", ctypes.c_void_p),
                ("list_len", ctypes.c_void_p), ("bits", ctypes.c_void_p),
                ("clock", ctypes.c_void_p), ("done", ctypes.c_void_p),
                ("recs", ctypes.c_void_p), ("kicks", ctypes.c_void_p),
                ("drive_idx", ctypes.c_void_p), ("drive_len", ctypes.c_void_p),
                ("nnz", ctypes.c_int64),
                ("list_cap", ctypes.c_int64), ("n", ctypes.c_int32),
                ("batch", ctypes.c_int32), ("chunk", ctypes.c_int32),
                ("n_recs", ctypes.c_int32), ("ring16", ctypes.c_int32),
                ("wait_polls", ctypes.c_uint32), ("inject_stall", ctypes.c_uint32),
                ("raster", ctypes.c_int32), ("scatter_mode", ctypes.c_int32),
                ("scat_ctas", ctypes.c_int32), ("drive_ctas", ctypes.c_int32),
                ("update_streams", ctypes.c_int32), ("update_tiles", ctypes.c_int32),
                ("pad3_", ctypes.c_int32), ("p", LifParams)]


_lib = None


def load(path=None):
    """Load the library once per process; refuse loudly if it is unusable."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path or os.environ.get("FIS_LIB") or LIB_PATH)
    if not p.exists():
        raise KernelUnavailable(
            "CUDA library %s is not built. Build it with `python -c \"import fis.build as b; "
            "b.build()\"` (nvcc for sm_100a). There is no CPU fallback." % p)
    try:
        L = ctypes.CDLL(str(p))
    except OSError as exc:
        raise KernelUnavailable("cannot load %s: %s" % (p, exc)) from exc
    missing = [s for s in EXPORTS if not hasattr(L, s)]
    if missing:
        raise KernelUnavailable("%s lacks exports %s; rebuild it" % (p, missing))
    P, I32, I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    for name in ("fis_abi", "fis_sizeof_engine", "fis_sizeof_trial", "ev_spmv_abi"):
        getattr(L, name).restype = ctypes.c_int
        getattr(L, name).argtypes = []
    L.fis_check.argtypes = [P]
    L.fis_block.argtypes = [P, I32, I32, I32, P, P, I32, P]
    L.fis_scatter.argtypes = [P, I32, I32, I32, P, P]
    L.fis_advance.argtypes = [P, I64, I64, I32, I32, P, P, P, I32, I32, P]
    L.fis_advance_overlap.argtypes = [P, I64, I64, I32, I32, P, P, P, I32, I32, P]
    L.fis_update.argtypes = [P, I32, I32, I32, P, P, I32, P]
    L.fis_red_rate.argtypes = [P, I64, I32, I32, P]
    L.fis_delay_buffer.argtypes = [P, I32, I32, P, P, P]
    L.fis_spikes_f32.argtypes = [P, I32, I32, I64, P, P]
    L.fis_load_spikes.argtypes = [P, I32, I32, P, P]
    L.fis_add_rows.argtypes = [P, I32, I32, P, I64, I64, P, I64, I64, P]
    L.fis_graded_step.argtypes = [P, I64, P, P, P, P, P, I32, P, P, P]
    L.fis_graded_step.restype = ctypes.c_int
    L.fis_block_noalloc.argtypes = [P, I32, I32, I32, P, I32, P]
    L.fis_block_noalloc.restype = ctypes.c_int
    L.fis_ring_row.argtypes = [I32]
    L.fis_ring_row.restype = ctypes.c_int
    L.ev_spmv_i32.argtypes = [P, P, P, P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
    L.ev_spmv_i64.argtypes = [P, P, P, P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
    for s in ("fis_check", "fis_block", "fis_scatter", "fis_update", "fis_advance",
              "fis_advance_overlap", "fis_delay_buffer", "fis_spikes_f32",
              "fis_load_spikes", "fis_add_rows", "ev_spmv_i32", "ev_spmv_i64"):
        getattr(L, s).restype = ctypes.c_int
    if L.fis_abi() != FIS_ABI_VERSION:
        raise KernelUnavailable("%s has ABI %d, this binding expects %d; rebuild it"
                                % (p, L.fis_abi(), FIS_ABI_VERSION))
    if L.fis_sizeof_engine() != ctypes.sizeof(EngineDesc) or \
            L.fis_sizeof_trial() != ctypes.sizeof(Trial):
        raise KernelUnavailable("struct layout of %s differs from the binding" % p)
    if L.ev_spmv_abi() != REF_EV_ABI:
        raise KernelUnavailable("ev_spmv_abi() != %d" % REF_EV_ABI)
    if path is None:
        _lib = L
    return L


def check(rc, what):
    """Raise on a non-zero status (the reference: evspmv.py:1135-1137)."""
    if rc:
        if rc < 0:
            why = STATUS.get(rc, "FIS error %d" % rc)
        else:
            try:
                import torch

                why = "cudaError %d (%s)" % (rc, torch.cuda.cudart().cudaGetErrorString(rc))
            except Exception:
                why = "cudaError %d" % rc
        raise RuntimeError("%s failed: %s" % (what, why))
