"""Connectome in the layout the B200 kernels read: CSR by presynaptic neuron.

Two sources feed it:

* :func:`synthetic` -- a seeded stand-in for the FlyWire v783 matrix the
  reference loads from the upstream parquet (``lab/flybrain/data.py:221-259``),
  which is not available here.  Statistics: N=138,639 neurons, E=15,091,983
  directed edges, out-degree Pareto(alpha=1.8)+1 rescaled to the mean E/N,
  uniform postsynaptic targets without duplicates or self-loops, synapse counts
  ``clip(round(lognormal(0.9, 1.0)), 1, 2400)``, sign per presynaptic neuron
  (30 % inhibitory).
* :func:`from_weights` -- the reference's own weight object, a torch sparse COO
  ``W[post, pre]`` of signed synapse counts (``data.py:221-226``), so callers of
  ``sim.build_engine(weights=...)`` keep working.
* :func:`from_parquet` / :func:`from_upstream` -- the upstream connectivity
  table itself (``data.py:240-259``), read without torch and cached as packed
  CSR arrays, for when the FlyWire files are at hand.

The kernel format packs one edge into one 32-bit word: the postsynaptic index
in the high 18 bits and the signed synapse count in the low 14 bits (two's
complement).  :meth:`Connectome.packed` refuses loudly when a matrix does not
fit (N > 2**18 or |count| > 8191) instead of truncating.
"""

from __future__ import annotations

import hashlib
import os
import tempfile
from dataclasses import dataclass
from pathlib import Path

import numpy as np

N_FLYWIRE = 138_639
E_FLYWIRE = 15_091_983

# Exactness bound of float32 integer sums (reference ``evspmv.py:108``): a sum
# of integers is exact in any order while every partial sum stays below 2**24.
F32_EXACT_INT = 1 << 24

PACK_COL_BITS = 18
PACK_CNT_BITS = 14
PACK_MAX_N = 1 << PACK_COL_BITS
PACK_CNT_MAX = (1 << (PACK_CNT_BITS - 1)) - 1
PACK_CNT_MIN = -(1 << (PACK_CNT_BITS - 1))


class ConnectomeError(ValueError):
    """The matrix cannot be represented exactly in the kernel format."""


@dataclass
class Connectome:
    """CSR by presynaptic neuron: row ``pre`` lists ``(post, count)``.

    ``row_ptr`` int64 [n+1], ``col`` int32 [E] (postsynaptic index, ascending
    within a row), ``cnt`` int32 [E] (signed synapse count, never zero).
    """

    n: int
    row_ptr: np.ndarray
    col: np.ndarray
    cnt: np.ndarray
    seed: int | None = None

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def out_degree(self) -> np.ndarray:
        return np.diff(self.row_ptr)

    def in_abs_sum(self) -> np.ndarray:
        """Sum of |count| per postsynaptic neuron (one row of ``W[post, :]``)."""
        return np.bincount(self.col, weights=np.abs(self.cnt).astype(np.float64),
                           minlength=self.n)

    def exactness(self) -> dict:
        """The conditions under which int32 accumulation equals the reference.

        Mirrors ``evspmv.exactness`` (reference ``evspmv.py:957-994``): integral
        values (true by construction here) and a maximum per-post absolute row
        sum below 2**24, so every partial sum of a float32 accumulation is an
        exact integer and the order of additions cannot matter.
        """
        worst = float(self.in_abs_sum().max()) if self.nnz else 0.0
        return {
            "integral": True,
            "max_abs_row_sum": worst,
            "f32_exact_limit": F32_EXACT_INT,
            "margin": round(F32_EXACT_INT / worst, 1) if worst else None,
            "ok": bool(0.0 <= worst < F32_EXACT_INT),
        }

    def packed(self) -> np.ndarray:
        """Edges as uint32 words ``post << 14 | (count & 0x3fff)``."""
        if self.n > PACK_MAX_N:
            raise ConnectomeError(
                "packed edge format holds postsynaptic indices below 2**18 = %d; "
                "this matrix has n = %d" % (PACK_MAX_N, self.n))
        if self.nnz:
            lo, hi = int(self.cnt.min()), int(self.cnt.max())
            if lo < PACK_CNT_MIN or hi > PACK_CNT_MAX:
                raise ConnectomeError(
                    "packed edge format holds synapse counts in [%d, %d]; this "
                    "matrix has [%d, %d]" % (PACK_CNT_MIN, PACK_CNT_MAX, lo, hi))
        col = self.col.astype(np.uint32)
        cnt = self.cnt.astype(np.int64) & ((1 << PACK_CNT_BITS) - 1)
        return (col << np.uint32(PACK_CNT_BITS)) | cnt.astype(np.uint32)

    def check_bounds(self) -> None:
        """Host-side bounds check before any kernel sees the arrays.

        Same role as ``Events._check_bounds`` (reference ``evspmv.py:1057-1113``):
        an out-of-range index would not fault under a caching allocator, it
        would silently write into a neighbouring tensor.
        """
        bad = csr_faults(self.n, self.row_ptr, self.col, self.cnt.shape[0])
        if bad:
            raise ConnectomeError("connectome fails its bounds check:\n  "
                                  + "\n  ".join(bad))

    def by_post(self):
        """The weights as CSR by postsynaptic neuron: ``(t_ptr`` int64 [n+1],
        ``t_pre`` int32 [E], ``t_val`` float32 [E]``)``, presynaptic indices
        ascending within a row -- torch's CSR of ``W[post, pre]``, the layout
        and order of the reference's csrmv pull (``sim.py:357, 910-913``)."""
        pre = np.repeat(np.arange(self.n, dtype=np.int32), np.diff(self.row_ptr))
        order = np.argsort(self.col, kind="stable")
        t_ptr = np.zeros(self.n + 1, dtype=np.int64)
        np.cumsum(np.bincount(self.col, minlength=self.n), out=t_ptr[1:])
        return t_ptr, np.ascontiguousarray(pre[order]), self.cnt[order].astype(np.float32)

    def to_torch_weights(self, device="cpu"):
        """The reference's weight object: sparse COO ``W[post, pre]`` float32."""
        import torch

        pre = np.repeat(np.arange(self.n, dtype=np.int64), self.out_degree())
        idx = torch.from_numpy(np.vstack([self.col.astype(np.int64), pre]))
        val = torch.from_numpy(self.cnt.astype(np.float32))
        import warnings
        with warnings.catch_warnings():
            warnings.filterwarnings("ignore", message=".*[Ss]parse.*")
            w = torch.sparse_coo_tensor(idx, val, (self.n, self.n)).coalesce()
        return w.to(device)

    def without(self, silenced) -> "Connectome":
        """Drop rows and columns of ``silenced`` neurons (``sim.py:324-336``)."""
        silenced = np.asarray(silenced, dtype=np.int64)
        if silenced.size == 0:
            return self
        dead = np.zeros(self.n, dtype=bool)
        dead[silenced] = True
        pre = np.repeat(np.arange(self.n), self.out_degree())
        keep = ~(dead[pre] | dead[self.col])
        deg = np.bincount(pre[keep], minlength=self.n)
        rp = np.zeros(self.n + 1, dtype=np.int64)
        np.cumsum(deg, out=rp[1:])
        return Connectome(self.n, rp, self.col[keep].copy(), self.cnt[keep].copy(),
                          self.seed)


def csr_faults(n, row_ptr, col, n_values) -> list:
    """Every way a CSR of ``n`` rows would send a kernel outside its arrays.

    ``row_ptr`` [n+1] must run from 0 to the edge count without decreasing,
    ``col`` must hold one index in [0, n) per value.  Returns a list of
    messages, empty when the arrays are safe to hand to a kernel.
    """
    row_ptr = np.asarray(row_ptr)
    col = np.asarray(col)
    nnz = int(col.shape[0])
    faults = []
    if row_ptr.shape != (n + 1,):
        faults.append("row_ptr has %d entries, expected n+1 = %d" % (row_ptr.size, n + 1))
    else:
        first, last = int(row_ptr[0]), int(row_ptr[-1])
        if (first, last) != (0, nnz):
            faults.append("row_ptr spans [%d, %d], expected [0, %d]" % (first, last, nnz))
        elif np.any(row_ptr[1:] < row_ptr[:-1]):
            faults.append("row_ptr decreases")
    if int(n_values) != nnz:
        faults.append("%d indices but %d values" % (nnz, int(n_values)))
    if nnz:
        lo, hi = int(col.min()), int(col.max())
        if lo < 0 or hi >= n:
            faults.append("indices in [%d, %d], outside [0, %d)" % (lo, hi, n))
    return faults


def from_weights(weights, n=None) -> Connectome:
    """Build the CSR-by-pre form from the reference's ``W[post, pre]`` tensor.

    Values must be integral (signed synapse counts); anything else is refused
    loudly, as the reference refuses its exact event path on such a matrix
    (``sim.py:466-479``).
    """
    import torch

    w = weights.coalesce() if weights.layout == torch.sparse_coo else weights
    if w.layout == torch.sparse_csr:
        w = w.to_sparse_coo().coalesce()
    if w.layout != torch.sparse_coo:
        w = w.to_sparse_coo().coalesce()
    if w.shape[0] != w.shape[1]:
        raise ConnectomeError("weight matrix is not square: %s" % (tuple(w.shape),))
    n = int(w.shape[0]) if n is None else int(n)
    if n != w.shape[0]:
        raise ConnectomeError("n = %d but the weight matrix is %s" % (n, tuple(w.shape)))
    idx = w.indices().cpu().numpy()
    val = w.values().detach().cpu().numpy().astype(np.float64)
    return _from_coo(n, idx[0].astype(np.int64), idx[1].astype(np.int64), val)


def _from_coo(n, post, pre, val) -> Connectome:
    """CSR by pre from coalesced ``(post, pre, value)`` triples (no repeated
    pair), refusing values that are not integral synapse counts."""
    if val.size and not np.all(val == np.rint(val)):
        frac = float(np.max(np.abs(val - np.rint(val))))
        raise ConnectomeError(
            "weights are not integral synapse counts (largest fractional part "
            "%g); the int32 ring accumulates exact counts only" % frac)
    cnt = np.rint(val).astype(np.int64)
    nz = cnt != 0
    post, pre, cnt = post[nz], pre[nz], cnt[nz]
    if cnt.size and (np.abs(cnt).max() >= 1 << 31):
        raise ConnectomeError("synapse count exceeds int32")
    order = np.lexsort((post, pre))
    pre, post, cnt = pre[order], post[order], cnt[order]
    deg = np.bincount(pre, minlength=n)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(deg, out=rp[1:])
    c = Connectome(n, rp, post.astype(np.int32), cnt.astype(np.int32))
    c.check_bounds()
    return c


# Column names and file names of the upstream FlyWire v783 release, as the
# reference reads them (data.py:43-44, 240-243).
UPSTREAM_PRE = "Presynaptic_Index"
UPSTREAM_POST = "Postsynaptic_Index"
UPSTREAM_VALUE = "Excitatory x Connectivity"
UPSTREAM_CONN_FILE = "2025_Connectivity_783.parquet"
UPSTREAM_COMP_FILE = "2025_Completeness_783.csv"


def _cache_root() -> Path:
    return Path(os.environ.get("FIS_CACHE") or (Path(tempfile.gettempdir()) / "fis_cache"))


def _csv_rows(path) -> int:
    """Data rows of a CSV with a header line (the reference's ``len(read_csv)``)."""
    import csv

    with open(path, newline="") as f:
        return max(0, sum(1 for _ in csv.reader(f)) - 1)


def from_parquet(path, n=None, comp=None, cache=True) -> Connectome:
    """The upstream connectivity table as a :class:`Connectome` (data.py:221-259).

    ``path``: a parquet file with the columns ``Presynaptic_Index``,
    ``Postsynaptic_Index`` and ``Excitatory x Connectivity`` (the signed synapse
    count of the connection).  ``n``: the neuron count, or ``comp``: the
    completeness CSV, whose row count the reference takes as ``n``.  Repeated
    (post, pre) pairs are summed, as the reference's ``coalesce()`` does, and
    pairs summing to zero dropped (they add nothing); values must be integral
    and indices inside [0, n), else :class:`ConnectomeError`.  The packed CSR
    arrays are cached on disk (``FIS_CACHE``) keyed by the file's path, size and
    modification time and by ``n``.
    """
    path = Path(path)
    if n is None:
        if comp is None:
            raise ConnectomeError("give n= or comp= (the completeness CSV) for %s" % path)
        n = _csv_rows(comp)
    n = int(n)
    st = path.stat()
    key = "%s|%d|%d|%d|v1" % (path.resolve(), st.st_size, st.st_mtime_ns, n)
    cpath = None
    if cache:
        cpath = _cache_root() / ("upstream_%s.npz" % hashlib.sha1(key.encode()).hexdigest()[:16])
        if cpath.exists():
            try:
                z = np.load(cpath)
                c = Connectome(n, z["row_ptr"], z["col"], z["cnt"])
                c.check_bounds()
                return c
            except Exception:
                pass
    try:
        import pyarrow.parquet as pq
    except ImportError as e:  # pragma: no cover - pyarrow ships with this image
        raise ImportError("reading the upstream parquet needs pyarrow") from e
    t = pq.read_table(str(path), columns=[UPSTREAM_PRE, UPSTREAM_POST, UPSTREAM_VALUE])
    pre = t.column(UPSTREAM_PRE).to_numpy().astype(np.int64)
    post = t.column(UPSTREAM_POST).to_numpy().astype(np.int64)
    val = t.column(UPSTREAM_VALUE).to_numpy().astype(np.float32).astype(np.float64)
    if pre.size and (min(pre.min(), post.min()) < 0 or max(pre.max(), post.max()) >= n):
        raise ConnectomeError("neuron index outside [0, %d) in %s" % (n, path))
    # coalesce: one entry per (pre, post), values summed; the key order is
    # the CSR order (pre major, post ascending)
    ukey, inv = np.unique(pre * n + post, return_inverse=True)
    sums = np.bincount(inv.ravel(), weights=val, minlength=ukey.size)
    c = _from_coo(n, ukey % n, ukey // n, sums)
    if cpath is not None:
        try:
            cpath.parent.mkdir(parents=True, exist_ok=True)
            tmp = cpath.with_suffix(".tmp.npz")
            np.savez(tmp, row_ptr=c.row_ptr, col=c.col, cnt=c.cnt)
            os.replace(tmp, cpath)
        except OSError:
            pass
    return c


def from_upstream(data_dir, cache=True) -> Connectome:
    """``from_parquet`` on an upstream data directory (the reference's
    ``upstream/data``): its connectivity parquet, ``n`` from its completeness
    CSV (data.py:43-44, 236-237)."""
    d = Path(data_dir)
    return from_parquet(d / UPSTREAM_CONN_FILE, comp=d / UPSTREAM_COMP_FILE, cache=cache)


def _out_degrees(rng, n, e, alpha):
    raw = rng.pareto(alpha, n) + 1.0
    scaled = raw * (e / raw.sum())
    cap = n - 1
    d = np.clip(np.floor(scaled), 1, cap).astype(np.int64)
    frac = scaled - np.floor(scaled)
    # Largest-remainder rounding to hit exactly e edges; capped rows are skipped.
    rem = int(e - d.sum())
    order = np.argsort(-frac, kind="stable")
    while rem != 0:
        if rem > 0:
            room = order[d[order] < cap]
            take = room[:rem]
            d[take] += 1
        else:
            room = np.argsort(-d, kind="stable")
            room = room[d[room] > 1]
            take = room[:-rem]
            d[take] -= 1
        if take.size == 0:
            raise ConnectomeError("cannot place %d edges on %d neurons" % (e, n))
        rem = int(e - d.sum())
    return d


def _unique_targets(rng, d, n):
    rows = np.repeat(np.arange(n, dtype=np.int64), d)
    tgt = rng.integers(0, n - 1, size=rows.shape[0], dtype=np.int64)
    # Rows that cover a large share of all neurons are drawn without
    # replacement directly; rejection would need many rounds for them.
    dense = np.flatnonzero(d > (n - 1) // 4)
    if dense.size:
        starts = np.concatenate([[0], np.cumsum(d)[:-1]])
        for r in dense:
            tgt[starts[r]:starts[r] + d[r]] = rng.choice(n - 1, size=int(d[r]), replace=False)
    tgt += tgt >= rows
    key = np.sort(rows * n + tgt)
    for _ in range(1000):
        dup = np.flatnonzero(key[1:] == key[:-1]) + 1
        if dup.size == 0:
            break
        r = key[dup] // n
        t = rng.integers(0, n - 1, size=dup.size, dtype=np.int64)
        t += t >= r
        key[dup] = r * n + t
        key.sort()
    else:  # pragma: no cover - only for degenerate inputs
        raise ConnectomeError("could not draw unique targets")
    return (key % n).astype(np.int32)


def synthetic(n=N_FLYWIRE, e=E_FLYWIRE, seed=0, alpha=1.8, mu=0.9, sigma=1.0,
              max_count=2400, p_inhibitory=0.3, cache=True) -> Connectome:
    """Seeded synthetic connectome with FlyWire-v783 statistics.

    All randomness comes from ``numpy.random.default_rng(seed)`` in a fixed
    order: degrees, targets, counts, signs.  Results are cached on disk keyed by
    every parameter, so repeated test processes do not regenerate 15 M edges.
    """
    if e > n * (n - 1):
        raise ConnectomeError("%d edges do not fit %d neurons without self-loops"
                              % (e, n))
    key = "n%d_e%d_s%d_a%g_m%g_s%g_c%d_p%g_v2" % (n, e, seed, alpha, mu, sigma,
                                                   max_count, p_inhibitory)
    path = None
    if cache:
        root = Path(os.environ.get("FIS_CACHE") or
                    (Path(tempfile.gettempdir()) / "fis_cache"))
        path = root / ("connectome_%s.npz" %
                       hashlib.sha1(key.encode()).hexdigest()[:16])
        if path.exists():
            try:
                z = np.load(path)
                return Connectome(n, z["row_ptr"], z["col"], z["cnt"], seed)
            except Exception:
                pass
    rng = np.random.default_rng(seed)
    d = _out_degrees(rng, n, e, alpha)
    col = _unique_targets(rng, d, n)
    cnt = np.clip(np.rint(rng.lognormal(mu, sigma, e)), 1, max_count).astype(np.int32)
    inh = rng.random(n) < p_inhibitory
    sign = np.where(np.repeat(inh, d), -1, 1).astype(np.int32)
    cnt *= sign
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(d, out=rp[1:])
    c = Connectome(n, rp, col, cnt, seed)
    if path is not None:
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            tmp = path.with_suffix(".tmp.npz")
            np.savez(tmp, row_ptr=rp, col=col, cnt=cnt)
            os.replace(tmp, path)
        except OSError:
            pass
    return c


def sensory_subset(n, k, seed):
    """A seeded random subset of ``k`` neurons (the stimulated population)."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=k, replace=False)).astype(np.int64)
