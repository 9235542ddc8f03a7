"""Autotuner for the block launch shape, cached per (N, E, batch, GPU).

Tunables (all exact: they change scheduling, never results):

* ``group`` -- trials per launch of the block (the batch width of one
  scatter + update pair).  Narrow groups keep the scratch ring
  ([K][group][NR] int32) resident in L2; wide groups cut launches and the
  tail of the last wave.
* ``chunk`` -- edges per scatter work item (a warp walks one chunk of one
  spiking row): the load balance over the Pareto-tailed out-degrees.

The ring layout is fixed (trial-major rows padded to 256 neurons, one update
CTA per trial tile); the block length is the delay lag (20 steps), the longest
that keeps steps within a block independent.

Each candidate runs a short seeded trial mix on a scratch engine and is timed
with CUDA events; the winner is stored in a JSON cache (``FIS_TUNE_CACHE`` or
``~/.cache/fis/tune.json``).
"""

from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np
import torch

from .connectome import Connectome
from .engine import Core


def cache_path() -> Path:
    p = os.environ.get("FIS_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "fis" / "tune.json"


def _key(conn: Connectome, batch: int) -> str:
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return "%s|n=%d|e=%d|b=%d" % (name, conn.n, conn.nnz, batch)


def load_cache() -> dict:
    p = cache_path()
    try:
        return json.loads(p.read_text())
    except Exception:
        return {}


def _mix(core: Core, seed=7, frac=0.02, rate=150.0):
    """Drive a seeded 2 % of the neurons of every slot (the working point)."""
    rng = np.random.default_rng(seed)
    n = core.n
    for b in range(core.batch):
        idx = torch.as_tensor(np.sort(rng.choice(n, max(1, int(frac * n)), replace=False)),
                              device=core.device)
        core.rates[b].zero_()
        core.rates[b, idx] = rate
        core.trials[b].seed = int(rng.integers(0, 2 ** 62))
        core.trials[b].start = core.step
        core.trials[b].end = 2 ** 62
    core.mark_trials()
    core.reset_slots(slice(None))


def _time(core: Core, steps: int, reps: int) -> float:
    core.advance(core.max_block * 10)  # warm: lists, caches, clocks
    torch.cuda.synchronize(core.device)
    best = float("inf")
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        core.advance(steps)
        e.record()
        torch.cuda.synchronize(core.device)
        best = min(best, s.elapsed_time(e))
    return best / steps


def tune(conn: Connectome, batch: int, params=None, groups=None, chunks=None, steps=400,
         reps=2, use_cache=True, verbose=False) -> dict:
    """Best ``{"group", "chunk", "ms_per_step"}`` for this connectome and batch."""
    key = _key(conn, batch)
    cache = load_cache() if use_cache else {}
    if key in cache:
        return cache[key]
    deg = conn.out_degree()
    maxdeg = int(deg.max()) if conn.n else 0
    base_chunk = max(256, 128 * -(-maxdeg // (255 * 128)))
    chunks = chunks or sorted({base_chunk, max(base_chunk, 512), max(base_chunk, 1024)})
    groups = groups or sorted({g for g in (1, 2, 4, 8, 16, 32, 64, 128, 256) if g <= batch}
                              | {batch})
    results = []
    for chunk in chunks:
        core = Core(conn, batch, params=params, chunk=chunk, group=groups[0], raster=False)
        _mix(core)
        for g in groups:
            core.set_group(g)
            ms = _time(core, steps, reps)
            results.append({"group": g, "chunk": chunk, "ms_per_step": ms})
            if verbose:
                print("tune: group %3d chunk %4d  %.4f ms/step" % (g, chunk, ms), flush=True)
        del core
        torch.cuda.empty_cache()
    best = min(results, key=lambda r: r["ms_per_step"])
    best = dict(best, candidates=results)
    if use_cache:
        cache[key] = best
        try:
            p = cache_path()
            p.parent.mkdir(parents=True, exist_ok=True)
            p.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    return best
