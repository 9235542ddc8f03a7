"""Autotuner for the block launch shape, cached per (N, E, batch, GPU).

Tunables (all exact: they change scheduling and storage, never results):

* ``group`` -- the batch width of one launch pair (trials per phase-A +
  update launch), from 1 up to the whole batch (8-256 at a batch of 256).
  Narrow groups keep the scratch ring in L2; wide groups cut launches and the
  tail of the last wave.
* ``ring`` -- the scratch ring's layout: ``int16`` interleaves two trials in
  each 32-bit word (rows of trial pairs, half the bytes; exact when no
  neuron's incoming |count| sum reaches 2**15), ``int32`` one row per trial.
* ``scatter_mode`` -- the warps a spiking row gets: 0 = a warp per work item
  (spike, chunk of its row), i.e. ceil(degree / chunk) warps per row, one
  item per warp at a time; 1 = tasks of 1-32 work items per warp (about two
  tasks per warp of the grid), resolved together and walked as one stream of
  edge quads (a row shares its warp with up to 31 others).
* ``chunk`` -- edges per work item (the row split behind warps-per-row):
  256, 512 or 1024.
* ``scat_ctas`` / ``drive_ctas`` -- phase-A CTAs per 8 SMs for the scatter and
  the Poisson drive (0 = the library's default for the mode).
* ``update_streams`` -- 1, or 2: consecutive updates (of different trial
  groups, so independent) alternate between two streams and overlap their
  tails.
* ``update_tiles`` -- 1 (one 256-neuron tile per update CTA) or 2 (streamed
  tiles: each CTA pipelines a run of tiles, the next one's input fetched by
  bulk copies while the current one's steps run).

The block length stays the delay lag (20 steps), the longest that keeps the
steps of a block independent.  The search is coordinate-wise: group x ring at
the default launch, then scatter mode x chunk at the best of those, then the
phase-A grid, then the update streams, then the update form (one tile per
CTA or streamed tiles); the three fastest then run again over three times
the steps, and that runoff picks the winner.  Each candidate runs a short
seeded trial mix (the caller's own trials when given) on a scratch engine
and is timed with CUDA events; the winner is stored in a JSON cache
(``FIS_TUNE_CACHE`` or ``~/.cache/fis/tune.json``).
"""

from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np
import torch

from .connectome import Connectome
from .engine import Core

KEYS = ("group", "ring", "scatter_mode", "chunk", "scat_ctas", "drive_ctas",
        "update_streams", "update_tiles")


def cache_path() -> Path:
    p = os.environ.get("FIS_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "fis" / "tune.json"


def _key(conn: Connectome, batch: int) -> str:
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return "%s|n=%d|e=%d|b=%d|v7" % (name, conn.n, conn.nnz, batch)


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


def default_groups(batch):
    return sorted({g for g in (1, 2, 4, 8, 16, 32, 64, 128, 256) if g <= batch} | {batch})


def _load_specs(core: Core, specs):
    """The caller's own trials (``fis.batch.TrialSpec``) in the scratch core,
    running past every candidate's steps."""
    from .batch import Batch

    Batch(core.conn, core.batch, core=core).load(list(range(len(specs))), specs)
    for b in range(core.batch):
        core.trials[b].end = 2 ** 62
    core.mark_trials()


def tune(conn: Connectome, batch: int, params=None, groups=None, rings=None, modes=(1, 0),
         chunks=None, grids=None, steps=1000, reps=2, use_cache=True, verbose=False,
         specs=None, tag="mix", runoff=3) -> dict:
    """Best launch shape ``{group, ring, scatter_mode, chunk, scat_ctas,
    drive_ctas, update_streams, update_tiles, ms_per_step, candidates}`` for
    this connectome and batch.  ``specs``: time the candidates on these trials
    (``batch`` of them) instead of the seeded 2 % mix -- the choices differ by a
    few percent, so the workload that will run is the one to tune on; ``tag``
    names it in the cache key.  ``runoff``: how many of the fastest candidates
    are timed again, over three times the steps, to pick the winner."""
    key = _key(conn, batch) + "|" + str(tag)
    cache = load_cache() if use_cache else {}
    if key in cache:
        return cache[key]
    maxdeg = int(conn.out_degree().max()) if conn.n else 0
    base_chunk = max(256, 128 * -(-maxdeg // (255 * 128)))
    chunks = chunks or sorted({base_chunk, max(base_chunk, 512), max(base_chunk, 1024)})
    groups = groups or default_groups(batch)
    fits16 = conn.exactness()["max_abs_row_sum"] < (1 << 15)
    rings = rings or (["int16", "int32"] if fits16 else ["int32"])
    grids = grids or [(8, 16), (8, 8), (4, 16), (12, 16), (8, 24), (16, 24)]
    results = []
    cores = {}

    def core_for(ring, chunk):
        if (ring, chunk) not in cores:
            cores.clear()
            torch.cuda.empty_cache()
            c = Core(conn, batch, params=params, chunk=chunk, group=groups[0], ring=ring,
                     raster=False)
            if specs is not None:
                _load_specs(c, specs)
            else:
                _mix(c)
            cores[(ring, chunk)] = c
        return cores[(ring, chunk)]

    def seen(cand):
        return any(all(r[k] == cand[k] for k in KEYS) for r in results)

    def trial(cand):
        c = core_for(cand["ring"], cand["chunk"])
        c.set_group(cand["group"])
        c.set_launch(cand["scatter_mode"], cand["scat_ctas"], cand["drive_ctas"],
                     cand["update_streams"], cand["update_tiles"])
        ms = _time(c, steps, reps)
        results.append(dict(cand, ms_per_step=ms))
        if verbose:
            print("tune: %s  %.4f ms/step" % (" ".join("%s=%s" % (k, cand[k]) for k in KEYS), ms),
                  flush=True)

    def best_so_far():
        return {k: min(results, key=lambda r: r["ms_per_step"])[k] for k in KEYS}

    best = {"group": groups[0], "ring": rings[0], "scatter_mode": modes[0],
            "chunk": base_chunk, "scat_ctas": 0, "drive_ctas": 0, "update_streams": 1,
            "update_tiles": 1}
    # 1. batch width x ring layout at the default launch
    for ring in rings:
        for g in groups:
            trial(dict(best, ring=ring, group=g))
    best = best_so_far()
    # 2. warps per row: scatter mode x chunk
    for chunk in chunks:
        for mode in modes:
            cand = dict(best, chunk=chunk, scatter_mode=mode)
            if not seen(cand):
                trial(cand)
    best = best_so_far()
    # 3. the phase-A grid for that mode
    for sc, dr in grids:
        cand = dict(best, scat_ctas=sc, drive_ctas=dr)
        if not seen(cand):
            trial(cand)
    best = best_so_far()
    # 4. one or two update streams, at the best width and its neighbours
    for g in groups:
        if best["group"] // 2 <= g <= best["group"] * 2:
            cand = dict(best, group=g, update_streams=2)
            if not seen(cand):
                trial(cand)
    best = best_so_far()
    # 5. one tile per update CTA, or the streamed tiles
    for tiles in (1, 2):
        cand = dict(best, update_tiles=tiles)
        if not seen(cand):
            trial(cand)
    # 6. runoff: the leaders are often within a percent of each other, so the
    # three fastest are timed again over three times the steps and the
    # runoff decides
    top = sorted(results, key=lambda r: r["ms_per_step"])[:runoff]
    if len(top) > 1:
        for r in top:
            c = core_for(r["ring"], r["chunk"])
            c.set_group(r["group"])
            c.set_launch(r["scatter_mode"], r["scat_ctas"], r["drive_ctas"],
                         r["update_streams"], r["update_tiles"])
            r["runoff_ms_per_step"] = _time(c, 3 * steps, reps)
        win = min(top, key=lambda r: r["runoff_ms_per_step"])
    else:
        win = min(results, key=lambda r: r["ms_per_step"])
    cores.clear()
    torch.cuda.empty_cache()
    out = dict(win, candidates=results)
    if use_cache:
        cache[key] = out
        try:
            p = cache_path()
            p.parent.mkdir(parents=True, exist_ok=True)
            p.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    return out


def core_kwargs(best: dict) -> dict:
    """The Core arguments of a tuning result."""
    return {"group": best["group"], "chunk": best.get("chunk"), "ring": best.get("ring"),
            "scatter_mode": best.get("scatter_mode"), "scat_ctas": best.get("scat_ctas", 0),
            "drive_ctas": best.get("drive_ctas", 0),
            "update_streams": best.get("update_streams", 1),
            "update_tiles": best.get("update_tiles")}
