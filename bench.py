"""Benchmark: batched whole-brain LIF trials on B200.

One bench step is one complete batch: 64 trials x 10,000 steps (1 s of
simulated time each) on the 138,639-neuron, 15,091,983-edge synthetic
connectome, every trial with its own Philox seed, 500-5,000 stimulated
neurons at 50-300 Hz and 1-100 silenced neurons.  The metric is simulated
neuron-steps per second over all GPUs.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Arms:
  default           the B200 engine (libfis_b200.so); ``value`` is timed with
                    the inputs resident on the device, ``e2e`` through
                    ``fis.batch.Batch.run`` with host inputs and host results.
  --impl reference  the reference's algorithm on the host cores (the C port of
                    its default csrmv path under oracle/), all threads, on a
                    bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "fly-in-silico_b200"))
sys.path.insert(0, str(ROOT))

N_TRIALS = 64
SIM_STEPS = 10_000
WORKLOAD = ("batched 64 trials x 10,000 steps (1 s), N=138,639, E=15,091,983 synthetic "
            "connectome; per trial: own Philox seed, 500-5,000 stimulated at 50-300 Hz, "
            "1-100 silenced")
SPEC_SEED = 2024
CONN_SEED = 0
# Update-kernel DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum)
# per trial-neuron and block, from one ncu capture of an 8-trial, 20-step
# launch at steady activity with the caches kept warm, as the live pipeline
# leaves them (83.3 MB: the scratch ring is partly served from L2).  Scaled to
# the bench's launch size by the neurons it processes.
NCU_TRAFFIC_PER_NEURON_BLOCK = 83.34e6 / (8 * 138_639)


def update_bytes_per_neuron_block(core):
    """Algorithmic bytes the update moves per trial-neuron and block of K
    steps: state v, g, refrac read and written (24), flags (1), rates (4),
    kick steps (4), the previous and last step's raster bits (2/8), and the
    scratch ring -- each of the K slots staged into shared memory and stored
    back empty (2 + 2 bytes a slot with the paired int16 ring, 4 + 4 with
    int32)."""
    ring = core.max_block * (4 if core.ring16 else 8)
    return 24 + 1 + 4 + 4 + 2 / 8 + ring


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fis", choices=["fis", "reference"])
    ap.add_argument("--trials", type=int, default=N_TRIALS)
    ap.add_argument("--sim-steps", type=int, default=SIM_STEPS)
    ap.add_argument("--group", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true",
                    help="skip the uneven-duration and serving measurements")
    ap.add_argument("--block-steps", type=int, default=None,
                    help="steps per block (1-20; default 20, the delay lag): shorter blocks "
                         "separate the update's per-block cost from its per-step cost")
    return ap.parse_args()


def uneven_run(conn):
    """256 trials, durations U[500, 20,000] steps, retired in place as they end,
    with the launch shape tuned for a batch of 256 (widths 1-256)."""
    import torch

    from fis.batch import Batch, random_specs
    from fis.tune import core_kwargs, tune

    specs = random_specs(conn.n, 256, SPEC_SEED + 7, (500, 20000))
    best = tune(conn, 256, specs=specs, tag="uneven-mix-%d" % (SPEC_SEED + 7))
    b = Batch(conn, 256, **core_kwargs(best))
    b.run(specs[:8])  # warm the allocations
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    b.run(specs)
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e)
    trial_steps = sum(int(x.steps) for x in specs)
    del b
    torch.cuda.empty_cache()
    return {"value": trial_steps * conn.n / (ms / 1000.0), "unit": "neuron-steps/s",
            "trials": 256, "durations": "U[500, 20000] steps", "trial_steps": trial_steps,
            "ms": ms, "tuned": {k: best[k] for k in best if k != "candidates"},
            "autotune_candidates": len(best["candidates"]),
            "how": "host trial specs in, host counts out; finished trials frozen "
                   "in place until the longest ends"}


SERVING_RATES_HZ = (2.0, 10.0, 50.0)


def serving_run(conn, launch, plain_value, rates=SERVING_RATES_HZ, count=100):
    """Open-loop streams of ``count`` requests at each Poisson arrival rate:
    1-64 trials and 1,000-50,000 steps per request, 10 ms bins.  Latency is
    arrival to result on the host; it splits into the admission wait (queued
    until slots and recording memory are free) and the service time."""
    import torch

    from fis.serve import Server, poisson_requests

    lines = []
    srv = Server(conn, capacity=256, **launch)
    for j, hz in enumerate(rates):
        reqs = poisson_requests(conn.n, SPEC_SEED + 9 + j, hz, count, trials=(1, 64),
                                steps=(1000, 50000), bin_steps=100)
        srv.replies = []
        t0 = time.perf_counter()
        replies = srv.run(reqs, realtime=True)
        wall = time.perf_counter() - t0
        srv.core.check_errors()
        lat = Server.latency_stats(replies)
        units = sum(r.trial_steps for r in replies) * conn.n
        lines.append({"arrival_rate_hz": hz, "requests": len(replies), **lat,
                      "throughput": units / wall, "unit": "neuron-steps/s", "wall_s": wall,
                      "serial_plain_s": units / plain_value if plain_value else None})
    del srv
    torch.cuda.empty_cache()
    return {"rates": lines,
            "how": "Poisson arrivals, %d requests per rate, admission by free slots and "
                   "recording memory, continuous batching into 256 slots, 10 ms bins per "
                   "request; latency = wait (arrival to admission) + service" % count}


def activity_sweep(conn, steps=SIM_STEPS, fracs=(0.001, 0.01, 0.10)):
    """The plain single trial at 0.1 %, 1 % and 10 % Poisson drive (150 Hz)
    for ``steps`` steps through ``fis.batch.Batch``: neuron-steps/s from CUDA
    events around the device work, and spikes per step from the counts."""
    import numpy as np
    import torch

    from fis.batch import Batch, TrialSpec

    out = []
    b = Batch(conn, 1, group=1)
    for frac in fracs:
        rng = np.random.default_rng(int(frac * 1e4) + 17)
        stim = np.sort(rng.choice(conn.n, size=int(frac * conn.n), replace=False))
        spec = TrialSpec(seed=1234 + int(frac * 1e4), steps=steps, stim=stim, rate_hz=150.0)
        b.run([spec])  # warm
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        counts = b.run([spec])
        e.record()
        torch.cuda.synchronize()
        ms = s.elapsed_time(e)
        out.append({"drive_frac": frac, "driven": int(stim.size), "steps": steps,
                    "value": conn.n * steps / (ms / 1000.0), "unit": "neuron-steps/s",
                    "ms": ms, "spikes_per_step": float(counts.sum()) / steps})
    del b
    torch.cuda.empty_cache()
    return out


def red_rate_peak(device, words=16 << 20, iters=256):
    """The sustained rate of 32-bit L2 atomic adds (adds per second), from the
    library's calibration kernel on a 64 MB buffer that stays in L2: the
    ceiling of the scatter, which makes one such add per pushed synapse."""
    import ctypes

    import torch

    import fis._lib as L

    lib = L.load()
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    ctas = sms * 8
    buf = torch.zeros(words, dtype=torch.int32, device=device)
    st = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    best = 0.0
    for rep in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        L.check(lib.fis_red_rate(ctypes.c_void_p(buf.data_ptr()), words, iters, ctas, st),
                "fis_red_rate")
        e.record()
        torch.cuda.synchronize(device)
        if rep:  # the first launch warms the buffer into L2
            best = max(best, ctas * 256 * iters / (s.elapsed_time(e) / 1000.0))
    del buf
    return best


def propagation_roofline(core, batch, specs, hbm, peak_kind, warm_blocks=10, blocks=20):
    """Roofline of the propagation kernel (k_phase_a: the scatter of the spikes
    that reach a block, and the block's Poisson drive), each launch timed alone
    with CUDA events on its stream, over ``blocks`` blocks of the resident
    64-trial workload at steady activity.

    Algorithmic HBM bytes of one launch, from the spikes it delivers (those of
    the previous block, read back from the trials' recordings): per spike
    chunk (work item) its list entry (4 B) and row bounds (2 x 8 B), 4 B per
    edge pushed, the rates of the group (4 B per trial-neuron) and the kick
    words of driven neurons (4 B).  Each pushed edge is also one 32-bit atomic
    add in L2, reported beside as L2 bytes (4 B read + 4 B written)."""
    import numpy as np
    import torch

    dev = core.device
    deg = torch.as_tensor(core.conn.out_degree().astype(np.int64), device=dev)
    nch = core.nchunks.to(torch.int64)
    rec = batch.last_recording[:, 0]          # [B][N] spikes so far, slot order
    driven = (core.rates > 0).to(torch.int64)
    for b in range(len(specs)):
        t = core.trials[b]
        t.start, t.end = core.step, core.step + (warm_blocks + blocks + 1) * core.max_block
    core.mark_trials()
    core.reset_slots(slice(None))
    rec.zero_()
    core.advance((warm_blocks - 1) * core.max_block)
    prev = rec.clone()
    core.advance(core.max_block)
    G = core.group
    evs, bytes_, edges = [], [], []
    for _ in range(blocks):
        pairs = []

        def timer(st, start, pairs=pairs):
            if start:
                pairs.append([torch.cuda.Event(enable_timing=True),
                              torch.cuda.Event(enable_timing=True)])
            pairs[-1][0 if start else 1].record(torch.cuda.current_stream(dev))

        cur = rec.clone()
        delivered = cur - prev                # the spikes this block's scatter pushes
        prev = cur
        core.block(core.max_block, scatter_timer=timer)
        for j, g0 in enumerate(range(0, core.batch, G)):
            per = delivered[g0:g0 + G].sum(0)
            items = int((per * nch).sum())
            e = int((per * deg).sum())
            nb = min(G, core.batch - g0)
            b = 20 * items + 4 * e + 4 * nb * core.n + 4 * int(driven[g0:g0 + G].sum())
            evs.append(pairs[j])
            bytes_.append(b)
            edges.append(e)
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in evs]
    core.check_errors()
    sec = sum(ms) / 1000.0
    achieved = sum(bytes_) / sec / 1e9
    adds = sum(edges) / sec
    red_peak = red_rate_peak(dev)
    return {"bound": "l2_atomics", "achieved": adds / 1e9, "peak": red_peak / 1e9,
            "unit": "G atomic adds/s", "frac": adds / red_peak,
            "peak_kind": "measured here: fis_red_rate, random 32-bit red.add into 64 MB in L2",
            "hbm": {"achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                    "peak_kind": peak_kind},
            "traffic": None, "kernel": "k_phase_a",
            "launch_ms": statistics.mean(ms), "launches": len(ms),
            "algorithmic_bytes_per_launch": statistics.mean(bytes_),
            "edges_per_launch": statistics.mean(edges),
            "l2_atomic_gbs": 8.0 * adds / 1e9,
            "how": "each phase-A launch alone (not overlapped), %d blocks of the 64-trial "
                   "workload after %d warm blocks; bytes and atomic adds from the spikes "
                   "each launch delivers" % (blocks, warm_blocks)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = Path("/tmp/fis_clocks_%d.csv" % os.getpid())

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def cpu_sample(conn, specs, steps, threads):
    """The reference's CPU algorithm (csrmv over every edge, the default path)."""
    import numpy as np

    from oracle import oracle as O
    from fis.batch import host_rows

    flags, rates = host_rows(specs, conn.n)
    o = O.Oracle.from_connectome(conn, batch=len(specs), no_refractory=None)
    o.rates[:] = rates
    o.refrac_steps[(flags & 16) != 0] = 0.0
    o.refrac[:] = o.refrac_steps
    sil = (flags & 32) != 0
    o.m_out[sil] = 0.0
    o.m_in[sil] = 0.0
    o.seeds[:] = np.array([s.seed for s in specs], dtype=np.uint64)
    o.streams[:] = 0
    t = time.perf_counter()
    o.run(steps, mode=O.Oracle.CSRMV, threads=threads)
    return time.perf_counter() - t


def reference_arm(args, rank):
    if rank != 0:
        return 0
    import fis.connectome as C
    from fis.batch import random_specs

    threads = os.cpu_count() or 1
    conn = C.synthetic(seed=CONN_SEED)
    specs = random_specs(conn.n, args.trials, SPEC_SEED, args.sim_steps)
    sample_steps = 2
    for _ in range(args.warmup):
        cpu_sample(conn, specs, sample_steps, threads)
    times = [cpu_sample(conn, specs, sample_steps, threads) for _ in range(args.steps)]
    total = sum(times)
    units = args.trials * conn.n * sample_steps * args.steps
    value = units / total
    line = {
        "impl": "reference", "metric": "batched neuron-steps/s", "value": value,
        "unit": "neuron-steps/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "trials": args.trials, "sim_steps": args.sim_steps,
                   "sample": "%d trials x %d steps per bench step" % (args.trials, sample_steps)},
        "cpu_baseline": {"value": value, "unit": "neuron-steps/s", "cores": threads,
                         "kind": "port",
                         "sample": "%d trials x %d steps, csrmv over all edges (the "
                                   "reference's default CPU path), C port in oracle/"
                                   % (args.trials, sample_steps)},
        "e2e": {"value": value, "unit": "neuron-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return reference_arm(args, rank)

    import numpy as np
    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist

    import fis.connectome as C
    from fis.batch import Batch, random_specs

    from fis.engine import Core
    from fis.tune import core_kwargs, tune

    conn = C.synthetic(seed=CONN_SEED)
    specs = random_specs(conn.n, args.trials, SPEC_SEED + 1000 * rank, args.sim_steps)
    if args.group is None:
        best = tune(conn, args.trials, specs=specs, tag="bench-mix-%d" % (SPEC_SEED + 1000 * rank))
    else:
        best = {"group": args.group, "chunk": None, "ring": None, "scatter_mode": None,
                "scat_ctas": 0, "drive_ctas": 0, "update_streams": 1, "update_tiles": None,
                "candidates": []}
    core = Core(conn, args.trials, raster=False, max_block=args.block_steps or 20,
                **core_kwargs(best))
    batch = Batch(conn, args.trials, core=core)
    core = batch.core
    slots = list(range(args.trials))
    batch.load(slots, specs)

    def resident_run(events=None, every=1):
        for b in slots:
            t = core.trials[b]
            t.start = core.step
            t.end = core.step + specs[b].steps
        core.mark_trials()
        core.reset_slots(slice(None))
        for r in batch.recordings():
            r.zero_()
        core.advance(args.sim_steps, events=events, every=every)

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()

    def max_over_ranks(x):
        if pg is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        resident_run()
    blocks = -(-args.sim_steps // core.max_block)
    upd_per_run = blocks * (-(-args.trials // core.group))
    n_pairs = 64
    every = max(1, upd_per_run // n_pairs)
    events = [[torch.cuda.Event(enable_timing=True) for _ in range(2 * n_pairs)]
              for _ in range(args.steps)]

    gpu_index = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            gpu_index = int(vis.split(",")[local])
        except ValueError:
            pass
    sampler = ClockSampler(gpu_index)
    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with sampler:
        time.sleep(0.3)
        barrier()
        start.record()
        for k in range(args.steps):
            resident_run(events=events[k], every=every)
        end.record()
        barrier()
    ms = max_over_ranks(start.elapsed_time(end))
    core.check_errors()
    clocks = sampler.summary()
    durs = []
    for evs in events:
        for j in range(n_pairs):
            d = evs[2 * j].elapsed_time(evs[2 * j + 1])
            if d > 0:
                durs.append(d)
    upd_ms = statistics.mean(durs) if durs else None

    units_rank = args.trials * conn.n * args.sim_steps
    value = world * units_rank * args.steps / (ms / 1000.0)

    # end to end through the public API: host specs in, host counts out; one
    # untimed run first warms the pinned staging buffers and the path
    batch.run(specs)
    barrier()
    t0 = time.perf_counter()
    for _ in batch.run_many(specs for _ in range(args.steps)):
        pass
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = world * units_rank * args.steps / e2e_s
    # bytes copied per run: the sparse trial rows, the trial table and the
    # recording pointer table in; the per-trial counts out
    h2d = batch.last_h2d_bytes + args.trials * 48 + 8 * len(batch.recordings())
    d2h = batch.last_d2h_bytes

    # the plain single-trial step through the reference-compatible API
    plain = None
    if rank == 0:
        from fis import sim

        rng = np.random.default_rng(1)
        drive = np.sort(rng.choice(conn.n, 2249, replace=False))
        eng = sim.build_engine(weights=conn, batch=1, seed=0, no_refractory=drive, graphs=True)
        rates = torch.zeros(1, conn.n, device="cuda")
        rates[0, torch.as_tensor(drive, device="cuda")] = 150.0
        for _ in range(50):
            eng.step(rates)
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n_plain = 2000
        s0.record()
        for _ in range(n_plain):
            eng.step(rates)
        s1.record()
        torch.cuda.synchronize()
        pms = s0.elapsed_time(s1) / n_plain
        plain = {"value": conn.n / (pms / 1000.0), "unit": "neuron-steps/s",
                 "ms_per_step": pms,
                 "how": "Engine.step() per 0.1 ms tick, 1 trial, CUDA graph, 2,249 driven "
                        "at 150 Hz"}
        del eng

    hbm, peak_kind = peaks()
    roof = None
    if upd_ms:
        G = core.group
        bytes_launch = G * conn.n * update_bytes_per_neuron_block(core)
        achieved = bytes_launch / (upd_ms / 1000.0) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm,
                "traffic": NCU_TRAFFIC_PER_NEURON_BLOCK * G * conn.n,
                "kernel": "k_update", "launch_ms": upd_ms,
                "algorithmic_bytes_per_launch": bytes_launch,
                "bytes_per_neuron_block": update_bytes_per_neuron_block(core),
                "peak_kind": peak_kind}

    uneven = serving = sweep = prop = None
    if rank == 0 and world == 1 and not args.quick:
        prop = propagation_roofline(core, batch, specs, hbm, peak_kind)
        sweep = activity_sweep(conn)
        uneven = uneven_run(conn)
        serving = serving_run(conn, core_kwargs(best), plain["value"] if plain else None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample_steps = 10
        dt = cpu_sample(conn, specs, sample_steps, threads)
        cpu = {"value": args.trials * conn.n * sample_steps / dt, "unit": "neuron-steps/s",
               "cores": threads, "kind": "port",
               "sample": "%d trials x %d steps, csrmv over all edges (the reference's default "
                         "CPU path), C port in oracle/" % (args.trials, sample_steps)}

    if rank == 0:
        line = {
            "metric": "batched neuron-steps/s", "value": value, "unit": "neuron-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "trials_per_gpu": args.trials,
                       "sim_steps": args.sim_steps, "trial_group": core.group,
                       "scatter_chunk": core.chunk,
                       "ring": "int16 pairs" if core.ring16 else "int32",
                       "scatter_mode": core.scatter_mode,
                       "phase_a_ctas_per_8_sms": [core.scat_ctas, core.drive_ctas],
                       "autotune_candidates": len(best["candidates"]),
                       "update_streams": core.update_streams,
                       "update_tiles": core.update_tiles,
                       # per candidate: its launch, us per step, and (the three
                       # fastest) us per step in the longer runoff that decides
                       "autotune": [[c[k] for k in ("group", "ring", "scatter_mode", "chunk",
                                                    "scat_ctas", "drive_ctas",
                                                    "update_streams", "update_tiles")]
                                    + [round(c["ms_per_step"] * 1000.0, 2)]
                                    + ([round(c["runoff_ms_per_step"] * 1000.0, 2)]
                                       if "runoff_ms_per_step" in c else [])
                                    for c in best["candidates"]],
                       "block_steps": core.max_block,
                       "l2": "inputs larger than L2 (trial state 150 MB, spike lists "
                             "%.0f MB, CSR 60 MB)" % (core.lists.numel() * 4 / 1e6),
                       "parallelism": "replicas x%d" % world},
            "clocks": clocks,
            "e2e": {"value": e2e, "unit": "neuron-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps * blocks * core.launches_per_block(),
            "roofline": roof,
            "roofline_propagation": prop,
            "plain_1trial": plain,
            "batched_over_plain": (value / world) / plain["value"] if plain else None,
            "uneven_256": uneven,
            "activity_sweep_1trial": sweep,
            "serving": serving,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
