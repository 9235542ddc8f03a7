"""Experiment serving: continuous batching of requests into running trial slots.

The reference's worker runs one job at a time and rebuilds the engine and its
19 CUDA graphs per job (``lab/flybrain/worker.py:298-313, 454-505``,
``jobs._job_stim`` ``jobs.py:367-412``).  Here one engine holds every trial
slot for the life of the server:

* a request carries 1..N trials (each a :class:`fis.batch.TrialSpec`) and a
  recording bin width; it is admitted as soon as enough slots are free and the
  device memory it needs (state rows are pre-allocated; its recording buffer
  int32 [n_bins][N] is not) fits the budget;
* admitted trials start at the next block boundary and run in the same
  launches as everything else on the GPU; a trial that finishes stops being
  updated in place (its slot is frozen, then freed when the whole request is
  done);
* results are the reference's ``Result`` fields summed over the request's
  trials: spike counts per neuron and the binned raster ``int16 [n_bins, N]``
  (``sim.py:1040-1081``); latency is measured from arrival to result on the
  host.

A request's result does not depend on what else runs: its trials' drive is
keyed by their own seeds and own steps, their inputs come only from their own
spikes, and integer accumulation is order-free.
"""

from __future__ import annotations

import heapq
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .batch import Batch, TrialSpec
from .connectome import Connectome


@dataclass
class Request:
    trials: list
    bin_steps: int | None = None     # None: one bin over the longest trial
    arrival: float = 0.0             # seconds on the server's clock
    rid: int = -1

    def steps(self):
        return max(int(t.steps) for t in self.trials)

    def n_bins(self):
        bs = self.bin_steps or self.steps()
        return max(1, -(-self.steps() // bs))


@dataclass
class Reply:
    rid: int
    counts: np.ndarray               # int64 [N], summed over the request's trials
    bins: np.ndarray                 # int16 [n_bins, N]
    arrival: float
    admitted: float
    finished: float
    trial_steps: int
    slots: list = field(default_factory=list)
    released: float = 0.0            # its slots were freed (its trials had all ended)

    @property
    def latency(self):
        return self.finished - self.arrival

    @property
    def wait(self):
        """Time from arrival to admission (queued for slots or memory)."""
        return self.admitted - self.arrival

    @property
    def service(self):
        """Time from admission to the result on the host."""
        return self.finished - self.admitted


class Server:
    """Slots on one GPU, filled from a queue as they free up."""

    def __init__(self, conn: Connectome, capacity: int = 256, params=None, device="cuda",
                 group=None, chunk=None, memory_budget: int | None = None,
                 advance_steps: int = 200, **launch):
        self.batch = Batch(conn, capacity, params=params, device=device, group=group,
                           chunk=chunk, **launch)
        self.core = self.batch.core
        self.n = self.core.n
        self.capacity = capacity
        self.free = list(range(capacity))
        heapq.heapify(self.free)
        self.queue: list = []                 # arrived, not yet admitted (FIFO)
        self.running: dict = {}               # rid -> (request, slots, end_step, rec index, t_admit)
        self.replies: list = []
        self._next_rid = 0
        if memory_budget is None:
            free_b, _ = torch.cuda.mem_get_info(self.core.device)
            memory_budget = int(free_b * 0.8)
        self.memory_budget = int(memory_budget)
        self.memory_used = 0
        for b in range(capacity):             # idle slots: never active
            self.core.trials[b].start = self.core.trials[b].end = 0
        self.core.mark_trials()
        # steps enqueued per turn of the serving loop (cut at the next trial
        # end): new arrivals wait at most this long for admission
        self.advance_steps = max(1, int(advance_steps))
        self._in_flight = None                # event after the previous turn's work
        self._copy_stream = None              # recordings of retired requests go out here
        self._retiring = []                   # retired, their recordings on the way out
        self.clock0 = time.perf_counter()

    # --- host side --------------------------------------------------------

    def now(self):
        return time.perf_counter() - self.clock0

    def request_bytes(self, req: Request) -> int:
        """Device memory a request adds: its recording buffer."""
        return req.n_bins() * self.n * 4

    def submit(self, req: Request) -> int:
        if req.rid < 0:
            req.rid = self._next_rid
            self._next_rid += 1
        if not req.trials:
            raise ValueError("a request needs at least one trial")
        if len(req.trials) > self.capacity:
            raise ValueError("%d trials exceed the %d slots" % (len(req.trials), self.capacity))
        if self.request_bytes(req) > self.memory_budget:
            raise MemoryError("request %d needs %d bytes of recording, budget %d"
                              % (req.rid, self.request_bytes(req), self.memory_budget))
        self.queue.append(req)
        return req.rid

    def _admit(self):
        """Admit queued requests in arrival order while slots and memory allow."""
        admitted = []
        while self.queue:
            req = self.queue[0]
            need = self.request_bytes(req)
            if len(req.trials) > len(self.free) or self.memory_used + need > self.memory_budget:
                break
            self.queue.pop(0)
            slots = sorted(heapq.heappop(self.free) for _ in req.trials)
            for t in req.trials:
                t.bin_steps = req.bin_steps or req.steps()
            rec = torch.zeros((req.n_bins(), self.n), dtype=torch.int32, device=self.core.device)
            self.batch.load(slots, req.trials, rec=rec)
            self.memory_used += need
            self.running[req.rid] = (req, slots, self.core.step + req.steps(), rec, self.now())
            admitted.append(req.rid)
        return admitted

    def _retire(self):
        """Retire the requests whose trials end with the stretch just enqueued.

        Their slots are freed at once (a new occupant's load runs after that
        stretch in stream order), while their recordings are reduced and
        copied to pinned host memory on a copy stream that waits only for that
        stretch, so the device keeps running; ``_finish`` turns them into
        replies once the copies have landed.
        """
        done = [rid for rid, (_, _, end, _, _) in self.running.items() if self.core.step >= end]
        if not done:
            return done
        dev = self.core.device
        if self._copy_stream is None:
            self._copy_stream = torch.cuda.Stream(dev)
        cs = self._copy_stream
        cs.wait_event(self._in_flight)
        for rid in done:
            req, slots, end, rec, t_adm = self.running.pop(rid)
            with torch.cuda.stream(cs):
                bins = torch.empty(rec.shape, dtype=torch.int16, pin_memory=True)
                counts = torch.empty(rec.shape[1], dtype=torch.int64, pin_memory=True)
                bins.copy_(rec.to(torch.int16), non_blocking=True)
                counts.copy_(rec.to(torch.int64).sum(0), non_blocking=True)
                err = self.core.errors_async()
                landed = torch.cuda.Event()
                landed.record(cs)
            rec.record_stream(cs)
            for b in slots:
                self.core.trials[b].start = self.core.trials[b].end = 0
                self.batch.release(b)
                heapq.heappush(self.free, b)
            self.core.mark_trials()
            self._retiring.append((rid, req, slots, t_adm, landed, bins, counts, err, rec,
                                   self.now()))
        return done

    def _finish(self, wait=False):
        """Replies for the retired requests whose recordings have landed."""
        keep = []
        for item in self._retiring:
            rid, req, slots, t_adm, landed, bins, counts, err, rec, t_rel = item
            if not (wait or landed.query()):
                keep.append(item)
                continue
            landed.synchronize()
            self.core.raise_errors(err)
            self.memory_used -= self.request_bytes(req)
            self.replies.append(Reply(rid, counts.numpy(), bins.numpy(), req.arrival, t_adm,
                                      self.now(), sum(int(t.steps) for t in req.trials), slots,
                                      t_rel))
        self._retiring = keep

    def _active_rows(self):
        """Slots [0, hi) hold every running trial; launches stop at hi."""
        hi = 0
        for _, slots, _, _, _ in self.running.values():
            hi = max(hi, max(slots) + 1)
        return hi

    def step_block(self):
        """Advance everything running by up to ``advance_steps`` steps.

        The stretch is cut at the next trial end, so every request finishes
        exactly on a block boundary, and it runs as the engine's native block
        loop (one library call, trial groups overlapped) rather than block by
        block from Python, whose per-block host cost exceeds the device time of
        a block when few trials run.  At most two stretches are in flight: the
        host waits for the previous one before enqueueing another, so a
        request admitted now does not queue behind a long backlog.
        """
        if not self.running:
            return 0
        ends = [end for _, _, end, _, _ in self.running.values()]
        k = max(1, min(self.advance_steps, min(ends) - self.core.step))
        self.core.advance(k, rows=self._active_rows())
        done = torch.cuda.Event()
        done.record(torch.cuda.current_stream(self.core.device))
        if self._in_flight is not None:
            self._in_flight.synchronize()
        self._in_flight = done
        return k

    # --- driving ------------------------------------------------------------

    def run(self, requests, realtime=True, max_idle_wait=0.05):
        """Serve ``requests`` (with ``arrival`` offsets in seconds) to completion.

        With ``realtime`` the arrivals follow the wall clock (an open-loop
        stream); otherwise every request is queued at once.  Returns the
        replies in completion order.
        """
        pending = sorted(requests, key=lambda r: r.arrival)
        self.clock0 = time.perf_counter()
        i = 0
        while i < len(pending) or self.queue or self.running or self._retiring:
            now = self.now()
            while i < len(pending) and (not realtime or pending[i].arrival <= now):
                if not realtime:
                    pending[i].arrival = now
                self.submit(pending[i])
                i += 1
            self._admit()
            if self.running:
                self.step_block()
                self._retire()
                self._finish()
            elif self._retiring:
                self._finish(wait=True)
            elif i < len(pending):
                time.sleep(min(max_idle_wait, max(0.0, pending[i].arrival - self.now())))
        torch.cuda.synchronize(self.core.device)
        return self.replies

    @staticmethod
    def latency_stats(replies):
        """p50/p99/mean of the latency (arrival to result), and p50/p99 of its
        two parts: the admission wait and the service time."""
        if not replies:
            return {"p50_s": None, "p99_s": None, "n": 0}
        out = {"n": len(replies)}
        for key, prefix in (("latency", ""), ("wait", "wait_"), ("service", "service_")):
            x = np.array([getattr(r, key) for r in replies], dtype=np.float64)
            out[prefix + "p50_s"] = float(np.percentile(x, 50))
            out[prefix + "p99_s"] = float(np.percentile(x, 99))
            if not prefix:
                out["mean_s"] = float(x.mean())
        return out


def poisson_requests(n, seed, rate_hz, count, trials=(1, 64), steps=(1000, 50000),
                     bin_steps=100):
    """Open-loop request stream: Poisson arrivals, per-trial mixes as in fis.batch."""
    from .batch import random_specs

    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for j in range(count):
        t += float(rng.exponential(1.0 / rate_hz))
        k = int(rng.integers(trials[0], trials[1] + 1))
        dur = int(rng.integers(steps[0], steps[1] + 1))
        specs = random_specs(n, k, int(rng.integers(0, 2 ** 31)), dur)
        reqs.append(Request(trials=specs, bin_steps=bin_steps, arrival=t))
    return reqs
