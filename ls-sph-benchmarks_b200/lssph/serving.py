"""Request loop: continuous batching of independent solves on one GPU.

Requests (a parameter set and a number of time steps) arrive over time.  The server keeps
every admitted solve resident on the device and advances all of them together through
one :class:`~lssph.batch.Batch` (one graph launch per step for all members).  Between
batch calls it
  * admits waiting requests, in arrival order, whose device footprint (computed exactly
    by lssph_estimate_device_bytes) fits the remaining HBM budget and a free slot;
    a request that does not fit does not block smaller ones behind it (first fit);
  * gives each new member a step budget equal to its remaining steps, so it stops on the
    device exactly where a solo run of that many steps stops, whatever the chunk size;
  * retires members that finished (budget used up, steady state or error): downloads the
    final state, frees the device memory and records the time to solution.
Each result is bit-identical to running the same request alone (the batched kernels run
the solo arithmetic per member); the serving test checks this.

Pre-emption: a request with a higher ``priority`` that has arrived but finds no slot or
memory suspends active members of lower priority (newest first) until it fits.  A
suspended member's state is downloaded (the checkpoint), its device memory freed, and it
waits again; when re-admitted it resumes from that state with its remaining step budget.
A solve restarted from its state continues bit for bit, so a pre-empted request still ends
with exactly its solo result.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from . import _abi
from ._abi import Params, check
from .batch import Batch
from .simulation import Simulation, State, estimate_device_bytes, setup_counts


def device_memory() -> tuple[int, int]:
    """(free, total) bytes of the current device."""
    lib = _abi.load()
    f, t = C.c_int64(), C.c_int64()
    check(lib.lssph_mem_info(C.byref(f), C.byref(t)))
    return f.value, t.value


@dataclass
class Request:
    rid: int
    params: Params
    nsteps: int
    arrival: float = 0.0                 # seconds on the server clock
    tag: str = ""
    init: Callable[[], State] | None = None   # builds the initial state (default: fresh start)
    priority: int = 0                    # higher pre-empts lower when slots or memory run out
    # filled in by the server
    footprint: int = 0
    admitted: float | None = None
    finished: float | None = None
    steps_done: int = 0
    status: int = 0
    stopped: str = ""                    # "budget" | "steady" | "error"
    result: State | None = None
    preemptions: int = 0
    resume: State | None = None          # checkpoint of a suspended request

    @property
    def latency(self) -> float | None:
        return None if self.finished is None else self.finished - self.arrival


@dataclass
class ServerStats:
    completed: int
    makespan_s: float
    solves_per_s: float
    p50_s: float
    p99_s: float
    particle_updates_per_s: float
    device_ms: float
    max_active: int
    batch_calls: int
    host_create_s: float = 0.0
    wait_s: float = 0.0
    host_retire_s: float = 0.0
    host_launch_s: float = 0.0
    host_join_s: float = 0.0
    max_queue: int = 0               # most requests waiting for admission at one scheduling point
    mean_queue: float = 0.0          # waiting requests averaged over scheduling points
    preemptions: int = 0             # active solves suspended for higher-priority requests
    latencies_s: list = field(default_factory=list)


class Server:
    """Continuous-batching request loop (single thread, one device)."""

    def __init__(self, hbm_budget: int | None = None, max_active: int = 64, chunk_steps: int = 50,
                 keep_results: bool = True, clock=time.perf_counter, preempt: bool = True):
        if hbm_budget is None:
            free, _ = device_memory()
            hbm_budget = int(0.8 * free)
        self.hbm_budget = int(hbm_budget)
        self.max_active = int(max_active)
        self.chunk_steps = int(chunk_steps)
        self.keep_results = keep_results
        self.preempt = preempt
        self.preemptions = 0
        self.clock = clock
        self.batch = Batch()
        self.waiting: deque[Request] = deque()
        self.active: list[tuple[Request, Simulation]] = []
        self.done: list[Request] = []
        self.used = 0
        self.peak_used = 0
        self.t0 = clock()
        self.device_ms = 0.0
        self.host_create_s = 0.0     # setting up admitted solves (overlaps batch calls)
        self.wait_s = 0.0            # waiting for batch calls after the set-up work
        self.host_retire_s = 0.0     # bookkeeping after each call, downloading results, freeing solves
        self.host_launch_s = 0.0     # starting batch calls (a changed membership re-captures the graph)
        self.host_join_s = 0.0       # adding set-up solves to the batch (first of a configuration: measured)
        self.batch_calls = 0
        self.queue_samples: list[int] = []
        self.peak_active = 0
        self.particle_steps = 0

    # ---- request intake ---------------------------------------------------------------
    def now(self) -> float:
        return self.clock() - self.t0

    def submit(self, req: Request) -> None:
        if req.footprint == 0:
            req.footprint = estimate_device_bytes(req.params)
        if req.footprint > self.hbm_budget:
            raise ValueError(f"request {req.rid} needs {req.footprint} bytes, over the HBM budget")
        self.waiting.append(req)

    def _pick(self) -> list[Request]:
        """Waiting requests that have arrived and fit (first fit, arrival order); their
        footprint and slot are reserved here."""
        now = self.now()
        picked: list[Request] = []
        keep: deque[Request] = deque()
        slots = self.max_active - len(self.active)
        while self.waiting:
            req = self.waiting.popleft()
            if req.arrival <= now and len(picked) < slots and self.used + req.footprint <= self.hbm_budget:
                self.used += req.footprint
                self.peak_used = max(self.peak_used, self.used)
                req.admitted = self.now()
                picked.append(req)
            else:
                keep.append(req)
        self.waiting = keep
        if self.preempt:
            picked += self._preempt_for(now, len(picked))
        return picked

    def _preempt_for(self, now: float, n_picked: int) -> list[Request]:
        """Admit arrived waiting requests that outrank active members by suspending those
        members (lowest priority first, newest first among equals)."""
        picked: list[Request] = []
        for req in sorted((r for r in self.waiting if r.arrival <= now), key=lambda r: -r.priority):
            victims = sorted((i for i, (a, _) in enumerate(self.active) if a.priority < req.priority),
                             key=lambda i: (self.active[i][0].priority, -(self.active[i][0].admitted or 0.0)))
            free_slots = self.max_active - len(self.active) - n_picked - len(picked)
            free_mem = self.hbm_budget - self.used
            chosen = []
            for i in victims:
                if free_slots >= 1 and free_mem >= req.footprint:
                    break
                chosen.append(i)
                free_slots += 1
                free_mem += self.active[i][0].footprint
            if free_slots < 1 or free_mem < req.footprint:
                continue
            for i in sorted(chosen, reverse=True):
                self.suspend(i)
            self.waiting = deque(r for r in self.waiting if r is not req)
            self.used += req.footprint
            self.peak_used = max(self.peak_used, self.used)
            req.admitted = self.now()
            picked.append(req)
        return picked

    def suspend(self, i: int) -> Request:
        """Checkpoint active member i to host memory, free its device memory and put it back
        at the head of the queue; it resumes from the checkpoint when re-admitted."""
        req, sim = self.active.pop(i)
        req.resume = sim.download()
        self.batch.remove(sim)
        sim.close()
        self.used -= req.footprint
        req.preemptions += 1
        self.preemptions += 1
        self.waiting.appendleft(req)
        return req

    def _create(self, req: Request) -> Simulation:
        ni = setup_counts(req.params)[1]
        if req.resume is not None:               # restart from the checkpoint, no extra ghost pass
            sim = Simulation(req.params, req.resume, ni)
            req.resume = None
        elif req.init is None:
            sim = Simulation.new(req.params)
        else:
            sim = Simulation(req.params, req.init(), ni)
            sim.ghost()
        sim.set_step_budget(req.nsteps - req.steps_done)
        return sim

    # ---- one batch call ---------------------------------------------------------------
    def step_once(self) -> int:
        """One batch call of up to chunk_steps steps.  Requests admitted now are set up on
        the host and copied to the device while the GPU steps the current members; they
        join the batch for the next call.  Returns the number of members retired."""
        picked = self._pick()
        launched = bool(self.active)
        t0 = self.clock()
        if launched:
            self.batch.launch(self.chunk_steps)
        tl = self.clock()
        self.host_launch_s += tl - t0
        created = [(req, self._create(req)) for req in picked]     # overlaps the batch call
        t1 = self.clock()
        self.host_create_s += t1 - tl
        retired = []
        if launched:
            status, steady, steps = self.batch.wait(raise_on_error=False)
            t2 = self.clock()
            self.wait_s += t2 - t1
            ms, _ = self.batch.last_step_stats()
            self.device_ms += ms
            self.batch_calls += 1
            for i, (req, sim) in enumerate(self.active):
                req.steps_done += int(steps[i])
                self.particle_steps += int(steps[i]) * sim.num_int
                if status[i] != _abi.OK:
                    req.status, req.stopped = int(status[i]), "error"
                elif steady[i] > 0:
                    req.stopped = "steady"
                elif req.steps_done >= req.nsteps:
                    req.stopped = "budget"
                if req.stopped:
                    retired.append(i)
            for i in reversed(retired):
                req, sim = self.active.pop(i)
                if self.keep_results and req.status == _abi.OK:
                    req.result = sim.download()
                self.batch.remove(sim)
                sim.close()
                self.used -= req.footprint
                req.finished = self.now()
                self.done.append(req)
            self.host_retire_s += self.clock() - t2
        tj = self.clock()
        for req, sim in created:
            self.batch.add(sim)
            self.active.append((req, sim))
        self.host_join_s += self.clock() - tj
        self.peak_active = max(self.peak_active, len(self.active))
        return len(retired)

    def run(self, requests: list[Request], realtime: bool = True) -> ServerStats:
        """Serve `requests` (arrival times relative to the start of this call).  With
        realtime=False every request is available at once."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        self.t0 = self.clock()
        total = len(pending)
        while len(self.done) < total:
            now = self.now()
            while pending and (not realtime or pending[0].arrival <= now):
                r = pending.popleft()
                if not realtime:
                    r.arrival = 0.0
                self.submit(r)
            if not self.active and pending and not any(r.arrival <= self.now() for r in self.waiting):
                time.sleep(max(0.0, min(pending[0].arrival - self.now(), 0.05)))
                continue
            self.queue_samples.append(len(self.waiting))
            self.step_once()
        return self.stats()

    def stats(self) -> ServerStats:
        lat = sorted(r.latency for r in self.done if r.latency is not None)
        span = max((r.finished for r in self.done), default=0.0) - min((r.arrival for r in self.done), default=0.0)
        q = lambda f: float(np.quantile(lat, f)) if lat else math.nan   # noqa: E731
        return ServerStats(completed=len(self.done), makespan_s=span,
                           solves_per_s=len(self.done) / span if span > 0 else math.nan,
                           p50_s=q(0.5), p99_s=q(0.99),
                           particle_updates_per_s=self.particle_steps / span if span > 0 else math.nan,
                           device_ms=self.device_ms, max_active=self.peak_active, batch_calls=self.batch_calls,
                           host_create_s=self.host_create_s, wait_s=self.wait_s, host_retire_s=self.host_retire_s,
                           host_launch_s=self.host_launch_s, host_join_s=self.host_join_s,
                           max_queue=max(self.queue_samples, default=0),
                           mean_queue=float(np.mean(self.queue_samples)) if self.queue_samples else 0.0,
                           preemptions=self.preemptions,
                           latencies_s=lat)

    def close(self) -> None:
        for _, sim in self.active:
            sim.close()
        self.active = []
        self.batch.close()
