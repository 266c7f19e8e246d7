"""Continuous-batching request loop for simulation requests.

Requests arrive over time (``Job.arrival``, seconds from the start).  The
loop admits them in arrival order while a slot is free and their device
footprint fits an HBM budget, keeps every admitted grid resident on the GPU,
and advances all live grids together in rounds of at most ``chunk`` steps
(one CUDA graph per step holding every live grid's launches on parallel
branches).  A request leaves as
soon as its own steps are done: its result is copied back, its memory is
freed and the next waiting request takes the slot.  Requests that arrive
while a round runs are set up on the host and device during the round and
join the next one.

The loop is written against a small engine interface so its scheduling can
be tested on the CPU with a fake engine:

* ``footprint(job) -> int`` device bytes of the job's state
* ``create(job) -> handle`` allocate, initialise (on the GPU) and prepare
* ``launch(handles, steps)`` / ``wait()`` advance live grids by per-grid steps
* ``finish(job, handle) -> result`` copy the result back and free the grid

Time-to-solution of a request is its completion time minus its arrival time
(host wall clock, both on the loop's clock).
"""
from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import FIRST_COMPLETED, Future, ThreadPoolExecutor, wait
from dataclasses import dataclass, field

import numpy as np


class AdmissionError(RuntimeError):
    pass


@dataclass
class Outcome:
    rid: int
    arrival: float
    admitted: float = 0.0
    done: float = 0.0
    cells: int = 0
    steps: int = 0
    result: object = None

    @property
    def time_to_solution(self) -> float:
        return self.done - self.arrival


@dataclass
class ServeReport:
    outcomes: list = field(default_factory=list)
    makespan: float = 0.0
    rounds: int = 0
    peak_live: int = 0
    peak_bytes: int = 0
    # host seconds by activity (launch includes building a batch that was
    # not prebuilt; wait is the host blocked on the round)
    seconds: dict = field(default_factory=lambda: dict(launch=0.0, retire=0.0, admit=0.0,
                                                       prebuild=0.0, wait=0.0, idle=0.0))

    def cell_updates(self) -> int:
        return sum(o.cells * o.steps for o in self.outcomes)

    def latency(self, q) -> float:
        return float(np.percentile([o.time_to_solution for o in self.outcomes], q))

    def summary(self) -> dict:
        return dict(requests=len(self.outcomes), makespan_s=self.makespan, rounds=self.rounds,
                    peak_live=self.peak_live, peak_bytes=self.peak_bytes,
                    host_seconds={k: round(v, 3) for k, v in self.seconds.items()},
                    mcell_updates_per_s=self.cell_updates() / self.makespan / 1e6,
                    p50_s=self.latency(50), p99_s=self.latency(99))


class Server:
    """Admission by slots and HBM budget, resident state, batched rounds."""

    def __init__(self, engine, hbm_budget: int, max_live: int = 32, chunk: int = 50,
                 clock=time.perf_counter, sleep=time.sleep, workers: int = 0):
        """``workers`` > 0 runs request set-up (``create``) and result
        copy-back (``finish``) on that many host threads, so neither holds
        up the loop that feeds the GPU; 0 runs them inline."""
        if chunk <= 0 or max_live <= 0:
            raise ValueError("chunk and max_live must be positive")
        self.engine, self.budget, self.max_live, self.chunk = engine, int(hbm_budget), max_live, chunk
        self.clock, self.sleep, self.workers = clock, sleep, int(workers)

    def run(self, jobs) -> ServeReport:
        eng = self.engine
        pending = deque(sorted(jobs, key=lambda j: (j.arrival, j.rid)))
        for j in pending:
            if eng.footprint(j) > self.budget:
                raise AdmissionError(f"request {j.rid} needs {eng.footprint(j)} bytes, "
                                     f"more than the budget of {self.budget}")
        pool = ThreadPoolExecutor(self.workers) if self.workers > 0 else None
        rep = ServeReport()
        sec = rep.seconds
        starting = []  # [job, future of handle, outcome]: being set up
        ready = []     # [job, handle, remaining, outcome]: join the next round
        live = []      # in the next / current round
        leaving = []   # [job, future of result, outcome]: result being copied back
        used = 0
        t0 = self.clock()

        def now():
            return self.clock() - t0

        def timed(key, fn, *a):
            t = self.clock()
            r = fn(*a)
            sec[key] += self.clock() - t
            return r

        def run_async(fn, *a):
            if pool is not None:
                return pool.submit(fn, *a)
            f = Future()
            f.set_result(fn(*a))
            return f

        def admit():
            nonlocal used
            while (pending and pending[0].arrival <= now()
                   and len(live) + len(ready) + len(starting) < self.max_live):
                j = pending[0]
                fp = eng.footprint(j)
                if used + fp > self.budget:
                    break  # first come, first served: the head waits for memory
                pending.popleft()
                out = Outcome(j.rid, j.arrival, admitted=now(), cells=j.cells, steps=j.steps)
                used += fp
                starting.append([j, run_async(eng.create, j), out])
                rep.peak_live = max(rep.peak_live, len(live) + len(ready) + len(starting))
                rep.peak_bytes = max(rep.peak_bytes, used)

        def collect(block=False):
            """Moves set-up and copy-back work that has finished along."""
            nonlocal used
            if block and not any(e[1].done() for e in starting + leaving):
                wait([e[1] for e in starting + leaving], return_when=FIRST_COMPLETED)
            for e in [e for e in starting if e[1].done()]:
                starting.remove(e)
                ready.append([e[0], e[1].result(), e[0].steps, e[2]])
            for e in [e for e in leaving if e[1].done()]:
                leaving.remove(e)
                j, f, out = e
                out.result = f.result()
                out.done = now()
                used -= eng.footprint(j)
                rep.outcomes.append(out)

        try:
            while pending or live or ready or starting or leaving:
                timed("admit", collect)
                timed("admit", admit)
                live += ready
                ready.clear()
                if not live:
                    if starting or leaving:
                        timed("idle", collect, True)
                    elif pending and pending[0].arrival > now():
                        # idle until the next arrival
                        timed("idle", self.sleep, pending[0].arrival - now())
                    continue
                steps = [min(self.chunk, e[2]) for e in live]
                timed("launch", eng.launch, [e[1] for e in live], steps)
                rep.rounds += 1
                # while the round runs: new arrivals are set up, the next
                # round's batch is prepared
                timed("admit", collect)
                timed("admit", admit)
                nxt = [e[1] for e, s in zip(live, steps) if e[2] > s] + [e[1] for e in ready]
                if nxt:
                    timed("prebuild", eng.prebuild, nxt)
                timed("wait", eng.wait)
                for e, s in zip(live, steps):
                    e[2] -= s
                for e in live:
                    if e[2] == 0:
                        leaving.append([e[0], run_async(eng.finish, e[0], e[1]), e[3]])
                live = [e for e in live if e[2] > 0]
        finally:
            if pool is not None:
                pool.shutdown(wait=True)
        rep.makespan = now()
        rep.outcomes.sort(key=lambda o: o.rid)
        return rep


def serial(jobs, run_one, clock=time.perf_counter) -> ServeReport:
    """One request at a time, in arrival order: each request's service time
    (set-up, steps, result copy) is measured and its time-to-solution follows
    from a first-come-first-served queue on the arrival times."""
    rep = ServeReport()
    free_at = 0.0
    for j in sorted(jobs, key=lambda j: (j.arrival, j.rid)):
        t = clock()
        res = run_one(j)
        service = clock() - t
        start = max(free_at, j.arrival)
        free_at = start + service
        rep.outcomes.append(Outcome(j.rid, j.arrival, admitted=start, done=free_at, cells=j.cells,
                                    steps=j.steps, result=res))
        rep.rounds += 1
    rep.makespan = free_at
    rep.peak_live = 1
    rep.outcomes.sort(key=lambda o: o.rid)
    return rep


class GpuEngine:
    """The engine of the GPU library: one gop.Instance per request, a
    gop.Batch over the live set (built for the next round while the current
    one runs)."""

    def __init__(self, keep=lambda job: False, precision=None, device_init=True):
        from . import Batch
        from . import workloads
        self._Batch, self._wl = Batch, workloads
        self.keep, self.precision = keep, precision
        self.device_init = device_init  # initial state built on the GPU
        self._batch, self._members = None, ()
        self._next, self._next_members = None, ()
        self._fp = {}
        self.stats = dict(builds=0, build_s=0.0, prebuilt_used=0, launch_s=0.0)

    def footprint(self, job):
        key = (job.n, job.precision if self.precision is None else self.precision)
        if key not in self._fp:
            self._fp[key] = self._wl.footprint(job, self.precision)
        return self._fp[key]

    def _buffers(self, name):
        # host buffers per worker thread (set-up and copy-back may run on
        # several threads at once)
        return self.__dict__.setdefault(f"{name}_{threading.get_ident()}", {})

    def create(self, job):
        if self.device_init:
            return self._wl.build(job, self.precision, device_init=True)
        return self._wl.build(job, self.precision, host=self._buffers("init"))

    def _build(self, members):
        t = time.perf_counter()
        b = self._Batch(members)
        self.stats["builds"] += 1
        self.stats["build_s"] += time.perf_counter() - t
        return b

    def prebuild(self, handles):
        members = tuple(handles)
        if members not in (self._members, self._next_members):
            if self._next is not None:
                self._next.close()
            self._next, self._next_members = self._build(members), members

    def launch(self, handles, steps):
        members = tuple(handles)
        if members != self._members:
            if self._batch is not None:
                self._batch.close()
            if members == self._next_members:
                self._batch, self._members = self._next, members
                self._next, self._next_members = None, ()
                self.stats["prebuilt_used"] += 1
            else:
                self._batch, self._members = self._build(members), members
        t = time.perf_counter()
        self._batch.launch(steps)
        self.stats["launch_s"] += time.perf_counter() - t

    def wait(self):
        self._batch.wait()

    def finish(self, job, inst):
        res = download_result(inst, self._buffers("host"), copy=self.keep(job))
        inst.close()
        return res

    def close(self):
        for b in (self._batch, self._next):
            if b is not None:
                b.close()
        self._batch = self._next = None
        self._members = self._next_members = ()


def download_result(inst, pool, copy=False):
    """Copies a grid's state (6 primitives, 3 face fields) to host buffers
    reused across requests of the same shape; returns the stats and, when
    ``copy``, private copies of the arrays."""
    key = inst.N
    if key not in pool:
        pool[key] = {"gas": np.zeros(inst.shape(6)), "face_b": np.zeros(inst.shape(3))}
    out = inst.download(("gas", "face_b"), out=pool[key])
    res = inst.stats()
    if copy:
        res["gas"] = out["gas"].copy()
        res["face_b"] = out["face_b"].copy()
    return res


# ------------------------------------------------------------ several GPUs
# The path does not shard: with several ranks (one process per GPU) every
# rank serves its own share of the stream on its own GPU and nothing crosses
# between GPUs on the data path.  Only the reports are combined.

def shard(jobs, rank: int, world: int):
    """The jobs rank `rank` of `world` serves: request ids rank, rank+world, ..."""
    return [j for j in jobs if j.rid % world == rank]


def combine(report: ServeReport, dist=None, group=None) -> dict:
    """Whole-job summary over ranks: cell-updates summed, makespan the
    maximum over ranks, latency percentiles over every rank's requests.
    ``dist`` is torch.distributed (or None for one rank)."""
    tts = [o.time_to_solution for o in report.outcomes]
    cu = float(report.cell_updates())
    span = float(report.makespan)
    if dist is not None and dist.get_world_size(group) > 1:
        import torch
        world = dist.get_world_size(group)
        t = torch.tensor([cu], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        cu = float(t.item())
        t = torch.tensor([span], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        span = float(t.item())
        gathered = [None] * world
        dist.all_gather_object(gathered, tts, group=group)
        tts = [v for part in gathered for v in part]
    return dict(requests=len(tts), makespan_s=span, cell_updates=cu,
                mcell_updates_per_s=cu / span / 1e6 if span > 0 else 0.0,
                p50_s=float(np.percentile(tts, 50)) if tts else 0.0,
                p99_s=float(np.percentile(tts, 99)) if tts else 0.0)
