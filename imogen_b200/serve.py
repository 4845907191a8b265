"""Serving loop: simulation jobs admitted by HBM budget, batched while they run.

Jobs arrive over time (``Job.arrival``, seconds after the loop starts).  The loop admits the
oldest arrived jobs while their device memory (``img_bytes_required``) fits the budget, runs each
new job's first iteration on its own (it captures the job's stored edges) and then moves it into
the running batch of its kind (same precision, physics and swept dimensions), where every step
advances all members with one launch per kernel.  Batches of different kinds run on their own
streams and overlap on the device.  A job completes when its run stops (TIMEMAX or ITERMAX); its
result is read back, its memory returns to the budget, and its latency (completion - arrival) is
recorded.  Each member's arithmetic is the same as alone, so a job's result does not depend on
what else was in the mix.

No reference counterpart: the reference runs one simulation per MATLAB session.
"""
from __future__ import annotations

import dataclasses
import time
from typing import Callable, Dict, List, Optional

import numpy as np

from . import problems
from ._lib import ImogenError
from .run import ImogenBatch, ImogenRun, bytes_required  # noqa: F401  (bytes_required is re-exported)


@dataclasses.dataclass
class Job:
    """One simulation request: run settings, initial state, arrival time (s)."""
    id: int
    settings: dict
    state: tuple
    arrival: float = 0.0
    precision: str = "mixed"
    # filled by the server
    admitted: Optional[float] = None
    completed: Optional[float] = None
    iterations: int = 0
    result: Optional[dict] = None

    @property
    def cells(self) -> int:
        return int(np.prod(self.settings["grid"]))

    @property
    def latency(self) -> Optional[float]:
        return None if self.completed is None else self.completed - self.arrival


def _kind(run: ImogenRun):
    c = run.config
    return (c.precision, c.fluid_active, c.magnet_active, c.update_mode, tuple(int(n) >= 3 for n in c.grid))


class Server:
    """Continuous-batching server over one GPU.

    hbm_budget: device bytes the jobs' state may use together.  check_every: batch steps between
    polls of the members' stop flags (a poll synchronises the batch's stream).  keep: what to read
    back from a finished job -- "state" (all arrays), "totals" (conserved totals) or a callable
    taking the ImogenRun."""

    def __init__(self, hbm_budget: int, check_every: int = 4, keep="state",
                 clock: Callable[[], float] = time.perf_counter):
        self.budget = int(hbm_budget)
        self.check_every = max(1, int(check_every))
        self.keep = keep
        self.clock = clock
        self.used = 0
        self.queue: List[Job] = []
        self.done: List[Job] = []
        self.batches: Dict[tuple, ImogenBatch] = {}
        self.running: Dict[int, tuple] = {}     # job id -> (job, run, bytes)
        self.t0 = None
        self._n = 0

    def now(self) -> float:
        return self.clock() - self.t0

    def submit(self, job: Job):
        self.queue.append(job)
        self.queue.sort(key=lambda j: j.arrival)

    def _need(self, job: Job) -> int:
        return bytes_required(**dict(job.settings, precision=job.precision))

    def _admit(self):
        t = self.now()
        while self.queue and self.queue[0].arrival <= t:
            job = self.queue[0]
            need = self._need(job)
            if need > self.budget:
                raise ValueError(f"job {job.id} needs {need} bytes, more than the whole budget {self.budget}")
            if self.used + need > self.budget:
                break                                    # first come, first served: wait for memory
            self.queue.pop(0)
            run = ImogenRun(precision=job.precision, **job.settings)
            run.set_state(*job.state)
            run.iterate()                                # first iteration alone (captures stored edges)
            job.admitted = t
            key = _kind(run)
            b = self.batches.get(key)
            if b is None:
                b = self.batches[key] = ImogenBatch()
            b.add(run)                                   # waits for the run's own stream
            run.batch_ref = b
            self.running[job.id] = (job, run, need)
            self.used += need

    def _retire(self, batch: ImogenBatch):
        flags = batch.status()                           # synchronises the batch's stream
        finished = [(m, f) for m, f in zip(list(batch.members), flags) if f & 3]
        for run, flag in finished:
            jid = next(k for k, v in self.running.items() if v[1] is run)
            job, _, need = self.running.pop(jid)
            batch.remove(run)
            if flag & 2:                                 # the job's device error flag (CFL, non-finite)
                try:
                    run.progress()
                    job.result = {"error": "device error flag set", "code": None}
                except ImogenError as e:
                    job.result = {"error": str(e), "code": e.code}
            else:
                if callable(self.keep):
                    job.result = self.keep(run)
                elif self.keep == "totals":
                    job.result = {"totals": run.totals()}
                else:
                    job.result = run.state()
                job.result["time"], job.iterations, _ = run.progress()
            job.completed = self.now()
            run.close()
            self.used -= need
            self.done.append(job)

    def start(self):
        """Start the clock (arrival times are measured from here)."""
        self.t0 = self.clock()
        self._n = 0

    def tick(self, idle_sleep: float = 2e-4) -> bool:
        """One scheduling round: admit what fits, advance every running batch one iteration, and
        every check_every rounds retire the finished jobs.  Returns False once nothing is queued or
        running.  Jobs may be submitted, polled and cancelled between rounds."""
        if self.t0 is None:
            self.start()
        if not (self.queue or self.running):
            return False
        self._admit()
        active = [b for b in self.batches.values() if b.members]
        if not active:
            if self.queue:
                time.sleep(min(idle_sleep, max(0.0, self.queue[0].arrival - self.now())))
            return True
        for b in active:
            b.step()
        self._n += 1
        if self._n % self.check_every == 0:
            for b in active:
                self._retire(b)
        return True

    def poll(self, job_id: int) -> dict:
        """State of a job: queued, running (with simulated time and iterations), done or cancelled."""
        for j in self.queue:
            if j.id == job_id:
                return {"state": "queued"}
        if job_id in self.running:
            job, run, _ = self.running[job_id]
            t, n, _ = run.progress()
            return {"state": "running", "time": t, "iterations": n}
        for j in self.done:
            if j.id == job_id:
                r = j.result or {}
                st = "cancelled" if r.get("cancelled") else ("failed" if "error" in r else "done")
                return {"state": st, "latency_s": j.latency, **({"error": r["error"]} if "error" in r else {})}
        raise KeyError(job_id)

    def cancel(self, job_id: int) -> bool:
        """Drop a queued job, or stop a running one and free its memory.  False if it already ended."""
        for i, j in enumerate(self.queue):
            if j.id == job_id:
                self.queue.pop(i)
                j.result = {"cancelled": True}
                self.done.append(j)
                return True
        if job_id in self.running:
            job, run, need = self.running.pop(job_id)
            run.batch_ref.remove(run)
            run.close()
            self.used -= need
            job.result = {"cancelled": True}
            self.done.append(job)
            return True
        return False

    def close(self):
        for b in self.batches.values():
            b.close()
        self.batches = {}

    def serve(self, jobs: List[Job]) -> List[Job]:
        """Run until every job has completed; returns them in completion order."""
        for j in jobs:
            self.submit(j)
        self.start()
        while self.tick():
            pass
        self.close()
        return self.done


def latency_summary(jobs: List[Job]) -> dict:
    lat = np.array([j.latency for j in jobs if j.latency is not None])
    zu = sum(j.cells * 2 * j.iterations for j in jobs)
    return {"jobs": len(lat), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "zone_updates": int(zu)}


def sedov_stream(count: int, rate: float = 50.0, seed: int = 0, sizes2=(64, 512), sizes3=(32, 192),
                 precision: str = "mixed", time_max: float = 0.05) -> List[Job]:
    """Poisson arrivals (mean `rate` jobs/s) of Sedov-Taylor blasts: half 2-D grids n^2 with n
    log-uniform in sizes2, half 3-D grids n^3 with n log-uniform in sizes3 (seeded)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    jobs = []
    for k in range(count):
        t += rng.exponential(1.0 / rate)
        dims = 2 if rng.uniform() < 0.5 else 3
        lo, hi = sizes2 if dims == 2 else sizes3
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        s, st = problems.sedov(n, dims=dims, time_max=time_max)
        jobs.append(Job(id=k, settings=s, state=st, arrival=t, precision=precision))
    return jobs


def one_at_a_time(jobs: List[Job], precision: str = "fp64", keep="totals",
                  clock: Callable[[], float] = time.perf_counter) -> List[Job]:
    """The baseline: the same jobs in arrival order, one on the GPU at a time, each run alone."""
    out = []
    t0 = clock()
    for j in sorted(jobs, key=lambda j: j.arrival):
        while clock() - t0 < j.arrival:
            time.sleep(1e-4)
        job = dataclasses.replace(j, precision=precision, admitted=clock() - t0, result=None)
        run = ImogenRun(precision=precision, **j.settings)
        run.set_state(*j.state)
        run.run()
        job.result = {"totals": run.totals()} if keep == "totals" else run.state()
        job.result["time"], job.iterations, _ = run.progress()
        run.close()
        job.completed = clock() - t0
        out.append(job)
    return out
