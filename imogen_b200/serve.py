"""Serving: simulation jobs admitted by HBM budget and batched while they run, on the native job
server of the C ABI (img_server_create / img_batch_submit / img_batch_poll / img_batch_cancel, see
imogen_b200/csrc/server.cpp).

Jobs arrive over time (``Job.arrival``, seconds after the server starts); ``Server`` hands each to the
native server when it arrives.  The server's worker thread admits the oldest jobs while their device
memory (``img_bytes_required``) fits the budget, adds each to the running batch of its kind (same
precision, physics and swept dimensions) -- a new member takes its first, edge-capturing iteration
inside the batch -- and advances every batch one iteration per round.  A job completes when its run
stops (TIMEMAX or ITERMAX); its result is read back, its memory returns to the budget, and its latency
(completion - arrival) is recorded.  Each member's arithmetic is the same as alone, so a job's result
does not depend on what else was in the mix.

No reference counterpart: the reference runs one simulation per MATLAB session.
"""
from __future__ import annotations

import ctypes
import dataclasses
import time
from typing import Callable, Dict, List, Optional

import numpy as np

from . import problems
from ._lib import ImgJobInfo, ImgServerInfo, ImogenError, lib
from .run import VAR, ImogenRun, bytes_required, make_config  # noqa: F401  (bytes_required is re-exported)

STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


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


class Server:
    """Continuous-batching server over one GPU (a native img_server).

    hbm_budget: device bytes the jobs' state may use together.  check_every: rounds between checks of
    the members' stop flags (a check synchronises).  keep: what a finished job keeps -- "state" (all
    arrays) or "totals" (conserved totals).  Arrival times are measured from start() on the server's
    monotonic clock."""

    def __init__(self, hbm_budget: int, check_every: int = 4, keep="state", clock: Callable[[], float] = None):
        if keep not in ("state", "totals"):
            raise ValueError("keep must be 'state' or 'totals'")
        self.budget = int(hbm_budget)
        self.keep = keep
        self.clock = clock or lib().img_monotonic_seconds
        h = ctypes.c_void_p()
        rc = lib().img_server_create(ctypes.byref(h), self.budget, max(1, int(check_every)), 0 if keep == "state" else 1)
        if rc != 0:
            raise ImogenError(rc, "img_server_create failed")
        self._h = h
        self.pending: List[Job] = []            # not yet arrived
        self.jobs: Dict[int, Job] = {}          # job id -> Job
        self.native: Dict[int, int] = {}        # job id -> native job id
        self.collected: Dict[int, bool] = {}
        self.done: List[Job] = []
        self.t0 = None
        self._final: Dict[int, ImgJobInfo] = {}   # job records kept when the native server is closed
        self._final_stats = None

    def now(self) -> float:
        return self.clock() - self.t0

    def start(self):
        """Start the clock (arrival times are measured from here)."""
        self.t0 = self.clock()

    def submit(self, job: Job):
        self.jobs[job.id] = job
        self.pending.append(job)
        self.pending.sort(key=lambda j: j.arrival)

    def _hand_over(self):
        t = self.now()
        while self.pending and self.pending[0].arrival <= t:
            job = self.pending.pop(0)
            cfg = make_config(precision=job.precision, **job.settings)
            shp = tuple(int(g) for g in cfg.grid)
            f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shp).ravel(order="F"))
            mass, ener = f(job.state[0]), f(job.state[2])
            mom = np.concatenate([f(job.state[1][c]) for c in range(3)])
            mag = np.concatenate([f(job.state[3][c]) for c in range(3)])
            dp = ctypes.POINTER(ctypes.c_double)
            jid = ctypes.c_int()
            rc = lib().img_batch_submit(self._h, ctypes.byref(cfg), mass.ctypes.data_as(dp), mom.ctypes.data_as(dp),
                                        ener.ctypes.data_as(dp), mag.ctypes.data_as(dp), ctypes.byref(jid))
            if rc != 0:
                raise ImogenError(rc, f"job {job.id} could not be submitted (needs more than the budget?)")
            self.native[job.id] = jid.value

    def _info(self, job_id) -> ImgJobInfo:
        if self._h is None:
            return self._final[job_id]
        info = ImgJobInfo()
        rc = lib().img_batch_poll(self._h, self.native[job_id], ctypes.byref(info))
        if rc != 0:
            raise ImogenError(rc, "img_batch_poll failed")
        return info

    def _collect(self, job: Job, info: ImgJobInfo):
        if self.collected.get(job.id):
            return
        self.collected[job.id] = True
        st = STATES[info.status]
        job.completed = info.completed - self.t0
        job.admitted = None if info.admitted == 0 else info.admitted - self.t0
        job.iterations = info.iterations
        if st == "done":
            nid = self.native[job.id]
            if self.keep == "totals":
                out = np.zeros(8)
                lib().img_batch_result(self._h, nid, -1, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 8)
                job.result = {"totals": out}
            else:
                shp = tuple(int(g) for g in job.settings["grid"]) + (1,) * (3 - len(job.settings["grid"]))
                n = int(np.prod(shp))

                def get(name):
                    a = np.zeros(n)
                    lib().img_batch_result(self._h, nid, VAR[name], a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n)
                    return a.reshape(shp, order="F")
                job.result = dict(mass=get("mass"), ener=get("ener"),
                                  mom=np.stack([get("momx"), get("momy"), get("momz")]),
                                  mag=np.stack([get("magx"), get("magy"), get("magz")]),
                                  cellmag=np.stack([get("cmagx"), get("cmagy"), get("cmagz")]))
            job.result["time"] = info.time
        elif st == "cancelled":
            job.result = {"cancelled": True}
        else:
            job.result = {"error": info.error.decode(), "code": info.error_code}
        self.done.append(job)

    def tick(self, idle_sleep: float = 2e-4) -> bool:
        """Hand the arrived jobs to the native server and collect the finished ones.  Returns False
        once every submitted job has finished.  Jobs may be submitted, polled and cancelled between
        calls."""
        if self.t0 is None:
            self.start()
        self._hand_over()
        busy = bool(self.pending)
        for jid in list(self.native):
            if self.collected.get(jid):
                continue
            info = self._info(jid)
            if info.status >= 2:
                self._collect(self.jobs[jid], info)
            else:
                busy = True
        if busy:
            time.sleep(idle_sleep)
        return busy

    @property
    def running(self) -> List[int]:
        return [j for j in self.native if self._info(j).status == 1]

    def stats(self) -> dict:
        if self._h is None:
            return dict(self._final_stats)
        info = ImgServerInfo()
        lib().img_server_stats(self._h, ctypes.byref(info))
        return {k: getattr(info, k) for k, _ in ImgServerInfo._fields_}

    @property
    def used(self) -> int:
        return int(self.stats()["used"])

    def poll(self, job_id: int) -> dict:
        """State of a job: queued, running, done, failed or cancelled."""
        if job_id not in self.native:
            if job_id in self.jobs:
                return {"state": "queued"}                     # not yet arrived
            raise KeyError(job_id)
        info = self._info(job_id)
        st = STATES[info.status]
        out = {"state": st}
        if st in ("done", "failed", "cancelled"):
            out["latency_s"] = info.completed - self.t0 - self.jobs[job_id].arrival
        if st == "failed":
            out["error"] = info.error.decode()
        return out

    def cancel(self, job_id: int) -> bool:
        """Drop a queued job, or stop a running one and free its memory (waits until the worker has
        stopped it).  False if it already ended."""
        if job_id not in self.native:
            job = self.jobs.get(job_id)
            if job is None or job not in self.pending:
                return False
            self.pending.remove(job)
            job.result = {"cancelled": True}
            self.done.append(job)
            return True
        if lib().img_batch_cancel(self._h, self.native[job_id]) != 0:
            return False
        while self._info(job_id).status < 2:
            time.sleep(1e-4)
        return self._info(job_id).status == 4

    def close(self):
        if self._h:
            self._final = {j: self._info(j) for j in self.native}
            self._final_stats = self.stats()
            lib().img_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def serve(self, jobs: List[Job]) -> List[Job]:
        """Run until every job has completed; returns them in completion order."""
        for j in jobs:
            self.submit(j)
        self.start()
        while self.tick():
            pass
        out = sorted(self.done, key=lambda j: j.completed)
        self.close()
        return out


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
