#!/usr/bin/env python
"""Benchmark of the B200 relaxing-TVD MHD path (one JSON line on stdout, rank 0).

Workload (default): Orszag-Tang vortex, 2-D ideal MHD, 512 x 512 periodic, gamma 5/3, synthetic
IC (imogen_b200.problems.orszag_tang).  One bench step = one iteration of the reference main loop
(imogen.m:60-66) = two timesteps, each sweeping X and Y (fluid + magnet), with the CFL timestep
computed on the device.  Metric: zone-updates/s = cells x timesteps / s.  The state (16.8 MB FP64)
fits in the 126 MB L2, so L2 is flushed (a 512 MB write) before every timed step and each step is
timed alone with CUDA events on the library's stream.

Headline `value` is the mixed-precision form (FP32 state and fluxes, FP64 pressure recovery and
CFL); the plain FP64 form is measured in the same run (`fp64`), with the relative L1 error of the
mixed state against the FP64 state after the same iterations (`l1_mixed_vs_fp64`).

--impl reference times the C++ FP64 restatement of the reference (oracle/) on all host threads
(the MATLAB reference itself cannot run here).  With torchrun (N > 1) every rank advances its own
replica (the path does not shard: replicas only) and the max time over ranks is used.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAK_FALLBACK_GBS = 6650.0


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        # NVML when available: a sample every 2 ms, so that even a timed region of a few
        # milliseconds is covered; otherwise nvidia-smi every 200 ms
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
            bits = (0x8, 0x40, 0x20, 0x4)   # hw slowdown, hw thermal, sw thermal, sw power cap
            while not self._stop.is_set():
                sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                r = get_reasons(h)
                self.samples.append([str(sm), str(mx), ""] + ["Active" if r & b else "Not Active" for b in bits])
                self._stop.wait(0.002)
            return
        except Exception:
            pass
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def profiled_traffic(key):
    """DRAM bytes (read + write) per launch of a kernel, from the committed ncu summary."""
    import re
    try:
        with open(os.path.join(ROOT, "profiles", "pencil_kernels_orszag_tang_512_mixed.md")) as f:
            m = re.search(r"traffic_bytes %s = (\d+)" % re.escape(key), f.read())
        return int(m.group(1)) if m else None
    except OSError:
        return None


def max_over_ranks(x, device):
    """The largest of x over the ranks of the default process group (x itself with one rank): the job's
    time is the slowest rank's."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload(name):
    from imogen_b200 import problems
    if name == "ot512":
        s, st = problems.orszag_tang(512)
        return s, st, "orszag_tang_512x512_mhd", 2, 16   # dims swept, MHD words/dir
    if name == "kh256":
        s, st = problems.kelvin_helmholtz(256)
        return s, st, "kelvin_helmholtz_256^3_mhd", 3, 16
    if name == "ot64":
        s, st = problems.orszag_tang(64)
        return s, st, "orszag_tang_64x64_mhd", 2, 16
    raise SystemExit(f"unknown workload {name}")


# ---------------------------------------------------------------------------------------------------
def run_reference(args):
    """C++ FP64 restatement of the reference path, all host threads, bounded sample."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import cpp_oracle
    from imogen_b200 import problems
    s, st, wname, _, _ = workload(args.workload)
    ncell = int(np.prod(s["grid"]))
    cores = os.cpu_count() or 1
    cpp_oracle.set_threads(cores)
    o = cpp_oracle.Sim(**problems.oracle_kwargs(dict(s, iter_max=10 ** 7, time_max=1e5)))
    o.set_state(*st)
    for _ in range(args.warmup):
        o.iterate()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.iterate()
    el = time.perf_counter() - t0
    v = ncell * 2 * args.steps / el
    line = {
        "impl": "reference", "metric": "MHD zone-updates/s", "value": v, "unit": "zone-updates/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Orszag-Tang IC)",
        "config": {"workload": wname, "cells": ncell, "step": "1 iteration = 2 timesteps",
                   "l2": "host run"},
        "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": cpp_oracle.max_threads(),
                         "kind": "port", "sample": f"{args.steps} iterations of {wname} after {args.warmup} warm-up"},
        "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(s, st, wname, budget_s=20.0):
    """The C++ oracle on all host threads, timed on a bounded number of iterations."""
    from oracle import cpp_oracle
    from imogen_b200 import problems
    cores = os.cpu_count() or 1
    cpp_oracle.set_threads(cores)
    ncell = int(np.prod(s["grid"]))
    o = cpp_oracle.Sim(**problems.oracle_kwargs(dict(s, iter_max=10 ** 7, time_max=1e5)))
    o.set_state(*st)
    o.iterate()   # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        o.iterate()
        n += 1
        el = time.perf_counter() - t0
        if el > budget_s or n >= 200:
            break
    return {"value": ncell * 2 * n / el, "unit": "zone-updates/s", "cores": cpp_oracle.max_threads(),
            "kind": "port", "sample": f"{n} iterations of {wname} (C++ FP64 oracle, OpenMP)"}


def run_ours(args):
    import torch
    import imogen_b200
    from imogen_b200 import ImogenRun
    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    s, st, wname, ndir, words = workload(args.workload)
    ncell = int(np.prod(s["grid"]))
    s = dict(s, iter_max=10 ** 7, time_max=1e5)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # 512 MB > 126 MB L2

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed_steps(run, k, per_launch=None):
        """k iterations, each after an L2 flush, each timed alone on the run's stream."""
        ext = torch.cuda.ExternalStream(run.stream)
        tot = 0.0
        evs = []
        for _ in range(k):
            with torch.cuda.stream(ext):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(ext)
            (per_launch or run.iterate)()
            with torch.cuda.stream(ext):
                e1.record(ext)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        for e0, e1 in evs:
            tot += e0.elapsed_time(e1) * 1e-3
        return tot

    results = {}
    runs = {}
    tilings = {}
    for prec in ("fp64", "mixed"):
        r = ImogenRun(precision=prec, **s)
        r.set_state(*st)
        r.iterate()
        if args.autotune:
            tilings[prec] = {kind: {"xyz"[d - 1]: t for d, t in tl.items() if s["grid"][d - 1] >= 3}
                             for kind, tl in r.autotune(trials=3).items()}
        for _ in range(args.warmup):
            r.iterate()
        r.sync()
        runs[prec] = r
    clocks = ClockSampler(local)
    launches = {}
    with clocks:
        for prec in ("fp64", "mixed"):
            r = runs[prec]
            barrier()
            l0 = r.launches
            el = timed_steps(r, args.steps)
            launches[prec] = r.launches - l0
            results[prec] = max_over_ranks(el, dev)
    clk = clocks.summary()

    # relative L1 of mixed vs FP64 after the same iterations
    sf, sm = runs["fp64"].state(), runs["mixed"].state()
    l1 = {}
    for k in ("mass", "ener"):
        l1[k] = float(np.abs(sm[k] - sf[k]).sum() / np.abs(sf[k]).sum())
    for k in ("mom", "mag"):
        for c in range(3):
            den = np.abs(sf[k][c]).sum()
            if den > 0:
                l1[f"{k}{'xyz'[c]}"] = float(np.abs(sm[k][c] - sf[k][c]).sum() / den)

    # per-kernel roofline: the fused fluid sweep of each swept direction timed alone, L2 flushed before
    # each launch; the slower direction (the dominant fluid kernel of the step) is the line's roofline
    peak, peak_kind = measured_hbm_peak()
    traffic = profiled_traffic("fluid_sweep_x_mixed") if args.workload == "ot512" else None
    roof, sweeps = {}, {}
    dims = [d for d in (1, 2, 3) if s["grid"][d - 1] >= 3]
    for prec in ("mixed", "fp64"):
        r = runs[prec]
        w = 4 if prec == "mixed" else 8
        alg = ncell * (8 + 5) * w     # reads rho,p,E,cellB (8 words), writes rho,p,E (5 words)
        sweeps[prec] = {}
        for X in dims:
            r.time.set(r.time.time, 1e-4, r.time.iteration)
            el = timed_steps(r, max(5, args.steps), per_launch=lambda r=r, X=X: r.relaxing_fluid(X))
            per = el / max(5, args.steps)
            sweeps[prec]["xyz"[X - 1]] = {"launch_us": per * 1e6, "achieved": alg / per / 1e9,
                                          "frac": alg / per / 1e9 / peak}
        dom = max(sweeps[prec], key=lambda k: sweeps[prec][k]["launch_us"])
        per = sweeps[prec][dom]["launch_us"] * 1e-6
        tr = traffic if (prec == "mixed" and dom == "x") else None
        roof[prec] = {"bound": "hbm", "achieved": alg / per / 1e9, "peak": peak, "unit": "GB/s",
                      "frac": alg / per / 1e9 / peak, "traffic": tr,
                      "traffic_source": "static figure from the ncu capture committed in "
                                        "profiles/pencil_kernels_orszag_tang_512_mixed.md (not measured in this run)"
                      if tr else None, "kernel": f"fluid sweep along {dom} (the slower swept direction)",
                      "launch_us": per * 1e6, "alg_bytes": alg, "peak_kind": peak_kind}

    # end to end through the C ABI: the step's state comes from pinned host memory (X.array = ...
    # for the 8 conserved arrays), one iteration runs, and the 8 arrays are read back to pinned host
    # memory (get.array), every step.
    e2e = None
    r = runs["mixed"]
    names = ("mass", "momx", "momy", "momz", "ener", "magx", "magy", "magz")
    src = [st[0], st[1][0], st[1][1], st[1][2], st[2], st[3][0], st[3][1], st[3][2]]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F"))
                                     ).pin_memory().numpy()
    ins = [pin(a) for a in src]
    outs = [pin(np.zeros(ncell)) for _ in range(8)]
    ke = max(3, args.steps // 2)
    up = dict(zip(names, ins))
    down = dict(zip(names, outs))
    for _ in range(args.warmup):   # untimed: first transfers set up the transfer stream and host buffers
        r.upload_many(up)
        r.iterate()
        r.download_many(down)
    r.sync()
    barrier()
    t0 = time.perf_counter()
    for _ in range(ke):
        r.upload_many(up)
        r.iterate()
        r.download_many(down)
    r.sync()
    el = time.perf_counter() - t0
    e2e = {"value": ncell * 2 * ke / el, "unit": "zone-updates/s",
           "h2d_bytes_per_step": 8 * ncell * 8, "d2h_bytes_per_step": 8 * ncell * 8,
           "pcie_bytes_per_step_each_way": 8 * ncell * 4,   # FP32: the library converts on the host
           "form": "mixed", "steps": ke}

    kh = run_kh(args, timed_steps, measured_hbm_peak()[0]) if args.kh > 0 else None
    accuracy = run_accuracy(args) if args.accuracy and rank == 0 else None
    serving = run_serving(args) if args.serve_jobs > 0 and not args.serve_small else None
    serving_small = run_serving(args, small=True) if args.serve_jobs > 0 else None
    ensemble = run_ensemble(args, timed_steps) if args.ensemble > 0 else None

    if rank == 0:
        v = ncell * 2 * args.steps * ws / results["mixed"]
        v64 = ncell * 2 * args.steps * ws / results["fp64"]
        line = {
            "metric": "MHD zone-updates/s", "value": v, "unit": "zone-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * results["mixed"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded Orszag-Tang IC, no dataset)",
            "config": {"workload": wname, "cells": ncell, "form": "mixed (FP32 state/fluxes, FP64 pressure+CFL)",
                       "step": "1 iteration = 2 timesteps (X,Y fluid+magnet each)",
                       "l2": "flushed (512 MB write) before every timed step", "parallelism": f"replicas x{ws}",
                       "tiling": tilings or None,
                       "tiling_fields": "pencils/CTA, threads/pencil, CTAs/cluster, threads/CTA, cells/thread, components/CTA"},
            "fp64": {"value": v64, "unit": "zone-updates/s", "ms_per_step": 1e3 * results["fp64"] / args.steps},
            "mixed_over_fp64": v / v64,
            "l1_mixed_vs_fp64": l1,
            "l1_mixed_vs_fp64_max": max(l1.values()),
            "l1_mixed_vs_fp64_after": f"{args.warmup + 1 + args.steps} iterations (plus autotuner trials)",
            "accuracy_t_end": accuracy,
            "roofline": roof["mixed"],
            "roofline_fp64": roof["fp64"],
            "roofline_sweeps": sweeps,
            "gpu_launches": launches["mixed"],
            "clocks": clk,
            "e2e": e2e,
            "p50_p99_job_latency": None if (serving or serving_small) is None else
            {"p50_s": (serving or serving_small)["served_mixed"]["p50_s"],
             "p99_s": (serving or serving_small)["served_mixed"]["p99_s"],
             "unit": "s", "workload": (serving or serving_small)["workload"]},
            "serving": serving,
            "serving_unsaturated": serving_small,
            "ensemble": ensemble,
            "kh3d": kh,
        }
        if not args.no_cpu_baseline and ws == 1:
            line["cpu_baseline"] = cpu_baseline(s, st, wname, budget_s=args.cpu_budget)
        print(json.dumps(line), flush=True)
    for r in runs.values():
        r.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def div_b_rel(mag, dgrid):
    """max |div B| * dx / max |B| of the face-centred field (B_d(i) on face i-1/2), periodic grid."""
    div = np.zeros(mag.shape[1:])
    for d in range(3):
        if mag.shape[1 + d] > 1:
            div += (np.roll(mag[d], -1, axis=d) - mag[d]) / dgrid[d]
    bmax = float(np.abs(mag).max())
    return float(np.abs(div).max() * min(dgrid[d] for d in range(3) if mag.shape[1 + d] > 1) / bmax) if bmax else 0.0


def run_accuracy(args):
    """The mixed form's acceptance point: Orszag-Tang 512^2 run to t = 0.5 in both forms (outside any
    timed region); relative L1 of the mixed state against the FP64 state per variable (rho, E; momentum
    and B per component and as vectors), the discrete div B of both, and their compensated totals."""
    from imogen_b200 import ImogenRun, problems
    s, st = problems.orszag_tang(512, time_max=0.5)
    out = {"workload": "orszag_tang_512x512_mhd", "t_end": 0.5}
    states, tots = {}, {}
    for prec in ("fp64", "mixed"):
        r = ImogenRun(precision=prec, **s)
        r.set_state(*st)
        n = r.run()
        t, _, _ = r.progress()
        states[prec] = r.state()
        tots[prec] = [float(v) for v in r.totals()]
        out[f"iterations_{prec}"] = n
        out[f"time_{prec}"] = t
        r.close()
    a, b = states["mixed"], states["fp64"]
    rel = lambda x, y: float(np.abs(x - y).sum() / np.abs(y).sum())
    l1 = {"rho": rel(a["mass"], b["mass"]), "E": rel(a["ener"], b["ener"]),
          "momentum": rel(a["mom"], b["mom"]), "B": rel(a["mag"], b["mag"])}
    for c in range(2):
        l1[f"mom{'xyz'[c]}"] = rel(a["mom"][c], b["mom"][c])
        l1[f"B{'xyz'[c]}"] = rel(a["mag"][c], b["mag"][c])
    out["l1_at_t_end"] = l1
    out["l1_at_t_end_max"] = max(l1.values())
    out["divb"] = {"fp64": div_b_rel(b["mag"], s["dgrid"]), "mixed": div_b_rel(a["mag"], s["dgrid"]),
                   "measure": "max|div B| * dx / max|B|"}
    out["totals"] = {"order": "rho, px, py, pz, E, Bx, By, Bz", "fp64": tots["fp64"], "mixed": tots["mixed"],
                     "initial": [float(v) for v in (st[0].sum(), *st[1].reshape(3, -1).sum(1), st[2].sum(),
                                                    *st[3].reshape(3, -1).sum(1))]}
    return out


def run_kh(args, timed_steps, peak):
    """3-D MHD Kelvin-Helmholtz at n^3 (default 256^3, 16.8 M cells: the state exceeds L2, so this is
    the HBM-bound configuration): iteration throughput of both forms and the x fluid sweep against
    the measured HBM bandwidth."""
    from imogen_b200 import ImogenRun, problems
    n = args.kh
    s, st = problems.kelvin_helmholtz(n)
    s = dict(s, iter_max=10 ** 7, time_max=1e5)
    cells = n ** 3
    out = {"workload": f"kelvin_helmholtz_{n}^3_mhd", "cells": cells}
    for prec, w in (("mixed", 4), ("fp64", 8)):
        r = ImogenRun(precision=prec, **s)
        r.set_state(*st)
        r.iterate()
        tiling = r.autotune(trials=2) if args.autotune else {"fluid": r.tiling("fluid"), "magnet": r.tiling("magnet")}
        for _ in range(2):
            r.iterate()
        k = 5
        el = timed_steps(r, k)
        alg = cells * (8 + 5) * w
        fl = {}
        for X in (1, 2, 3):   # each direction's fluid sweep alone (the inputs are larger than L2)
            r.time.set(r.time.time, 1e-5, r.time.iteration)
            per = timed_steps(r, k, per_launch=lambda r=r, X=X: r.relaxing_fluid(X)) / k
            fl["xyz"[X - 1]] = {"launch_us": per * 1e6, "alg_bytes": alg, "achieved_gbs": alg / per / 1e9,
                                "frac_of_measured_hbm": alg / per / 1e9 / peak}
        out[prec] = {"zone_updates_per_s": cells * 2 * k / el, "ms_per_step": 1e3 * el / k,
                     "fluid_x": fl["x"], "fluid_sweeps": fl,
                     "tiling": {kind: {"xyz"[d - 1]: t for d, t in tl.items()} for kind, tl in tiling.items()}}
        r.close()
    return out


def run_serving(args, small=False):
    """Poisson stream of Sedov-Taylor jobs: the continuous-batching server (mixed form) against the
    same jobs one at a time in plain FP64.  Latency = completion - arrival, wall clock.

    small=False: the stated grids (2-D 64^2..512^2, 3-D 32^3..192^3).  Their work at 50 jobs/s is
    several times what one GPU finishes in the 4 s over which they arrive, so the latencies measure
    the queue as much as the server.  small=True: 2-D 32^2..256^2, 3-D 24^3..96^3, a stream the server
    keeps up with, whose latencies show the time a job spends being served."""
    from imogen_b200 import serve
    sizes = dict(sizes2=(32, 256), sizes3=(24, 96)) if small else dict(sizes2=(64, 512), sizes3=(32, 192))
    lo2, hi2 = sizes["sizes2"]
    lo3, hi3 = sizes["sizes3"]
    # untimed warm-up: the first jobs of the same stream run to the end once (the first launch of
    # every kernel variant and batch shape they meet loads its code; launch plans are set up); the
    # one-at-a-time baseline warms on its first 20 jobs
    warm_n = args.serve_jobs if small else min(args.serve_jobs, 40)
    # rounds between checks for finished jobs (a check synchronises every batch): the stated stream's
    # rounds carry many large jobs and take tens of milliseconds, so it checks less often; the
    # unsaturated stream's rounds are short and a finished job should leave within a few of them
    ce = 4 if small else 32
    warm = serve.sedov_stream(warm_n, rate=1e6, seed=0, precision="mixed", **sizes)
    serve.Server(hbm_budget=args.serve_budget_gb << 30, check_every=ce, keep="totals").serve(warm)
    serve.one_at_a_time(serve.sedov_stream(20, rate=1e6, seed=0, precision="fp64", **sizes), precision="fp64")
    jobs = serve.sedov_stream(args.serve_jobs, rate=50.0, seed=0, precision="mixed", **sizes)
    t0 = time.perf_counter()
    done = serve.Server(hbm_budget=args.serve_budget_gb << 30, check_every=ce, keep="totals").serve(jobs)
    el = time.perf_counter() - t0
    a = serve.latency_summary(done)
    a.update(wall_s=el, zone_updates_per_s=a["zone_updates"] / el)
    t0 = time.perf_counter()
    base = serve.one_at_a_time(serve.sedov_stream(args.serve_jobs, rate=50.0, seed=0, precision="fp64", **sizes),
                               precision="fp64")
    el = time.perf_counter() - t0
    b = serve.latency_summary(base)
    b.update(wall_s=el, zone_updates_per_s=b["zone_updates"] / el)
    arrivals = max(j.arrival for j in jobs)
    return {"workload": f"{args.serve_jobs} Sedov-Taylor jobs, Poisson arrivals 50/s (seed 0), 2-D {lo2}^2..{hi2}^2 / "
                        f"3-D {lo3}^3..{hi3}^3 log-uniform, t=0.05, HBM budget {args.serve_budget_gb} GB",
            "server": "native job server (img_server_create / img_batch_submit / img_batch_poll)",
            "arrival_span_s": arrivals,
            "offered_load": a["zone_updates"] / arrivals / a["zone_updates_per_s"], "check_every": ce,
            "served_mixed": a, "one_at_a_time_fp64": b}


def run_ensemble(args, timed_steps):
    """Brio-Wu ensemble (N x 3 x 3 MHD tubes, N log-uniform in [256, 8192], seeded, mixed form): all
    members advanced by batched launches, against the same members stepped one at a time."""
    import torch
    from imogen_b200 import ImogenBatch, ImogenRun, problems
    tubes = problems.brio_wu_ensemble(count=args.ensemble, seed=0)
    cells = sum(int(np.prod(s["grid"])) for s, _ in tubes)
    members = []
    for s, st in tubes:
        r = ImogenRun(precision="mixed", **dict(s, time_max=1e5))
        r.set_state(*st)
        members.append(r)
    k = 20
    # one at a time: each member advances k iterations on its own stream, in turn
    for r in members:
        r.iterate()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in members:
        for _ in range(k):
            r.iterate()
    for r in members:
        r.sync()
    seq = time.perf_counter() - t0
    b = ImogenBatch(members)
    for _ in range(14):                        # into the graph-replay regime: the six sweep-order phases
        b.step()                               # are captured at steps 7-12, then replayed
    l0 = b.launches
    el = timed_steps(b, k, per_launch=b.step)
    out = {"members": len(members), "cells": cells, "form": "mixed", "steps": k,
           "batched_zone_updates_per_s": cells * 2 * k / el, "batched_ms_per_step": 1e3 * el / k,
           "batched_launches_per_step": (b.launches - l0) / k,
           "one_at_a_time_zone_updates_per_s": cells * 2 * k / seq}
    b.close()
    for r in members:
        r.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ot512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--serve-jobs", type=int, default=200, help="jobs of the serving leg (0: skip)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false", help="keep the default tilings")
    ap.add_argument("--kh", type=int, default=256, help="edge of the 3-D Kelvin-Helmholtz leg (0: skip)")
    ap.add_argument("--serve-budget-gb", type=int, default=64)
    ap.add_argument("--serve-small", action="store_true",
                    help="only the unsaturated serving leg (2-D 32^2..256^2 / 3-D 24^3..96^3 grids), not the stated "
                         "64^2..512^2 / 32^3..192^3 one")
    ap.add_argument("--ensemble", type=int, default=512, help="members of the batched-ensemble leg (0: skip)")
    ap.add_argument("--no-accuracy", dest="accuracy", action="store_false",
                    help="skip the Orszag-Tang run to t = 0.5 (mixed vs FP64 L1, div B, totals)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
