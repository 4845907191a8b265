"""Initial conditions of the five workloads (synthetic, seeded) in the reference's array layout.

Each builder returns ``(settings, state)``: ``settings`` are ImogenRun / oracle keyword arguments
(Initializer-style: grid, dgrid, gamma, cfl, bc, ...) and ``state`` = (mass, mom[3], ener, mag[3])
arrays shaped (nx, ny, nz).  B is face-centred: B_i(i) sits on face i-1/2 (MagnetArray.m:36-38).
Cell centres are x = (i + 1/2) dx.  The reference's own initializers differ in details (gamma,
BCs, coordinates), so these are the build's definitions of the workloads, fed identically to the
oracle and to the GPU path.
"""
from __future__ import annotations

import numpy as np


def _centres(n):
    return (np.arange(n) + 0.5) / n


def sod(n=1024, gamma=5 / 3, time_max=0.2):
    """1-D Sod tube on [0,1]: rho,P = 1,1 | 0.125,0.1, v = 0, transparent BCs."""
    x = _centres(n)
    grid = (n, 1, 1)
    rho = np.where(x < 0.5, 1.0, 0.125).reshape(grid)
    P = np.where(x < 0.5, 1.0, 0.1).reshape(grid)
    mom = np.zeros((3,) + grid)
    mag = np.zeros((3,) + grid)
    ener = P / (gamma - 1)
    settings = dict(grid=grid, dgrid=(1.0 / n, 1.0, 1.0), gamma=gamma, cfl=0.7, bc="trans",
                    limiter="vanleer", magnet=False, time_max=time_max, iter_max=10 ** 7)
    return settings, (rho, mom, ener, mag)


def orszag_tang(n=512, gamma=5 / 3, time_max=0.5, cfl=0.35):
    """2-D Orszag-Tang vortex on [0,1]^2, periodic."""
    x = _centres(n)[:, None]
    y = _centres(n)[None, :]
    grid = (n, n, 1)
    rho0 = 25.0 / (36.0 * np.pi)
    P0 = 5.0 / (12.0 * np.pi)
    B0 = 1.0 / np.sqrt(4.0 * np.pi)
    rho = np.full((n, n), rho0)
    mom = np.zeros((3, n, n))
    mom[0] = -rho * np.sin(2 * np.pi * y)
    mom[1] = rho * np.sin(2 * np.pi * x)
    mag = np.zeros((3, n, n))
    mag[0] = -B0 * np.sin(2 * np.pi * y) * np.ones((n, 1))   # Bx(y): divergence-free on faces
    mag[1] = B0 * np.sin(4 * np.pi * x) * np.ones((1, n))    # By(x)
    ener = P0 / (gamma - 1) + 0.5 * (mom ** 2).sum(0) / rho + 0.5 * (mag ** 2).sum(0)
    r = lambda a: a.reshape(grid)
    settings = dict(grid=grid, dgrid=(1.0 / n, 1.0 / n, 1.0), gamma=gamma, cfl=cfl, bc="circ",
                    limiter="vanleer", magnet=True, time_max=time_max, iter_max=10 ** 7)
    return settings, (r(rho), mom.reshape((3,) + grid), r(ener), mag.reshape((3,) + grid))


def kelvin_helmholtz(n=256, gamma=5 / 3, seed=0, iter_max=200):
    """3-D MHD Kelvin-Helmholtz on [0,1)^3, periodic: rho=2, vx=+0.5 for |y|<0.25 else rho=1,
    vx=-0.5; P=2.5; Bx=0.1; vy = 0.01*U(-1,1) inside the layer (PCG64(seed))."""
    grid = (n, n, n)
    y = _centres(n) - 0.5
    inside = (np.abs(y) < 0.25)[None, :, None] * np.ones(grid, dtype=bool)
    rho = np.where(inside, 2.0, 1.0)
    vx = np.where(inside, 0.5, -0.5)
    rng = np.random.Generator(np.random.PCG64(seed))
    vy = np.where(inside, 0.01 * rng.uniform(-1.0, 1.0, size=grid), 0.0)
    mom = np.stack([rho * vx, rho * vy, np.zeros(grid)])
    mag = np.stack([np.full(grid, 0.1), np.zeros(grid), np.zeros(grid)])
    ener = 2.5 / (gamma - 1) + 0.5 * (mom ** 2).sum(0) / rho + 0.5 * (mag ** 2).sum(0)
    settings = dict(grid=grid, dgrid=(1.0 / n,) * 3, gamma=gamma, cfl=0.35, bc="circ",
                    limiter="vanleer", magnet=True, time_max=1e5, iter_max=iter_max)
    return settings, (rho, mom, ener, mag)


def brio_wu_tube(n, rho_l, rho_r, p_l, p_r, gamma=2.0, time_max=0.1, width=3, xbc="const"):
    """One Brio-Wu-type MHD tube on an n x width x width grid: Bx = 0.75, By = +1 | -1.
    x: const BCs by default (the waves stay clear of the ends for the ensemble's steps; the reference's
    magnetic shock tube uses fade, experiment/MagneticShockTube/MagneticShockTubeInitializer.m:52, which
    xbc="fade" selects); y, z: periodic (uniform), so the Y/Z sweeps carry the v_y B_x induction."""
    grid = (n, width, width)
    x = _centres(n)[:, None, None] * np.ones(grid)
    left = x < 0.5
    rho = np.where(left, rho_l, rho_r)
    P = np.where(left, p_l, p_r)
    mom = np.zeros((3,) + grid)
    mag = np.stack([np.full(grid, 0.75), np.where(left, 1.0, -1.0), np.zeros(grid)])
    ener = P / (gamma - 1) + 0.5 * (mag ** 2).sum(0)
    bc = {"x": xbc, "y": "circ", "z": "circ"}
    settings = dict(grid=grid, dgrid=(1.0 / n, 1.0 / n, 1.0 / n), gamma=gamma, cfl=0.35, bc=bc,
                    limiter="vanleer", magnet=True, time_max=time_max, iter_max=10 ** 7)
    return settings, (rho, mom, ener, mag)


def brio_wu_ensemble(count=512, seed=0, nmin=256, nmax=8192, width=3, xbc="const"):
    """The batched ensemble: sizes log-uniform in [nmin, nmax], states U[0.1, 1] per side."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ns = np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=count)).astype(int)
    out = []
    for k in range(count):
        rl, rr, pl, pr = rng.uniform(0.1, 1.0, size=4)
        out.append(brio_wu_tube(int(ns[k]), rl, rr, pl, pr, width=width, xbc=xbc))
    return out


def sedov(n, dims=2, gamma=5 / 3, time_max=0.05, bc="fade"):
    """Sedov-Taylor blast: rho=1, P=1e-5, unit energy added to cell floor(n/2) of each dim."""
    grid = (n, n, n) if dims == 3 else (n, n, 1)
    dx = 1.0 / n
    rho = np.ones(grid)
    ener = np.full(grid, 1e-5 / (gamma - 1))
    c = n // 2
    vol = dx ** dims
    idx = (c, c, c) if dims == 3 else (c, c, 0)
    ener[idx] += 1.0 / vol
    mom = np.zeros((3,) + grid)
    mag = np.zeros((3,) + grid)
    settings = dict(grid=grid, dgrid=(dx, dx, dx if dims == 3 else 1.0), gamma=gamma, cfl=0.7,
                    bc=bc, limiter="vanleer", magnet=False, time_max=time_max, iter_max=10 ** 7)
    return settings, (rho, mom, ener, mag)


def oracle_kwargs(settings):
    """Translate run settings into oracle.Sim keyword arguments."""
    s = dict(settings)
    bc = s.pop("bc")
    if isinstance(bc, dict) and any(k in bc for k in "xyz"):
        lo = [bc[f] if isinstance(bc[f], str) else bc[f][0] for f in "xyz"]
        hi = [bc[f] if isinstance(bc[f], str) else bc[f][-1] for f in "xyz"]
        bc = {k: [lo, hi] for k in ("mass", "mom", "ener", "mag")}
    lim = s.pop("limiter", "vanleer")
    lim = (lim,) * 3 if isinstance(lim, str) else tuple(lim)
    lim = tuple("minmond" if l == "minmod" else l for l in lim)
    return dict(grid=s["grid"], dgrid=s["dgrid"], gamma=s.get("gamma", 5 / 3), cfl=s["cfl"],
                minmass=s.get("minmass", 1e-5), bc=bc, bc_infinity=s.get("bc_infinity", 20),
                limiter=lim, fluid_active=s.get("fluid", True), magnet_active=s.get("magnet", False),
                time_max=s.get("time_max", 1e5), iter_max=s.get("iter_max", 10),
                update_mode=s.get("update_mode", 1), viscosity=s.get("viscosity", "empty"),
                visc_linear=s.get("visc_linear", 0.0), visc_quadratic=s.get("visc_quadratic", 0.0),
                radiation=s.get("radiation", "empty"), rad_exponent=s.get("rad_exponent", 0.5),
                rad_initial_maximum=s.get("rad_initial_maximum", 0.0), treadmill=s.get("treadmill", 0),
                fade_location=s.get("fade_location"), fade_size=s.get("fade_size", 0.0),
                fade_active=s.get("fade_active", ()))


WORKLOADS = {
    "ot512": lambda: orszag_tang(512),
    "ot64": lambda: orszag_tang(64),
    "kh256": lambda: kelvin_helmholtz(256),
    "kh128": lambda: kelvin_helmholtz(128),
    "kh160": lambda: kelvin_helmholtz(160),
    "sod": lambda: sod(4096),
}


def main(argv=None):
    """Run a workload for a few iterations on the current CUDA device (e.g. under a profiler):
    python -m imogen_b200.problems ot512 --precision mixed --iters 3"""
    import argparse
    import time

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("workload", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--autotune", action="store_true", help="tune the pencil tilings first (as bench.py does)")
    ap.add_argument("--tiling", action="append", default=[],
                    help="dim=Wb,G,CL,NT,cpt for the fluid sweeps along one direction, e.g. x=2,128,1,256,4, or "
                         "mx=... for the magnet sweeps (repeatable)")
    a = ap.parse_args(argv)
    from imogen_b200 import ImogenRun

    s, st = WORKLOADS[a.workload]()
    run = ImogenRun(precision=a.precision, **dict(s, iter_max=10 ** 7, time_max=1e5))
    run.set_state(*st)
    for spec in a.tiling:
        dim, vals = spec.split("=")
        kind = "magnet" if dim.startswith("m") else "fluid"
        run.set_tiling("xyz".index(dim[-1]) + 1, [int(v) for v in vals.split(",")], kind=kind)
    if a.autotune:
        run.iterate()
        print("tiling", run.autotune(trials=3))
    t0 = time.perf_counter()
    for _ in range(a.iters):
        run.iterate()
    run.sync()
    el = time.perf_counter() - t0
    tot = run.totals()
    run.close()
    print(f"{a.workload} {a.precision}: {a.iters} iterations in {el * 1e3:.2f} ms, mass {tot[0]:.12e}")


if __name__ == "__main__":
    main()
