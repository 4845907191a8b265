"""Host-side mirror of the reference's call surface for the relaxing-TVD path.

``ImogenRun`` stands in for the ImogenManager plus the FluidArray/MagnetArray objects of one run
(classes/ImogenManager.m, imogen.m:34-45); its state is resident on the GPU.  The functions
``flux``, ``relaxingFluid`` and ``magnetFlux`` keep the reference signatures (flux/flux.m:1,
fluid/relaxingFluid.m:1, magnet/magnetFlux.m:1) so a driver written against the reference reads
the same; the array arguments are accepted for signature compatibility and ignored, because the
arrays live in the run.  ``run.time`` mirrors TimeManager (time/TimeManager.m).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import ImgConfig, ImgSliceMeta, ImgSliceState, ImogenError, check, lib

BC_MODES = ("circ", "const", "fade", "mirror", "trans", "wall", "flip", "zero", "linear", "wormhole")   # enums/ENUM.m:22-32
LIMITERS = {"vanleer": 0, "superbee": 1, "minmond": 2, "minmod": 2}   # FluxLimiterEnum.m:10-13
BC_CLASSES = ("mass", "mom", "ener", "mag")
PRECISIONS = {"fp64": 0, "mixed": 1}
# ENUM.ARTIFICIAL_VISCOSITY_* and ENUM.RADIATION_* (enums/ENUM.m)
VISCOSITIES = {"empty": 0, "none": 0, "neumann_richtmyer": 1, "caramana_shashkov_whalen": 2}
RADIATIONS = {"empty": 0, "none": 0, "optically_thin": 1}
FADE_IDS = {"mass": 1, "mom": 2, "ener": 4, "mag": 8, "grav": 16}   # ENUM.MASS .. ENUM.GRAV of a fade's activeList
VAR = dict(mass=0, momx=1, momy=2, momz=3, ener=4, magx=5, magy=6, magz=7, cmagx=8, cmagy=9, cmagz=10)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def bc_table(bc):
    """bcMode as initialize.m:24-40 accepts it: one mode string for everything, a struct-like
    dict {x, y, z} (each a mode or a (lower, upper) pair), or per-class {mass|mom|ener|mag: ...}.
    Returns int[4][2][3]."""
    def one(spec):
        out = [[0, 0, 0], [0, 0, 0]]
        if isinstance(spec, str):
            spec = {"x": spec, "y": spec, "z": spec}
        for d, f in enumerate("xyz"):
            v = spec.get(f, "circ")
            lo, hi = (v, v) if isinstance(v, str) else (v[0], v[-1])
            out[0][d] = BC_MODES.index(lo)
            out[1][d] = BC_MODES.index(hi)
        return out
    if bc is None:
        bc = "circ"
    if isinstance(bc, str) or any(k in bc for k in "xyz"):
        t = one(bc)
        return [t, t, t, t]
    if isinstance(bc, dict) and all(k in bc for k in BC_CLASSES):
        res = []
        for k in BC_CLASSES:
            v = bc[k]
            if isinstance(v, (list, tuple)) and len(v) == 2 and not isinstance(v[0], str):
                res.append([[BC_MODES.index(m) for m in v[0]], [BC_MODES.index(m) for m in v[1]]])
            else:
                res.append(one(v))
        return res
    raise ValueError(f"unrecognised bcMode {bc!r}")


def make_config(grid, dgrid=None, gamma=5 / 3, cfl=None, minmass=1e-5, bc="circ", bc_infinity=20,
                limiter="vanleer", fluid=True, magnet=False, time_max=1e5, iter_max=10,
                update_mode=1, precision="fp64", nonfinite_check=True, viscosity="empty", visc_linear=0.0,
                visc_quadratic=0.0, radiation="empty", rad_exponent=0.5, rad_initial_maximum=0.0, treadmill=0,
                fade_location=None, fade_size=0.0, fade_active=()):
    """img_config from Initializer-style settings (experiment/Initializer.m:73-184 defaults; run.viscosity
    and run.radiation as fluid/ArtificialViscosity.m:31-37 and fluid/Radiation.m:32-37 hold them)."""
    c = ImgConfig()
    lib().img_config_default(ctypes.byref(c))
    grid = tuple(int(g) for g in grid) + (1,) * (3 - len(grid))
    if dgrid is None:
        dgrid = (1.0, 1.0, 1.0)
    if np.isscalar(dgrid):
        dgrid = (float(dgrid),) * 3
    for d in range(3):
        c.grid[d] = grid[d]
        c.dgrid[d] = float(dgrid[d])
    c.gamma = float(gamma)
    c.cfl = float(cfl if cfl is not None else (0.35 if magnet else 0.7))   # Initializer.m:143-150
    c.minmass = float(minmass)
    c.bc_infinity = int(bc_infinity)
    t = bc_table(bc)
    for k in range(4):
        for s in range(2):
            for d in range(3):
                c.bc_modes[k][s][d] = t[k][s][d]
    lims = (limiter,) * 3 if isinstance(limiter, str) else tuple(limiter)
    for d in range(3):
        c.limiter[d] = LIMITERS[lims[d]]
    c.fluid_active = int(bool(fluid))
    c.magnet_active = int(bool(magnet))
    c.time_max = float(time_max)
    c.iter_max = int(iter_max)
    c.update_mode = int(update_mode)
    c.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    c.nonfinite_check = int(bool(nonfinite_check))
    c.viscosity_type = VISCOSITIES[viscosity] if isinstance(viscosity, str) else int(viscosity)
    c.visc_linear = float(visc_linear)
    c.visc_quadratic = float(visc_quadratic)
    c.radiation_type = RADIATIONS[radiation] if isinstance(radiation, str) else int(radiation)
    c.rad_exponent = float(rad_exponent)
    c.rad_initial_maximum = float(rad_initial_maximum)
    c.treadmill = int(treadmill)
    if fade_location is not None:   # one point fade (ini.fades): the arrays it acts on, location, radius
        c.fade_active = sum(FADE_IDS[name] for name in fade_active)
        for d in range(3):
            c.fade_location[d] = int(fade_location[d])
        c.fade_size = float(fade_size)
    return c


SLICE_TYPES = {"X": 1, "Y": 2, "Z": 3, "XY": 4, "XZ": 5, "YZ": 6, "XYZ": 7, "SP-XYZ": 8}   # SaveManager.SLICELABELS


def slice_meta(slice="XYZ", index=(1, 1, 1), suffix="FINAL", about="", version=0.0, wall_max=1e5, started=None):
    """img_slice_meta for one resultsHandler slice save (save/resultsHandler.m:26-113)."""
    m = ImgSliceMeta()
    m.type = SLICE_TYPES[slice] if isinstance(slice, str) else int(slice)
    for d in range(3):
        m.index[d] = int(index[d])
    m.suffix = suffix.encode()
    m.about = about.encode()
    m.version = float(version)
    m.wall_max = float(wall_max)
    m.started = started.encode() if started is not None else None
    return m


def write_slice(path, state, grid, dgrid=(1.0, 1.0, 1.0), gamma=5 / 3, time=0.0, iteration=0, iter_max=10,
                time_max=1e5, dt_history=(), magnet=True, treadmill=0, treadmill_history=(), **meta):
    """img_slice_write of host arrays (mass, mom[3], ener, mag[3]; x fastest): no device involved."""
    grid = tuple(int(g) for g in grid)
    f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F"))
    mass, ener = f(state[0]), f(state[2])
    mom = np.concatenate([f(state[1][c]) for c in range(3)])
    mag = np.concatenate([f(state[3][c]) for c in range(3)])
    hist = np.ascontiguousarray(np.asarray(dt_history, dtype=np.float64))
    th = np.ascontiguousarray(np.asarray(treadmill_history, dtype=np.int32))
    st = ImgSliceState()
    for d in range(3):
        st.grid[d] = grid[d]
        st.dgrid[d] = float(dgrid[d])
    st.gamma, st.time, st.iteration, st.iter_max, st.time_max = gamma, time, iteration, iter_max, time_max
    dp = ctypes.POINTER(ctypes.c_double)
    st.dt_history = hist.ctypes.data_as(dp) if hist.size else None
    st.n_history = int(hist.size)
    st.magnet_active = int(bool(magnet))
    st.mass, st.mom, st.ener, st.mag = (a.ctypes.data_as(dp) for a in (mass, mom, ener, mag))
    st.treadmill = int(treadmill)
    st.tread_history = th.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if th.size else None
    st.n_tread = int(th.size)
    m = slice_meta(**meta)
    rc = lib().img_slice_write(str(path).encode(), ctypes.byref(m), ctypes.byref(st))
    if rc != 0:
        raise ImogenError(rc, lib().img_slice_last_error().decode())


def read_slice(path):
    """img_slice_read: (mass, mom[3], ener, mag[3]) as grid-shaped arrays, and whether B was stored."""
    g = (ctypes.c_int * 3)()
    rc = lib().img_slice_read(str(path).encode(), g, None, None, None, None, None)
    if rc != 0:
        raise ImogenError(rc, lib().img_slice_last_error().decode())
    grid = tuple(g)
    n = grid[0] * grid[1] * grid[2]
    mass, ener = np.zeros(n), np.zeros(n)
    mom, mag = np.zeros(3 * n), np.zeros(3 * n)
    hm = ctypes.c_int()
    dp = ctypes.POINTER(ctypes.c_double)
    rc = lib().img_slice_read(str(path).encode(), g, mass.ctypes.data_as(dp), mom.ctypes.data_as(dp),
                              ener.ctypes.data_as(dp), mag.ctypes.data_as(dp), ctypes.byref(hm))
    if rc != 0:
        raise ImogenError(rc, lib().img_slice_last_error().decode())
    r = lambda a: a.reshape(grid, order="F")
    r3 = lambda a: np.stack([r(a[c * n:(c + 1) * n]) for c in range(3)])
    return (r(mass), r3(mom), r(ener), r3(mag)), bool(hm.value)


def bytes_required(**kw):
    c = make_config(**kw)
    return int(lib().img_bytes_required(ctypes.byref(c)))


class TimeManager:
    """run.time (time/TimeManager.m): update/running/step on the device-resident clock."""

    def __init__(self, run):
        self._run = run

    def update(self, flux_direction, sync=False):
        dt, gi = ctypes.c_double(), ctypes.c_int()
        r = self._run
        if sync:
            check(lib().img_time_update(r._h, int(flux_direction), ctypes.byref(dt), ctypes.byref(gi)), r._h)
            return dt.value, gi.value
        check(lib().img_time_update(r._h, int(flux_direction), None, None), r._h)
        return None

    def _get(self):
        t, dt, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        r = self._run
        check(lib().img_get_time(r._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it)), r._h)
        return t.value, dt.value, it.value

    @property
    def time(self):
        return self._get()[0]

    @property
    def dTime(self):
        return self._get()[1]

    @property
    def iteration(self):
        return self._get()[2]

    @property
    def running(self):
        t, _, it = self._get()
        return it <= self._run.config.iter_max and t < self._run.config.time_max

    def set(self, time, dt, iteration):
        r = self._run
        check(lib().img_set_time(r._h, float(time), float(dt), int(iteration)), r._h)


class ImogenRun:
    """One run of the hot path with its state resident on the current CUDA device."""

    def __init__(self, grid, **kw):
        self.config = make_config(grid, **kw)
        self.grid = tuple(self.config.grid)
        self.ncell = int(np.prod(self.grid))
        h = ctypes.c_void_p()
        rc = lib().img_create(ctypes.byref(h), ctypes.byref(self.config))
        check(rc, None)
        self._h = h
        self.time = TimeManager(self)

    def close(self):
        if getattr(self, "_h", None):
            lib().img_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- arrays (x fastest; numpy arrays shaped (nx, ny, nz) or flat) -----------------------------
    def _flat(self, a):
        a = np.asarray(a, dtype=np.float64)
        if a.ndim == 1:
            return np.ascontiguousarray(a)
        return np.ascontiguousarray(a.reshape(self.grid).ravel(order="F"))

    def set_state(self, mass, mom, ener, mag):
        """FluidArray/MagnetArray construction from the IC (imogen.m:34-42)."""
        m = self._flat(mass)
        e = self._flat(ener)
        p = np.concatenate([self._flat(mom[i]) for i in range(3)])
        b = np.concatenate([self._flat(mag[i]) for i in range(3)])
        check(lib().img_set_state(self._h, _dp(m), _dp(p), _dp(e), _dp(b)), self._h)

    def upload(self, name, arr):
        """X.array = value for one variable (ImogenArray.m:82-89); no copy when `arr` is already a
        flat C-contiguous float64 buffer (e.g. pinned host memory)."""
        a = self._flat(arr)
        check(lib().img_upload(self._h, VAR[name], _dp(a), a.size), self._h)

    def download(self, name, out=None):
        """get.array of one variable; `out` (a C-contiguous float64 buffer of ncell values, e.g.
        pinned host memory) is filled in place when given."""
        if out is None:
            out = np.empty(self.ncell)
            check(lib().img_download(self._h, VAR[name], _dp(out), out.size), self._h)
            return out.reshape(self.grid, order="F")
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == self.ncell
        check(lib().img_download(self._h, VAR[name], _dp(out), out.size), self._h)
        return out

    def upload_many(self, arrays):
        """{name: array} -> X.array = value for each, one synchronisation (flat C-contiguous float64
        buffers, e.g. pinned host memory, are used without a copy)."""
        names = list(arrays)
        flat = [self._flat(arrays[k]) for k in names]
        ids = (ctypes.c_int * len(names))(*[VAR[k] for k in names])
        ptrs = (ctypes.POINTER(ctypes.c_double) * len(names))(*[_dp(a) for a in flat])
        check(lib().img_upload_many(self._h, len(names), ids, ptrs, self.ncell), self._h)

    def download_many(self, outs):
        """{name: out} with out a C-contiguous float64 buffer of ncell values: filled in place, one
        synchronisation."""
        names = list(outs)
        for k in names:
            o = outs[k]
            assert o.dtype == np.float64 and o.flags.c_contiguous and o.size == self.ncell
        ids = (ctypes.c_int * len(names))(*[VAR[k] for k in names])
        ptrs = (ctypes.POINTER(ctypes.c_double) * len(names))(*[_dp(outs[k]) for k in names])
        check(lib().img_download_many(self._h, len(names), ids, ptrs, self.ncell), self._h)
        return outs

    def state(self):
        g = self.download
        return dict(mass=g("mass"), ener=g("ener"),
                    mom=np.stack([g("momx"), g("momy"), g("momz")]),
                    mag=np.stack([g("magx"), g("magy"), g("magz")]),
                    cellmag=np.stack([g("cmagx"), g("cmagy"), g("cmagz")]))

    # ---- the hot path ------------------------------------------------------------------------------
    def flux(self, order):
        check(lib().img_flux(self._h, int(order)), self._h)

    def relaxing_fluid(self, X):
        check(lib().img_fluid_sweep(self._h, int(X)), self._h)

    def source(self):
        """source.m for this path: the radiation sink E -= dTime * radiation.solve (source.m:30)."""
        check(lib().img_source(self._h), self._h)

    def save_slice(self, path, slice="XYZ", index=(1, 1, 1), suffix="FINAL", about="", version=0.0, wall_max=1e5,
                   started=None):
        """resultsHandler's save of one slice (save/resultsHandler.m:26-113) as a MAT-file (img_save_slice)."""
        m = slice_meta(slice, index, suffix, about, version, wall_max, started)
        check(lib().img_save_slice(self._h, str(path).encode(), ctypes.byref(m)), self._h)

    def load_slice(self, path):
        """Resume from a slice file as Initializer.loadDataFromFile does (img_load_slice)."""
        check(lib().img_load_slice(self._h, str(path).encode()), self._h)

    def treadmill(self):
        """treadmillGrid (treadmill/treadmillGrid.m) at the current iteration (iterate calls it after
        each flux)."""
        check(lib().img_treadmill(self._h), self._h)

    @property
    def treadmill_history(self):
        """(TreadmillManager.history as a list, TreadmillManager.last)."""
        n, last = ctypes.c_int(), ctypes.c_int()
        check(lib().img_treadmill_history(self._h, None, 0, ctypes.byref(n), ctypes.byref(last)), self._h)
        out = (ctypes.c_int * max(n.value, 1))()
        check(lib().img_treadmill_history(self._h, out, n.value, None, None), self._h)
        return list(out[:min(n.value, 1 << 16)]), last.value

    @property
    def radiation_strength(self):
        """Radiation.strength as Radiation.initialize set it from the state (0 without radiation)."""
        v = ctypes.c_double()
        check(lib().img_radiation_strength(self._h, ctypes.byref(v)), self._h)
        return v.value

    def magnet_flux(self, X, mag_indices):
        check(lib().img_magnet_sweep(self._h, int(X), int(mag_indices[0]), int(mag_indices[1])), self._h)

    def iterate(self):
        """imogen.m:60-66 loop body: two timesteps, then iteration += 1 (asynchronous)."""
        check(lib().img_step(self._h), self._h)

    def run(self, max_iterations=None):
        """while run.time.running: iterate (imogen.m:58-72).  Returns iterations executed."""
        n = ctypes.c_int()
        check(lib().img_run(self._h, -1 if max_iterations is None else int(max_iterations), ctypes.byref(n)),
              self._h)
        return n.value

    def sync(self):
        check(lib().img_sync(self._h), self._h)

    @property
    def stream(self):
        """cudaStream_t (as an int) that all of this run's kernels are launched on."""
        s = ctypes.c_void_p()
        check(lib().img_get_stream(self._h, ctypes.byref(s)), self._h)
        return s.value or 0

    @property
    def launches(self):
        n = ctypes.c_uint64()
        check(lib().img_launch_count(self._h, ctypes.byref(n)), self._h)
        return n.value

    def autotune(self, trials=3):
        """Pick the fastest pencil tiling per swept direction and kernel family (img_autotune);
        returns {"fluid": tiling("fluid"), "magnet": tiling("magnet")}."""
        check(lib().img_autotune(self._h, int(trials)), self._h)
        return {"fluid": self.tiling("fluid"), "magnet": self.tiling("magnet")}

    def tiling(self, kind="fluid"):
        """{dim: (pencils per CTA, threads per pencil, CTAs per cluster, threads per CTA, cells per thread,
        transverse components per CTA, segment layout)} of the fluid or the magnet sweeps."""
        out = {}
        base = 0 if kind == "fluid" else 3
        for d in (1, 2, 3):
            t = (ctypes.c_int * 7)()
            check(lib().img_get_tiling(self._h, base + d, t), self._h)
            out[d] = tuple(t)
        return out

    def set_tiling(self, dim, tiling, kind="fluid"):
        """Use one of the accepted tilings for direction dim (1..3) of the fluid or magnet sweeps."""
        vals = [int(v) for v in tiling]
        vals += [1, 0][len(vals) - 5:] if len(vals) < 7 else []
        t = (ctypes.c_int * 7)(*vals)
        check(lib().img_set_tiling(self._h, int(dim) + (0 if kind == "fluid" else 3), t), self._h)

    def checkpoint(self):
        """The run's complete resumable state as bytes (img_checkpoint_save)."""
        n = int(lib().img_checkpoint_bytes(self._h))
        buf = ctypes.create_string_buffer(n)
        check(lib().img_checkpoint_save(self._h, ctypes.cast(buf, ctypes.c_void_p), n), self._h)
        return buf.raw

    def restore(self, data):
        """Resume from checkpoint() bytes of a run with the same settings (img_checkpoint_load)."""
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        check(lib().img_checkpoint_load(self._h, ctypes.cast(buf, ctypes.c_void_p), len(data)), self._h)

    def progress(self):
        """(simulated time, iterations run, stopped) from the device clock (synchronises)."""
        t, n, st = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        check(lib().img_progress(self._h, ctypes.byref(t), ctypes.byref(n), ctypes.byref(st)), self._h)
        return t.value, n.value, bool(st.value)

    def totals(self):
        """Neumaier-compensated FP64 sums of rho, px, py, pz, E, Bx, By, Bz."""
        out = np.zeros(8)
        check(lib().img_totals(self._h, _dp(out)), self._h)
        return out

    def totals_static(self):
        """The same sums as totals(), computed in the library's static device scratch (no allocation)."""
        out = np.zeros(8)
        check(lib().img_totals_static(self._h, _dp(out)), self._h)
        return out


class ImogenBatch:
    """Many runs advanced together by batched launches (img_batch_*): one iteration of every member
    per step, each member with its own time step; members stay ImogenRun objects (upload,
    download, totals work on them as usual)."""

    def __init__(self, members=()):
        h = ctypes.c_void_p()
        rc = lib().img_batch_create(ctypes.byref(h))
        if rc != 0:
            raise ImogenError(rc, "batch creation failed")
        self._h = h
        self.members = []
        for m in members:
            self.add(m)

    def _check(self, rc):
        if rc != 0:
            msg = lib().img_batch_last_error(self._h)
            raise ImogenError(rc, msg.decode() if msg else "")

    def add(self, run):
        self._check(lib().img_batch_add(self._h, run._h))
        self.members.append(run)

    def remove(self, run):
        self._check(lib().img_batch_remove(self._h, run._h))
        self.members.remove(run)

    def step(self):
        self._check(lib().img_batch_step(self._h))

    def run(self, max_iterations=None, check_every=8):
        n = ctypes.c_int()
        self._check(lib().img_batch_run(self._h, -1 if max_iterations is None else int(max_iterations),
                                        int(check_every), ctypes.byref(n)))
        return n.value

    def status(self):
        """Per member: bit 0 stopped (TIMEMAX/ITERMAX), bit 1 error."""
        f = (ctypes.c_int * len(self.members))()
        self._check(lib().img_batch_status(self._h, f, len(self.members)))
        return list(f)

    @property
    def stream(self):
        s = ctypes.c_void_p()
        self._check(lib().img_batch_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    @property
    def launches(self):
        n = ctypes.c_uint64()
        self._check(lib().img_batch_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            lib().img_batch_destroy(self._h)
            self._h = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---- reference call surface ------------------------------------------------------------------------
def flux(run, mass, mom, ener, mag, grav, order):
    """flux(run, mass, mom, ener, mag, grav, order) -- flux/flux.m:1."""
    run.flux(order)


def source(run, mass, mom, ener, mag, grav):
    """source(run, mass, mom, ener, mag, grav) -- source.m:1 (radiation sink; no gravity)."""
    run.source()


def relaxingFluid(run, mass, mom, ener, mag, grav, X):
    """relaxingFluid(run, mass, mom, ener, mag, grav, X) -- fluid/relaxingFluid.m:1."""
    run.relaxing_fluid(X)


def magnetFlux(run, mass, mom, mag, X, magneticIndices):
    """magnetFlux(run, mass, mom, mag, X, magneticIndices) -- magnet/magnetFlux.m:1."""
    run.magnet_flux(X, magneticIndices)
