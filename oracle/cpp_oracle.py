"""ctypes front end of the C++ oracle (oracle/imogen_oracle.cpp).  TEST INFRASTRUCTURE ONLY.

Same call surface as ``oracle.np_oracle.Sim`` so tests can run either restatement.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from .np_oracle import (BC_MODES, MINMOD, PER_ITERATION, SUPERBEE, VANLEER, CIRC, VISC_NONE, VISC_NR, VISC_CSW,
                        RAD_NONE, RAD_THIN)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

BC_CLASSES = ("mass", "mom", "ener", "mag")
LIMITER_CODES = {VANLEER: 0, SUPERBEE: 1, MINMOD: 2}


def build():
    """Compile liboracle.so in place (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ip, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ip,
                                 ctypes.c_int, ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_state.argtypes = [ctypes.c_void_p, dp, dp, dp, dp]
        L.orc_get_state.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp]
        for name in ("orc_time_update", "orc_flux", "orc_relaxing_fluid", "orc_run"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_int]
            getattr(L, name).restype = ctypes.c_int
        L.orc_magnet_flux.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_iterate.argtypes = [ctypes.c_void_p]
        L.orc_source.argtypes = [ctypes.c_void_p]
        L.orc_set_fade.argtypes = [ctypes.c_void_p, ip, ctypes.c_double, ctypes.c_int]
        L.orc_treadmill.argtypes = [ctypes.c_void_p]
        L.orc_set_treadmill.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_treadmill_history.argtypes = [ctypes.c_void_p, ip, ctypes.c_int]
        L.orc_treadmill_history.restype = ctypes.c_int
        L.orc_treadmill_last.argtypes = [ctypes.c_void_p]
        L.orc_treadmill_last.restype = ctypes.c_int
        L.orc_radiation_strength.argtypes = [ctypes.c_void_p]
        L.orc_radiation_strength.restype = ctypes.c_double
        L.orc_get_time.argtypes = [ctypes.c_void_p, dp, dp, ip]
        L.orc_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.orc_get_cfl.argtypes = [ctypes.c_void_p, dp, ip]
        L.orc_pchip.argtypes = [dp, ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_int, dp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_sweep_order.argtypes = [ctypes.c_int, ctypes.c_int, ip]
        L.orc_set_physics.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_double]
        L.orc_max_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def bc_codes(bc):
    """bc (mode string, or {class: [[lower x,y,z],[upper x,y,z]]}) -> int32[4,2,3]."""
    out = np.zeros((4, 2, 3), dtype=np.int32)
    if bc is None or isinstance(bc, str):
        out[:] = BC_MODES.index(bc or CIRC)
        return out
    for c, name in enumerate(BC_CLASSES):
        for s in range(2):
            for d in range(3):
                out[c, s, d] = BC_MODES.index(bc[name][s][d])
    return out


def pchip(x, y, xi):
    x = np.ascontiguousarray(x, dtype=float)
    y = np.ascontiguousarray(np.atleast_2d(y), dtype=float)
    xi = np.ascontiguousarray(np.atleast_1d(xi), dtype=float)
    out = np.zeros((y.shape[0], xi.size))
    lib().orc_pchip(_dp(x), x.size, _dp(y), y.shape[0], _dp(xi), xi.size, _dp(out))
    return out


def sweep_order(order, iteration):
    """directVec of flux.m:17-27 as the C++ oracle's tables hold it."""
    out = np.zeros(3, np.int32)
    lib().orc_sweep_order(int(order), int(iteration), _ip(out))
    return tuple(int(v) for v in out)


def set_threads(n):
    lib().orc_set_threads(int(n))


def max_threads():
    return lib().orc_max_threads()


class Sim:
    """C++ oracle run; arrays are (nx, ny, nz) like np_oracle.Sim."""

    def __init__(self, grid, dgrid, gamma=5 / 3, cfl=0.7, minmass=1e-5, bc=None,
                 bc_infinity=20, limiter=(VANLEER,) * 3, fluid_active=True,
                 magnet_active=False, time_max=1e5, iter_max=10, update_mode=PER_ITERATION,
                 viscosity=VISC_NONE, visc_linear=0.0, visc_quadratic=0.0,
                 radiation=RAD_NONE, rad_exponent=0.5, rad_initial_maximum=0.0, treadmill=0,
                 fade_location=None, fade_size=0.0, fade_active=()):
        self.grid = tuple(int(g) for g in grid)
        g = np.array(self.grid, dtype=np.int32)
        dg = np.array(dgrid, dtype=float)
        bcc = bc_codes(bc)
        lim = np.array([LIMITER_CODES[l] for l in limiter], dtype=np.int32)
        self._h = lib().orc_create(_ip(g), _dp(dg), gamma, cfl, minmass, _ip(bcc), int(bc_infinity),
                                   _ip(lim), int(fluid_active), int(magnet_active), float(time_max),
                                   int(iter_max), int(update_mode))
        if not self._h:
            raise ValueError("BC settings not defined for this grid (see np_oracle.validate_bc)")
        lib().orc_set_physics(self._h, {VISC_NONE: 0, VISC_NR: 1, VISC_CSW: 2}[viscosity], float(visc_linear),
                              float(visc_quadratic), {RAD_NONE: 0, RAD_THIN: 1}[radiation], float(rad_exponent),
                              float(rad_initial_maximum))
        lib().orc_set_treadmill(self._h, int(treadmill))
        if fade_location is not None:
            mask = sum(b for name, b in (("mass", 1), ("mom", 2), ("ener", 4)) if name in fade_active)
            loc = np.array([int(v) for v in fade_location], dtype=np.int32)
            lib().orc_set_fade(self._h, _ip(loc), float(fade_size), mask)
        self.TIMEMAX = float(time_max)
        self.ITERMAX = int(iter_max)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def _flat(self, a):
        return np.ascontiguousarray(np.asarray(a, dtype=float).reshape(self.grid).ravel(order="F"))

    def set_state(self, mass, mom, ener, mag):
        m = self._flat(mass)
        e = self._flat(ener)
        p = np.concatenate([self._flat(mom[i]) for i in range(3)])
        b = np.concatenate([self._flat(mag[i]) for i in range(3)])
        lib().orc_set_state(self._h, _dp(m), _dp(p), _dp(e), _dp(b))

    def state(self):
        n = int(np.prod(self.grid))
        m, e = np.zeros(n), np.zeros(n)
        p, b, cb = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n)
        lib().orc_get_state(self._h, _dp(m), _dp(p), _dp(e), _dp(b), _dp(cb))
        r = lambda v: v.reshape(self.grid, order="F")
        r3 = lambda v: np.stack([r(v[i * n:(i + 1) * n]) for i in range(3)])
        return dict(mass=r(m), ener=r(e), mom=r3(p), mag=r3(b), cellmag=r3(cb))

    def time_update(self, flux_direction):
        if lib().orc_time_update(self._h, int(flux_direction)) != 0:
            raise FloatingPointError("CFL error")

    def flux(self, order):
        lib().orc_flux(self._h, int(order))

    def relaxing_fluid(self, X):
        lib().orc_relaxing_fluid(self._h, int(X))

    def magnet_flux(self, X, mag_indices):
        lib().orc_magnet_flux(self._h, int(X), int(mag_indices[0]), int(mag_indices[1]))

    def source(self):
        """source.m:30: the radiation sink with the current dTime."""
        lib().orc_source(self._h)

    def treadmill(self):
        """treadmillGrid (treadmill/treadmillGrid.m:14-37)."""
        lib().orc_treadmill(self._h)

    @property
    def treadmill_history(self):
        n = lib().orc_treadmill_history(self._h, None, 0)
        out = (ctypes.c_int * max(n, 1))()
        lib().orc_treadmill_history(self._h, out, n)
        return list(out[:n])

    @property
    def treadmill_last(self):
        return lib().orc_treadmill_last(self._h)

    @property
    def rad_strength(self):
        return lib().orc_radiation_strength(self._h)

    def iterate(self):
        if lib().orc_iterate(self._h) != 0:
            raise FloatingPointError("CFL error")

    def run(self, max_iterations=None):
        n = lib().orc_run(self._h, -1 if max_iterations is None else int(max_iterations))
        if n < 0:
            raise FloatingPointError("CFL error")
        return n

    def _time(self):
        t, dt, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        lib().orc_get_time(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it))
        return t.value, dt.value, it.value

    @property
    def time(self):
        return self._time()[0]

    @property
    def dTime(self):
        return self._time()[1]

    @property
    def iteration(self):
        return self._time()[2]

    def set_time(self, time, dt, iteration):
        lib().orc_set_time(self._h, float(time), float(dt), int(iteration))

    @property
    def last_cfl(self):
        c, g = ctypes.c_double(), ctypes.c_int()
        lib().orc_get_cfl(self._h, ctypes.byref(c), ctypes.byref(g))
        return c.value, g.value

    @property
    def running(self):
        t, _, it = self._time()
        return it <= self.ITERMAX and t < self.TIMEMAX
