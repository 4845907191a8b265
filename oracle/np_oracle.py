"""NumPy restatement of Imogen's relaxing-TVD fluid + magnet update (TEST INFRASTRUCTURE ONLY).

This module is an oracle: tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use it as a checker.  The product path (``imogen_b200``) never imports it.

It is a literal, array-at-a-time restatement of the reference MATLAB code, written so each
statement can be read against the file it follows:

* ``flux/flux.m:17-62``               sweep order table, forward/backward fluxing
* ``fluid/relaxingFluid.m:16-73``     predictor / TVD corrector for rho, p, E
* ``fluid/wFluidFlux.m:14-44``        freezing speed and relaxing W fluxes
* ``pressure/pressure.m:16-66``       pressure modes
* ``flux/{vanleer,minmod,superbee}Limiter.m``
* ``magnet/magnetFlux.m:14-31``, ``magnet/relaxingMagnet.m:15-60``, ``magnet/MagnetArray.m:36-38``
* ``time/TimeManager.m:55-99``        CFL timestep
* ``classes/ImogenArray.m:80-89,156-166``, ``classes/InitializedArray.m:43-47``
* ``shifting/{circ,constant,mirror,transparent,wall,fade}_shift.m``, ``shifting/Edges.m``
* ``imogen.m:50-72``                  main loop ordering

Parity status: the reference is MATLAB and cannot run here, so this oracle is pinned only at
the MATLAB-builtin boundary (``pchip`` against SciPy's PchipInterpolator, the ``perms`` row
order by a restatement of the R2009-era ``perms`` algorithm, ``matlab_perms``) and by analytic /
invariant checks
(exact Sod Riemann solution, conservation under periodic BCs, discrete div B under CT).
Parity against the reference itself is therefore *unpinned*.

Arrays are stored as numpy arrays of shape (nx, ny, nz) indexed a[x, y, z]; the MATLAB
dimension number d (1-based) is axis d-1 here.
"""
from __future__ import annotations

import math

import numpy as np

CIRC, CONST, FADE, MIRROR, TRANS, WALL = "circ", "const", "fade", "mirror", "trans", "wall"
FLIP, ZERO, LINEAR, WORMHOLE = "flip", "zero", "linear", "wormhole"
BC_MODES = (CIRC, CONST, FADE, MIRROR, TRANS, WALL, FLIP, ZERO, LINEAR, WORMHOLE)
# FluxArray.fluxType (flux/FluxArray.m:28-35) as zero_shift.m reads it (None: not a FluxArray)
FLUXR, FLUXL, FLUX = "fluxr", "fluxl", "flux"
VANLEER, SUPERBEE, MINMOD = "vanleer", "superbee", "minmond"   # FluxLimiterEnum.m:10-13
PER_STEP, PER_ITERATION = 0, 1                                  # enums/ENUM.m:33-34
VISC_NONE, VISC_NR, VISC_CSW = "empty", "neumann_richtmyer", "caramana_shashkov_whalen"   # ENUM.m:53-55
RAD_NONE, RAD_THIN = "empty", "optically_thin"                  # ENUM.m:49-50



def perms_positions(n):
    """Rows of ``perms(1:n)`` as MATLAB R2009a-R2010b builds them (the releases the reference
    targets).  Recursive on n: the first m = (n-1)! rows are ``[n, perms(1:n-1)]``; then, for
    i = n-1 down to 1, the next m rows are ``[i, q']`` where q' is ``perms(1:n-1)`` with the
    value i relabelled to n (``t(t == i) = n``).  The relabelling is monotone only for
    i = n-1, so the rows are not strictly reverse-lexicographic: for n = 3 they are
    321, 312, 231, 213, 123, 132."""
    if n <= 1:
        return ((1,),) if n == 1 else ((),)
    q = perms_positions(n - 1)
    rows = [(n,) + r for r in q]
    for i in range(n - 1, 0, -1):
        rows += [(i,) + tuple(n if t == i else t for t in r) for r in q]
    return tuple(rows)


def matlab_perms(v):
    """``perms(V)`` of that era: ``V(P)`` with P = ``perms_positions(numel(V))`` (the permutations
    are of positions, then applied to V, so ``perms([3 2 1])`` is ``4 - perms(1:3)``)."""
    return tuple(tuple(v[i - 1] for i in row) for row in perms_positions(len(v)))


# flux.m:19 and flux.m:24: the forward rows are perms([1 2 3]), the backward rows perms([3 2 1]);
# row mod(iteration-1, 6)+1 is used (flux.m:20,25).
FORWARD_ORDER = matlab_perms((1, 2, 3))
BACKWARD_ORDER = matlab_perms((3, 2, 1))
FORWARD_MAGIDX = {1: (2, 3), 2: (1, 3), 3: (1, 2)}     # flux.m:21
BACKWARD_MAGIDX = {1: (3, 2), 2: (3, 1), 3: (2, 1)}    # flux.m:27


# --------------------------------------------------------------------------------------------
# pchip (MATLAB pchip, Fritsch-Carlson slopes with Fritsch-Butland harmonic weights and the
# one-sided shape-preserving end formula, as published in Moler, "Numerical Computing with
# MATLAB", pchiptx).  Vectorised over the leading axes of y.
# --------------------------------------------------------------------------------------------
def pchip_slopes(x, y):
    x = np.asarray(x, dtype=float)
    h = np.diff(x)
    delta = np.diff(y, axis=-1) / h
    n = x.size
    d = np.zeros_like(y, dtype=float)
    for k in range(1, n - 1):
        dl, dr = delta[..., k - 1], delta[..., k]
        w1 = 2 * h[k] + h[k - 1]
        w2 = h[k] + 2 * h[k - 1]
        ok = (np.sign(dl) * np.sign(dr)) > 0
        with np.errstate(divide="ignore", invalid="ignore"):
            dk = (w1 + w2) / (w1 / dl + w2 / dr)
        d[..., k] = np.where(ok, dk, 0.0)

    def endslope(h0, h1, del0, del1):
        dd = ((2 * h0 + h1) * del0 - h0 * del1) / (h0 + h1)
        dd = np.where(np.sign(dd) != np.sign(del0), 0.0, dd)
        big = (np.sign(del0) != np.sign(del1)) & (np.abs(dd) > np.abs(3 * del0))
        return np.where(big, 3 * del0, dd)

    d[..., 0] = endslope(h[0], h[1], delta[..., 0], delta[..., 1])
    d[..., n - 1] = endslope(h[n - 2], h[n - 3], delta[..., n - 2], delta[..., n - 3])
    return d, delta, h


def pchip(x, y, xi):
    """pchip(x, y, xi) with y[..., len(x)] -> [..., len(xi)] (MATLAB pchip semantics)."""
    x = np.asarray(x, dtype=float)
    y = np.asarray(y, dtype=float)
    xi = np.atleast_1d(np.asarray(xi, dtype=float))
    d, delta, h = pchip_slopes(x, y)
    out = np.empty(y.shape[:-1] + (xi.size,))
    for m, xv in enumerate(xi):
        # interval index as ppval: the last breakpoint interval containing xv (clamped)
        k = int(np.searchsorted(x, xv, side="right") - 1)
        k = min(max(k, 0), x.size - 2)
        s = xv - x[k]
        c1 = (d[..., k] + d[..., k + 1] - 2 * delta[..., k]) / (h[k] * h[k])
        c2 = (3 * delta[..., k] - 2 * d[..., k] - d[..., k + 1]) / h[k]
        c3 = d[..., k]
        c4 = y[..., k]
        out[..., m] = ((c1 * s + c2) * s + c3) * s + c4
    return out


def fade_coefficients(fade_size):
    """fade_shift.m:31 -- pchip([0 ceil(f/4) round(f/2) f-1 f],[1 1 .01 0 0],1:f)."""
    f = int(fade_size)
    half = int(np.floor(f / 2 + 0.5))   # MATLAB round: half away from zero
    xk = [0, int(np.ceil(f / 4)), half, f - 1, f]
    return pchip(xk, np.array([1, 1, 0.01, 0, 0], dtype=float), np.arange(1, f + 1))


# --------------------------------------------------------------------------------------------
# Edges (shifting/Edges.m)
# --------------------------------------------------------------------------------------------
class Edges:
    """Per-array stored edge slices for trans/wall/fade edges (Edges.m:37-110)."""

    def __init__(self, bc_modes, array, ndims, tolerance):
        self.TOLERANCE = tolerance
        self.ACTIVE = np.zeros((2, 3), dtype=bool)
        self.store = ({}, {})          # (lower, upper) -> {dim: slice}
        for n in range(2):
            for i in range(ndims):
                mode = bc_modes[n][i]
                if mode in (TRANS, WALL):
                    self.ACTIVE[n, i] = True
                    idx = 0 if n == 0 else array.shape[i] - 1
                    self.store[n][i] = np.take(array, idx, axis=i).copy()
                elif mode == FADE:
                    # Edges.m:80-93 stores a 20-cell slab; fade_shift never reads it.
                    self.ACTIVE[n, i] = True

    def get_edge(self, upper, dim, array, bc_type):
        """Edges.getEdge (Edges.m:112-137); trans edges drift by <= TOLERANCE per call."""
        side = 1 if upper else 0
        if bc_type == TRANS:
            idx = 0 if not upper else array.shape[dim] - 1
            new_edge = np.take(array, idx, axis=dim)
            old_edge = self.store[side][dim]
            delta = np.minimum(np.abs(new_edge - old_edge), self.TOLERANCE)
            sign_test = (new_edge - old_edge) > 0
            result = old_edge + (sign_test.astype(float) - (~sign_test).astype(float)) * delta
            self.store[side][dim] = result
            return result
        return self.store[side][dim]   # fade / wall


def _lpow(x, e):
    """x**e elementwise with the C library's pow (correctly rounded; NumPy's vectorised power may differ
    in the last bit), and the square root for e = 0.5 as NumPy's power takes it."""
    x = np.asarray(x, dtype=float)
    if e == 0.5:
        return np.sqrt(x)

    def one(v):
        try:
            return math.pow(v, e)
        except (ValueError, OverflowError):
            return float("nan")
    return np.frompyfunc(one, 1, 1)(x).astype(float)


# --------------------------------------------------------------------------------------------
# ImogenArray (classes/ImogenArray.m) with the BC shift functions (shifting/*_shift.m)
# --------------------------------------------------------------------------------------------
class IArray:
    """An ImogenArray: data + component + per-side/per-dim BC modes + stored edges.

    ``initialized=False`` gives an InitializedArray (edges taken at first assignment,
    InitializedArray.m:43-47); ``True`` gives a primary array whose edges come from the IC.
    """

    def __init__(self, sim, component, bc_class, data=None, flux_type=None):
        self.sim = sim
        self.component = component          # 0 scalar, 1..3 vector component
        self.flux_type = flux_type          # FluxArray type, None for other arrays
        self.bc_modes = sim.bc[bc_class]    # [side][dim]
        self.a = None
        self.edges = None
        self.uninitialized = True
        if data is not None:
            self.set(data)

    # set.array (ImogenArray.m:82-89): point fades of the array (readFades, primaries only), then the
    # first-assignment edges; statics cannot occur (StaticsInitializer.m does not parse: one `end` short)
    def set(self, value):
        if getattr(self, "fades", None) is not None:   # PointFade.fadeArray (PointFade.m:46-49)
            A = self.fades
            value = 0.95 * value * A + value * (1 - A)
        self.a = value
        if self.uninitialized:
            self.edges = Edges(self.bc_modes, value, self.sim.ndims, 0.005)
            self.uninitialized = False

    def cleanup(self):
        self.a = None

    def shift_enabled(self, d):
        return d < self.sim.ndims

    def shift(self, DIRECT, n):
        """ImogenArray.shift (ImogenArray.m:156-166); DIRECT is 1-based."""
        d = DIRECT - 1
        if not self.shift_enabled(d):
            return self.a
        mode = self.bc_modes[1 if n > 0 else 0][d]
        fn = {CIRC: _circ_shift, CONST: _constant_shift, MIRROR: _mirror_shift,
              TRANS: _transparent_shift, WALL: _wall_shift, FADE: _fade_shift, FLIP: _flip_shift,
              ZERO: _zero_shift, LINEAR: _linear_shift, WORMHOLE: _wormhole_shift}[mode]
        return fn(self.a, DIRECT, n, self)

    def transparent_edge(self, dim, upper):
        """ImogenArray.transparentEdge (ImogenArray.m:170-172)."""
        d = dim - 1
        return self.edges.get_edge(upper, d, self.a, self.bc_modes[1 if upper else 0][d])


def _take(a, idx, axis):
    return np.take(a, np.asarray(idx, dtype=np.intp), axis=axis)


def _const_index(N, n):
    """0-based source index of constant_shift.m:21-29."""
    i = np.arange(N)
    return np.clip(i + n, 0, N - 1)


def _circ_shift(a, DIRECT, n, obj):
    return np.roll(a, -n, axis=DIRECT - 1)                       # circ_shift.m:21-29


def _constant_shift(a, DIRECT, n, obj):
    d = DIRECT - 1
    return _take(a, _const_index(a.shape[d], n), d)              # constant_shift.m:21-29


def point_fade_array(grid, location, fade_size):
    """PointFade(grid, location, fadeSize).array (classes/PointFade.m:29-38): with r the offset of a cell
    from `location` (1-based), d = max(s^2 - |r|^2, 0), the map pchip([-1 0 1 2], [1 1 0 0], 1 - d/max d):
    1 at the location, 0 beyond the radius s."""
    g = [int(v) for v in grid]
    loc = [float(v) for v in location]
    ax = [np.arange(1 - loc[i], g[i] - loc[i] + 1) for i in range(3)]
    x, y, z = np.meshgrid(*ax, indexing="ij")
    s = float(fade_size)
    d = np.maximum(s * s - (x * x + y * y + z * z), 0)
    d = 1 - d / float(np.max(d))
    return pchip([-1, 0, 1, 2], np.array([1.0, 1.0, 0.0, 0.0]), d.reshape(-1, order="F")).reshape(g, order="F")


def _mean_of_means(idx):
    """mean(mean(A)) of treadmillGrid.m:22 for the index array of the non-swept dimensions (x
    fastest): MATLAB's mean runs along the first non-singleton dimension, so the first mean averages
    along the lower of the two remaining dimensions, the second along the other (each a sum in index
    order divided by the count)."""
    a = np.asarray(idx, dtype=float)
    a = a.reshape([s for s in a.shape if s > 1] or [1])
    if a.ndim == 2:
        first = []
        for k in range(a.shape[1]):
            s = 0.0
            for j in range(a.shape[0]):
                s += a[j, k]
            first.append(s / a.shape[0])
        vals = first
    else:
        vals = list(a.reshape(-1))
    s = 0.0
    for v in vals:
        s += v
    return s / len(vals)


def _matlab_round(x):
    """MATLAB round: halves away from zero."""
    r = math.floor(abs(x))
    if abs(x) - r >= 0.5:
        r += 1
    return int(r) * (1 if x >= 0 else -1)


def _ghost_slice(a, d, n):
    sl = [slice(None)] * a.ndim
    N, m = a.shape[d], abs(n)
    sl[d] = slice(0, m) if n < 0 else slice(N - m, N)
    return tuple(sl)


def _flip_shift(a, DIRECT, n, obj):
    """flip_shift.m:22-40: the constant shift with its ghosts negated for the component along DIRECT."""
    result = _constant_shift(a, DIRECT, n, obj)
    if obj.component == DIRECT:
        g = _ghost_slice(result, DIRECT - 1, n)
        result[g] = -result[g]
    return result


def _zero_shift(a, DIRECT, n, obj):
    """zero_shift.m:14-46: a FluxArray's ghosts are 0, except that fluxl keeps the constant shift for
    n < 0 and fluxr for n > 0; any other array takes the constant shift."""
    result = _constant_shift(a, DIRECT, n, obj)
    if obj.flux_type is None or obj.flux_type == (FLUXL if n < 0 else FLUXR):
        return result
    result[_ghost_slice(result, DIRECT - 1, n)] = 0.0
    return result


def _linear_shift(a, DIRECT, n, obj):
    """linear_shift.m:20 indexes with the variable `dim`, which the function never defines: the
    reference stops with an undefined-variable error at the first shift."""
    raise NameError("linear_shift.m: undefined function or variable 'dim'")


def _wormhole_shift(a, DIRECT, n, obj):
    """wormhole_shift.m:16-61: for n < 0 the first |n| ghosts along DIRECT are the first |n| cells in
    reverse order along DIRECT and along nextDir = [2 3 1](DIRECT), negated for the component along
    DIRECT; for n > 0 the constant shift."""
    result = _constant_shift(a, DIRECT, n, obj)
    if n > 0:
        return result
    d, m = DIRECT - 1, abs(n)
    dn = (d + 1) % 3                       # nextDir(DIRECT) - 1
    sl = [slice(None)] * 3
    sl[d] = slice(0, m)
    temp = a[tuple(sl)]
    temp = np.flip(np.flip(temp, axis=d), axis=dn)
    result[tuple(sl)] = (-1.0 if obj.component == DIRECT else 1.0) * temp
    return result


def _mirror_shift(a, DIRECT, n, obj):
    """mirror_shift.m:23-39: reflect across the edge cell (excluded); flip if component==DIRECT."""
    d = DIRECT - 1
    N = a.shape[d]
    m = abs(n)
    idx = np.arange(N)
    if n < 0:
        idx[m:] = np.arange(N - m)
        flip = np.arange(m)
        idx[flip] = np.arange(m, 0, -1)            # (n+1):-1:2 (1-based)
    else:
        idx[:N - m] = np.arange(m, N)
        flip = np.arange(N - m, N)
        idx[flip] = np.arange(N - 2, N - 2 - m, -1)  # (N-1):-1:(N-n) (1-based)
    result = _take(a, idx, d)
    if obj.component == DIRECT:
        sl = [slice(None)] * a.ndim
        sl[d] = flip
        result[tuple(sl)] = -result[tuple(sl)]
    return result


def _transparent_shift(a, DIRECT, n, obj):
    """transparent_shift.m:23-99: pchip extrapolation toward the stored (drifting) edge."""
    d = DIRECT - 1
    N = a.shape[d]
    m = abs(n)
    inf = obj.sim.bc_infinity
    # edgeStore.ACTIVE(DIRECT): linear (column-major) index into the 2x3 matrix
    active = obj.edges.ACTIVE[(DIRECT - 1) % 2, (DIRECT - 1) // 2]
    src = _const_index(N, n)
    result = _take(a, src, d)
    ad = np.moveaxis(a, d, -1)
    rd = np.moveaxis(result, d, -1)
    vals = np.zeros(ad.shape[:-1] + (5,))
    if n < 0:
        pick = np.minimum(np.array([3, 2, 1]) + m, N) - 1       # min((3:-1:1)+n, NDim)
        vals[..., 0:3] = rd[..., pick]
        if active:
            e = obj.transparent_edge(DIRECT, False)
            vals[..., 3] = np.reshape(e, vals.shape[:-1])
            vals[..., 4] = vals[..., 3]
        out = pchip([1, 2, 3, inf, inf + 1], vals, 3 + np.arange(m, 0, -1))
        ghost = np.arange(m)
    else:
        pick = np.maximum(N - np.array([2, 1, 0]) - m, 1) - 1   # max(NDim-(2:-1:0)-n, 1)
        vals[..., 0:3] = rd[..., pick]
        if active:
            e = obj.transparent_edge(DIRECT, True)
            vals[..., 3] = np.reshape(e, vals.shape[:-1])
            vals[..., 4] = vals[..., 3]
        out = pchip([1, 2, 3, inf, inf + 1], vals, 3 + np.arange(1, m + 1))
        ghost = np.arange(N - m, N)
    orig = ad[..., ghost]
    test = np.abs(orig - out) < 1e-4
    out = (~test).astype(float) * out + test.astype(float) * orig
    rd = rd.copy()
    rd[..., ghost] = out
    return np.moveaxis(rd, -1, d)


def _wall_shift(a, DIRECT, n, obj):
    """wall_shift.m:12-33: constant shift, ghosts = edge stored at IC / first assignment."""
    d = DIRECT - 1
    N = a.shape[d]
    m = abs(n)
    result = _constant_shift(a, DIRECT, n, obj)
    rd = np.moveaxis(result, d, -1).copy()
    if n < 0:
        e = obj.transparent_edge(DIRECT, False)
        ghost = np.arange(m)
    else:
        e = obj.transparent_edge(DIRECT, True)
        ghost = np.arange(N - m, N)
    e = np.reshape(e, rd.shape[:-1])
    for g in ghost:
        rd[..., g] = e
    return np.moveaxis(rd, -1, d)


def _fade_shift(a, DIRECT, n, obj):
    """fade_shift.m:21-45: constant shift, then blend first/last f cells toward the edges."""
    d = DIRECT - 1
    N = a.shape[d]
    f = obj.sim.bc_infinity
    coeff = obj.sim.fade_coeff
    rd = np.moveaxis(_constant_shift(a, DIRECT, n, obj), d, -1).copy()
    anchor = rd[..., 0:1]
    rd[..., 0:f] = (1 - coeff) * rd[..., 0:f] + coeff * anchor
    anchor = rd[..., N - 1:N]
    cflip = coeff[::-1]
    rd[..., N - f:N] = (1 - cflip) * rd[..., N - f:N] + cflip * anchor
    return np.moveaxis(rd, -1, d)


# --------------------------------------------------------------------------------------------
# Limiters (flux/*Limiter.m): in-place correction of a flux array
# --------------------------------------------------------------------------------------------
def _vanleer(flux, dL, dR):
    with np.errstate(divide="ignore", invalid="ignore"):
        prod = dL * dR
        sign_test = np.where(prod > 0, prod, 0.0) / (dL + dR)   # max(dL.*dR,0)./(dL+dR)
    sign_test = np.where(np.isnan(sign_test), 0.0, sign_test)
    flux.set(flux.a + sign_test)


def _minmod(flux, dL, dR):
    corr = 0.125 * (np.sign(dL) + np.sign(dR)) * np.fmin(np.abs(dL), np.abs(dR))
    flux.set(flux.a + corr)


def _superbee(flux, dL, dR):
    coeff = (np.abs(dL) < np.abs(dR)).astype(float)
    _minmod(flux, (1 + coeff) * dL, (2 - coeff) * dR)


LIMITERS = {VANLEER: _vanleer, MINMOD: _minmod, SUPERBEE: _superbee}


# --------------------------------------------------------------------------------------------
# Simulation state holder (the managers + arrays of imogen.m)
# --------------------------------------------------------------------------------------------
class FluidVar:
    """FluidArray with its StorageArray and FluxArrays (FluidArray.m:102-106, StorageArray.m)."""

    def __init__(self, sim, component, bc_class, data):
        self.prim = IArray(sim, component, bc_class, data)
        self.store = IArray(sim, component, bc_class)
        self.store_fluxR = IArray(sim, component, bc_class, flux_type=FLUXR)   # StorageArray.m:69-70
        self.store_fluxL = IArray(sim, component, bc_class, flux_type=FLUXL)
        self.fluxR = IArray(sim, component, bc_class, flux_type=FLUXR)         # FluidArray.m:104-105
        self.fluxL = IArray(sim, component, bc_class, flux_type=FLUXL)
        self.w = None
        self.store_w = None


class MagComp:
    """MagnetArray (MagnetArray.m): primary face-centred B plus per-direction scratch arrays."""

    def __init__(self, sim, component, data):
        self.prim = IArray(sim, component, "mag", data)
        self.velGrid, self.store, self.store_fluxR, self.wMag, self.flux = {}, {}, {}, {}, {}
        for X in (1, 2, 3):
            if X == component:
                continue
            for tab in (self.velGrid, self.store, self.wMag):
                tab[X] = IArray(sim, component, "mag")
            self.store_fluxR[X] = IArray(sim, component, "mag", flux_type=FLUXR)   # StorageArray.m:70
            self.flux[X] = IArray(sim, component, "mag", flux_type=FLUX)           # MagnetArray.m:96
        self.cellMag = IArray(sim, component, "mag")
        self.update_cell_centered()

    def update_cell_centered(self):
        """MagnetArray.updateCellCentered (MagnetArray.m:36-38)."""
        c = self.prim.component
        self.cellMag.set(0.5 * (self.prim.a + self.prim.shift(c, 1)))


def validate_bc(grid, ndims, bc, bc_infinity):
    """Reject BC settings whose MATLAB shift functions index outside the array.

    mirror_shift.m:31-33 reads cell 2 / N-1, and fade_shift.m:34-44 plus Edges.m:80-93 read
    the first and last max(20, bcInfinity) cells, so on a shift-enabled dimension that is too
    short the reference stops with an index error.  Such runs are not defined.
    """
    for cls, sides in bc.items():
        for s in range(2):
            for d in range(ndims):
                mode = sides[s][d]
                if mode not in BC_MODES:
                    raise ValueError(f"unknown BC mode {mode!r}")
                if mode == MIRROR and grid[d] < 2:
                    raise ValueError(f"mirror BC on dim {d + 1} of extent {grid[d]}")
                if mode == FADE and grid[d] < max(20, bc_infinity):
                    raise ValueError(f"fade BC on dim {d + 1} of extent {grid[d]} < max(20, bcInfinity)")
                if mode == LINEAR:
                    raise ValueError("linear BC: linear_shift.m:20 uses the undefined variable 'dim'")
                if mode == WORMHOLE and s == 0 and ndims < 3:
                    raise ValueError("wormhole BC on a 2-D grid: wormhole_shift.m:27-33 indexes a third dimension")


class Sim:
    """One Imogen run of the relaxing-TVD hot path.

    bc: {'mass'|'mom'|'ener'|'mag': [[lower x,y,z], [upper x,y,z]]} of mode strings.
    """

    def __init__(self, grid, dgrid, gamma=5 / 3, cfl=0.7, minmass=1e-5, bc=None,
                 bc_infinity=20, limiter=(VANLEER,) * 3, fluid_active=True,
                 magnet_active=False, time_max=1e5, iter_max=10, update_mode=PER_ITERATION,
                 viscosity=VISC_NONE, visc_linear=0.0, visc_quadratic=0.0,
                 radiation=RAD_NONE, rad_exponent=0.5, rad_initial_maximum=0.0, treadmill=0,
                 fade_location=None, fade_size=0.0, fade_active=()):
        self.grid = tuple(int(g) for g in grid)
        self.ndims = 3 if self.grid[2] > 1 else 2
        self.dgrid = tuple(float(v) for v in dgrid)
        self.MINDGRID = self.dgrid
        self.GAMMA = float(gamma)
        self.CFL = float(cfl)
        self.MINMASS = float(minmass)
        if bc is None or isinstance(bc, str):
            mode = bc or CIRC
            bc = {k: [[mode] * 3, [mode] * 3] for k in ("mass", "mom", "ener", "mag")}
        self.bc = bc
        self.bc_infinity = int(bc_infinity)
        validate_bc(self.grid, self.ndims, bc, self.bc_infinity)
        self.fade_coeff = fade_coefficients(self.bc_infinity)
        self.limiter = tuple(limiter)
        self.fluid_active = fluid_active
        self.magnet_active = magnet_active
        self.TIMEMAX = float(time_max)
        self.ITERMAX = int(iter_max)
        self.updateMode = int(update_mode)
        self.time = 0.0
        self.dTime = 0.0
        self.iteration = 1
        self.history = []
        # ArtificialViscosity (ArtificialViscosity.m:31-57) and Radiation (Radiation.m:32-57) settings
        self.visc_type = viscosity
        self.visc_linear = float(visc_linear)
        self.visc_quadratic = float(visc_quadratic)
        self.rad_type = radiation
        self.rad_exponent = float(rad_exponent)
        self.rad_initial_maximum = float(rad_initial_maximum)
        self.rad_strength = 1.0
        # TreadmillManager (treadmill/TreadmillManager.m): ini.treadmill > 0 activates it along that
        # direction (initialize.m:328-331); `last` starts at -1 and the history is kept
        # one PointFade (ImogenManager.addFades, ImogenManager.m:262-280; classes/PointFade.m:29-38): the
        # damping map and the ids of the arrays it acts on ('mass', 'mom', 'ener'; 'mag' and 'grav' are
        # accepted there but no MagnetArray reads fades)
        self.fade_array = point_fade_array(self.grid, fade_location, fade_size) if fade_location is not None else None
        self.fade_active = tuple(fade_active)
        self.treadmill_dir = int(treadmill)
        self.treadmill_last = -1
        self.treadmill_history = []

    # imogen.m:30-42
    def set_state(self, mass, mom, ener, mag):
        shp = self.grid
        f = lambda v: np.array(v, dtype=float).reshape(shp)
        self.mass = FluidVar(self, 0, "mass", f(mass))
        self.ener = FluidVar(self, 0, "ener", f(ener))
        self.mom = [FluidVar(self, i + 1, "mom", f(mom[i])) for i in range(3)]
        self.mag = [MagComp(self, i + 1, f(mag[i])) for i in range(3)]
        for i in range(3):
            self.mag[i].isZero = (np.sum(self.mag[i].prim.a) == 0) and not self.magnet_active
        if self.fade_array is not None:   # FluidArray.readFades after the initial assignment (FluidArray.m:54)
            for name, vs in (("mass", [self.mass]), ("mom", self.mom), ("ener", [self.ener])):
                if name in self.fade_active:
                    for v in vs:
                        v.prim.fades = self.fade_array
        self.radiation_initialize()

    # ---------------------------------------------------------------------------------------
    # Radiation (fluid/Radiation.m) and ArtificialViscosity (fluid/ArtificialViscosity.m)
    def radiation_solve(self):
        """Radiation.solve: opticallyThinSolver (Radiation.m:86-88) or the empty solver (0)."""
        if self.rad_type != RAD_THIN:
            return 0.0
        gas, _ = self.pressure("gas", self.mass.prim.a, [m.prim.a for m in self.mom], self.ener.prim.a)
        return self.rad_strength * _lpow(self.mass.prim.a, 2 - self.rad_exponent) * _lpow(gas, self.rad_exponent)

    def radiation_initialize(self):
        """Radiation.initialize (Radiation.m:61-75), called by ImogenManager.initialize after the arrays
        are built (imogen.m:46): strength = initialMaximum/100 * min((E - KE - ME) / unscaled), with the
        kinetic energy from the momenta and the magnetic energy from the face-centred B."""
        if self.rad_type != RAD_THIN:
            self.rad_strength = 0.0
            return
        self.rad_strength = 1.0
        unscaled = self.radiation_solve()
        p = [m.prim.a for m in self.mom]
        b = [m.prim.a for m in self.mag]
        kinetic = 0.5 * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) / self.mass.prim.a
        magnetic = 0.5 * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2])
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = (self.ener.prim.a - kinetic - magnetic) / unscaled
        self.rad_strength = (self.rad_initial_maximum / 100) * float(np.nanmin(ratio))   # minFinderND

    def csw_sound_speed(self, mass, mom, ener, X):
        """ArtificialViscosity.cswSoundSpeed (ArtificialViscosity.m:157-190).  As written in the
        reference, only the z momentum of the velocity-squared sum is divided by rho^2."""
        G = self.GAMMA
        out = []
        for n in (1, -1):
            vel_sq = (mom[0].shift(X, n) ** 2 + mom[1].shift(X, n) ** 2
                      + mom[2].shift(X, n) ** 2 / mass.shift(X, n) ** 2)
            mag_sq = (self.mag[0].cellMag.shift(X, n) ** 2 + self.mag[1].cellMag.shift(X, n) ** 2
                      + self.mag[2].cellMag.shift(X, n) ** 2)
            s = (G - 1.0) * (ener.shift(X, n) - 0.5 * mass.shift(X, n) * vel_sq)
            s = s - (G - 1.0) * 0.5 * mag_sq
            with np.errstate(invalid="ignore"):
                s = np.sqrt(np.abs((G * s + 2.0 * mag_sq) / mass.shift(X, n)))
            out.append(s)
        snd_c, snd_b = out
        return np.fmax(np.fmin(snd_b, snd_c), 0)

    def viscosity_solve(self, mass, mom, ener, sound, X):
        """ArtificialViscosity.solve for the stage arrays (objects with .a and .shift)."""
        d = X - 1
        c1, c2 = self.visc_linear, self.visc_quadratic
        if self.visc_type == VISC_NR:   # ArtificialViscosity.m:73-77
            vm = np.fmin(mom[d].shift(X, 1) - mom[d].a, 0)
            return vm * (c1 * sound + c2 * vm / mass.a)
        if self.visc_type == VISC_CSW:  # ArtificialViscosity.m:81-148 (averaged densities)
            mass_b = mass.shift(X, -1)
            mass_c = mass.shift(X, 1)
            rho = 2 * mass_c * mass_b / (mass_c + mass_b)
            cs = self.csw_sound_speed(mass, mom, ener, X)
            v0 = mom[d].shift(X, -2) / mass.shift(X, -2)
            v1 = mom[d].shift(X, -1) / mass.shift(X, -1)
            v2 = mom[d].shift(X, 1) / mass.shift(X, 1)
            v3 = mom[d].shift(X, 2) / mass.shift(X, 2)
            dv = v2 - v1
            G = self.GAMMA
            with np.errstate(divide="ignore", invalid="ignore"):
                r_l = (v3 - v2) / (2 * dv)
                r_r = (v1 - v0) / (2 * dv)
                limiter = np.fmax(0, np.fmin(np.fmin(0.5 * (r_l + r_r), np.fmin(2 * r_l, 2 * r_r)), 1))
                return ((dv < 0) * rho * (c2 * (G + 1) * np.abs(dv) / 4
                                          + np.sqrt(c2 ** 2 * ((G + 1) / 4) ** 2 * dv ** 2 + c1 ** 2 * cs ** 2))
                        * (1 - limiter) * np.abs(dv))
        return 0.0

    def state(self):
        return dict(mass=self.mass.prim.a.copy(), ener=self.ener.prim.a.copy(),
                    mom=np.stack([m.prim.a for m in self.mom]),
                    mag=np.stack([m.prim.a for m in self.mag]),
                    cellmag=np.stack([m.cellMag.a for m in self.mag]))

    # ---------------------------------------------------------------------------------------
    def pressure(self, mode, mass, mom_arrays, ener):
        """pressure.m:16-66 (returns result, aux)."""
        G = self.GAMMA
        vel_sq = (mom_arrays[0] * mom_arrays[0] + mom_arrays[1] * mom_arrays[1]
                  + mom_arrays[2] * mom_arrays[2]) / (mass * mass)
        mag_sq = 0.0
        for i in range(3):
            if not self.mag[i].isZero:
                mag_sq = mag_sq + self.mag[i].cellMag.a * self.mag[i].cellMag.a
        result = (G - 1.0) * (ener - 0.5 * mass * vel_sq)
        aux = None
        if mode == "totsnd":
            with np.errstate(invalid="ignore"):
                aux = np.sqrt(np.abs((G * (result - (G - 1.0) * 0.5 * mag_sq) + 2.0 * mag_sq) / mass))
            result = result + 0.5 * (2.0 - G) * mag_sq
        elif mode == "sound":
            result = result - (G - 1.0) * 0.5 * mag_sq
            result = np.sqrt(np.abs((G * result + 2.0 * mag_sq) / mass))
        elif mode == "gas":
            result = result - (G - 1.0) * 0.5 * mag_sq
        elif mode == "total":
            result = result + 0.5 * (2.0 - G) * mag_sq
        elif mode == "magnetic":
            result = 0.5 * mag_sq * np.ones(self.grid)
        result = np.where(result < 0, 0.0, result)
        return result, aux

    def w_fluid_flux(self, objs, X):
        """wFluidFlux.m:14-44: freeze speed (per-pencil max, broadcast) and W arrays; objs are the
        stage's (mass, [mom x3], ener) array objects (primaries for the predictor, stores for the
        corrector)."""
        d = X - 1
        rho, mom, ener = objs[0].a, [m.a for m in objs[1]], objs[2].a
        press, sound = self.pressure("totsnd", rho, mom, ener)
        velocity = mom[d] / rho
        spd = np.nanmax(np.abs(velocity) + sound, axis=d, keepdims=True)
        freeze = np.broadcast_to(spd, rho.shape)
        press = press + self.viscosity_solve(objs[0], objs[1], objs[2], sound, X)   # wFluidFlux.m:24
        cm = [self.mag[i].cellMag.a for i in range(3)]
        w_mass = mom[d] / freeze
        w_ener = velocity * (ener + press) - cm[d] * (cm[0] * mom[0] + cm[1] * mom[1]
                                                       + cm[2] * mom[2]) / rho
        w_ener = w_ener / freeze
        w_mom = []
        for i in range(3):
            dirv = 1.0 if i == d else 0.0
            w_mom.append((velocity * mom[i] + press * dirv - cm[d] * cm[i]) / freeze)
        return freeze, [w_mass, w_mom[0], w_mom[1], w_mom[2], w_ener]

    def fluid_vars(self):
        return [self.mass, self.mom[0], self.mom[1], self.mom[2], self.ener]

    def relaxing_fluid(self, X):
        """relaxingFluid.m:16-73."""
        flux_factor = self.dTime / self.dgrid[X - 1]
        v = self.fluid_vars()
        freeze, w = self.w_fluid_flux((v[0].prim, [v[1].prim, v[2].prim, v[3].prim], v[4].prim), X)
        for i in range(5):
            vi = v[i]
            vi.store_fluxR.set(0.5 * (vi.prim.a + w[i]))
            vi.store_fluxL.set(0.5 * (vi.prim.a - w[i]))
            vi.store.set(vi.prim.a - 0.5 * flux_factor * freeze * (
                vi.store_fluxR.a - vi.store_fluxR.shift(X, -1)
                + vi.store_fluxL.a - vi.store_fluxL.shift(X, 1)))
            vi.store_fluxR.cleanup()
            vi.store_fluxL.cleanup()
        self.mass.store.set(np.fmax(self.mass.store.a, self.MINMASS))   # MATLAB max ignores NaN

        freeze, w = self.w_fluid_flux((v[0].store, [v[1].store, v[2].store, v[3].store], v[4].store), X)
        lim = LIMITERS[self.limiter[X - 1]]
        for i in range(5):
            vi = v[i]
            vi.fluxR.set(0.5 * (vi.store.a + w[i]))
            vi.fluxL.set(0.5 * (vi.store.a - w[i]))
            lim(vi.fluxR, vi.fluxR.a - vi.fluxR.shift(X, -1), vi.fluxR.shift(X, 1) - vi.fluxR.a)
            lim(vi.fluxL, vi.fluxL.shift(X, -1) - vi.fluxL.a, vi.fluxL.a - vi.fluxL.shift(X, 1))
            vi.prim.set(vi.prim.a - flux_factor * freeze * (
                vi.fluxR.a - vi.fluxR.shift(X, -1) + vi.fluxL.a - vi.fluxL.shift(X, 1)))
            vi.fluxR.cleanup()
            vi.fluxL.cleanup()
            vi.store.cleanup()
        self.mass.prim.set(np.fmax(self.mass.prim.a, self.MINMASS))

    # ---------------------------------------------------------------------------------------
    def magnet_flux(self, X, mag_indices):
        """magnetFlux.m:14-31."""
        I = None
        for I in mag_indices:
            m = self.mag[I - 1]
            vg = m.velGrid[X]
            momX = self.mom[X - 1].prim
            mass = self.mass.prim
            vg.set((momX.shift(I, -1) + momX.a) / (mass.shift(I, -1) + mass.a))
            vg.set(0.25 * (vg.shift(X, -1) + vg.shift(X, 1) + 2 * vg.a))
            self.relaxing_magnet(X, I, vg)
            for tab in (m.velGrid, m.store, m.store_fluxR, m.wMag, m.flux):
                tab[X].cleanup()
        self.mag[I - 1].update_cell_centered()
        self.mag[X - 1].update_cell_centered()

    def relaxing_magnet(self, X, I, velGrid):
        """relaxingMagnet.m:15-60."""
        m = self.mag[I - 1]
        flux_factor = 0.5 * self.dTime / self.dgrid[X - 1]
        vflow = ((velGrid.a + velGrid.shift(X, 1)) < 0.0).astype(float)

        sfr = m.store_fluxR[X]
        sfr.set(m.prim.a * velGrid.a)
        sfr.set(sfr.a * (1 - vflow) + sfr.shift(X, 1) * vflow)
        m.store[X].set(m.prim.a - flux_factor * (sfr.a - sfr.shift(X, -1)))

        flux_factor = 2 * flux_factor
        wm = m.wMag[X]
        wm.set(m.store[X].a * velGrid.a)
        fx = m.flux[X]
        fx.set(wm.a * (1 - vflow) + wm.shift(X, 1) * vflow)
        dFluxR = wm.shift(X, 1) - (vflow * wm.shift(X, 2) + (1 - vflow) * wm.a)
        dFluxL = wm.a - (vflow * wm.shift(X, 1) + (1 - vflow) * wm.shift(X, -1))
        LIMITERS[self.limiter[X - 1]](fx, dFluxL, dFluxR)
        m.prim.set(m.prim.a - flux_factor * (fx.a - fx.shift(X, -1)))

        flux_factor = self.dTime / self.dgrid[I - 1]
        fx.set(fx.a - fx.shift(I, 1))
        fx.set(fx.shift(X, -1))
        bx = self.mag[X - 1].prim
        bx.set(bx.a - flux_factor * fx.a)

    # ---------------------------------------------------------------------------------------
    def flux(self, order):
        """flux.m:17-62."""
        row = (self.iteration - 1) % 6
        if order == 1:
            dirs = FORWARD_ORDER[row]
            for X in dirs:
                if self.grid[X - 1] < 3:
                    continue
                if self.fluid_active:
                    self.relaxing_fluid(X)
                if self.magnet_active:
                    self.magnet_flux(X, FORWARD_MAGIDX[X])
        elif order == -1:
            dirs = BACKWARD_ORDER[row]
            for X in dirs:
                if self.grid[X - 1] < 3:
                    continue
                if self.magnet_active:
                    self.magnet_flux(X, BACKWARD_MAGIDX[X])
                if self.fluid_active:
                    self.relaxing_fluid(X)
        else:
            raise ValueError(f"{order} is not a recognized direction")

    def time_update(self, flux_direction):
        """TimeManager.update (TimeManager.m:55-99)."""
        if flux_direction > 1 and self.updateMode != PER_STEP:
            return
        cmax = 1e-2
        grid_index = 0
        sound, _ = self.pressure("sound", self.mass.prim.a,
                                 [m.prim.a for m in self.mom], self.ener.prim.a)
        for i in range(3):
            c = np.nanmax(np.abs(self.mom[i].prim.a / self.mass.prim.a) + sound)
            if c > cmax:
                cmax = c
                grid_index = i + 1
        if grid_index < 1:
            raise FloatingPointError(f"CFL error: cmax={cmax}")
        self.dTime = self.CFL * self.MINDGRID[grid_index - 1] / cmax
        new_time = self.time + (self.updateMode + 1) * self.dTime
        if new_time > self.TIMEMAX:
            self.dTime = (self.TIMEMAX - self.time) / (self.updateMode + 1)
            new_time = self.TIMEMAX
        self.time = new_time
        self.history.append(self.dTime)
        self.last_cfl = (cmax, grid_index)

    @property
    def running(self):
        return self.iteration <= self.ITERMAX and self.time < self.TIMEMAX

    def treadmill(self):
        """treadmillGrid (treadmill/treadmillGrid.m:14-37): after iteration 10, the mean over the
        pencils along DIRECTION of the (first) index of the largest forward difference of rho picks
        newIndex; the first call only records it as `last`, later calls shift every primary array
        by newIndex - last cells with its own boundary conditions."""
        X = self.treadmill_dir
        if X <= 0 or self.iteration < 10:
            return
        d = X - 1
        deriv = (self.mass.prim.shift(X, 1) - self.mass.prim.a) / self.dgrid[d]   # calculate2PtDerivative
        deriv = np.where(np.isnan(deriv), -np.inf, deriv)                         # max ignores NaN
        idx = np.argmax(deriv, axis=d).astype(float) + 1                           # first maximum, 1-based
        new_index = _matlab_round(_mean_of_means(idx))
        if self.treadmill_last < 0:
            self.treadmill_last = new_index
            return
        dc = new_index - self.treadmill_last
        self.mass.prim.set(self.mass.prim.shift(X, dc))
        self.ener.prim.set(self.ener.prim.shift(X, dc))
        for i in range(3):
            self.mom[i].prim.set(self.mom[i].prim.shift(X, dc))
            self.mag[i].prim.set(self.mag[i].prim.shift(X, dc))
        self.treadmill_history.append(dc)

    def source(self):
        """source.m:30: ener.array = ener.array - dTime * radiation.solve (the empty solver gives 0;
        gravity is not part of this path)."""
        if self.rad_type == RAD_THIN:
            self.ener.prim.set(self.ener.prim.a - self.dTime * self.radiation_solve())

    def iterate(self):
        """One pass of the imogen.m:58-72 loop body (two timesteps)."""
        for i, direction in ((1, 1), (2, -1)):
            self.time_update(i)
            self.flux(direction)
            self.treadmill()
            self.source()
        self.iteration += 1

    def run(self, max_iterations=None):
        n = 0
        while self.running and (max_iterations is None or n < max_iterations):
            self.iterate()
            n += 1
        return n
