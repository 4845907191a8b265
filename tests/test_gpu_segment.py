"""The segment fluid kernel (each thread owns consecutive cells; seg_fluid.cuh) against the pencil-tile
kernels (GPU required).  Every cell goes through the same formulas in the same order; the compiler may
contract them into FMAs differently in the two kernels, so runs agree to round-off: relative L1 at most
1e-13 in FP64 and 1e-6 in the mixed form after 6 iterations, max |difference| a few ulp of the values.
IMOGEN_B200_TILE_KERNELS=1 at creation gives a context that uses the tile kernels for every fluid
sweep.  Within one kernel family results are bitwise reproducible: a batch equals its members alone."""
import numpy as np
import pytest

from imogen_b200 import ImogenBatch, ImogenRun, problems
from tests.parity import smooth_state

pytestmark = pytest.mark.gpu


def _segment_tiling(n, d):
    """A segment fluid tiling for a pencil of n cells along dim d (the rules of the kernel's candidates)."""
    for C in (4, 2):
        if n % C:
            continue
        S = n // C
        if d == 1 and not (S % 32 == 0 or (S <= 32 and 32 % S == 0)):
            continue
        for Wb in ((1, 2, 4, 8) if d == 1 else (8, 16, 32, 4)):
            NT = Wb * S
            if 64 <= NT <= 512 and NT % 32 == 0:
                return (Wb, S, 1, NT, C, 1, 1)
    return None


def _run(settings, state, precision, tile, monkeypatch, iters=6):
    if tile:
        monkeypatch.setenv("IMOGEN_B200_TILE_KERNELS", "1")
    else:
        monkeypatch.delenv("IMOGEN_B200_TILE_KERNELS", raising=False)
    r = ImogenRun(precision=precision, **settings)
    if not tile and precision == "fp64":   # the FP64 default is the tile kernel: pick segment tilings
        for d, n in enumerate(settings["grid"], 1):
            t = _segment_tiling(n, d) if n >= 3 else None
            if t:
                r.set_tiling(d, t)
    r.set_state(*state)
    r.run(iters)
    return r


CASES = [
    ((64, 48, 1), "circ", True), ((64, 48, 1), "const", True), ((32, 32, 32), "circ", True),
    ((256, 1, 1), "const", False), ((128, 16, 8), "circ", False), ((64, 24, 20), "const", True),
]


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("grid,bc,mhd", CASES)
def test_segment_kernel_equals_tile_kernels(grid, bc, mhd, precision, monkeypatch):
    s = dict(grid=grid, dgrid=(1.0 / max(grid),) * 3, gamma=5 / 3, cfl=0.35, bc=bc,
             limiter=("vanleer", "minmod", "superbee"), magnet=mhd, time_max=1e5, iter_max=10 ** 6)
    st = smooth_state(grid, seed=4, mhd=mhd)
    a = _run(s, st, precision, False, monkeypatch)
    b = _run(s, st, precision, True, monkeypatch)
    segs = [d for d, t in a.tiling("fluid").items() if t[6] and grid[d - 1] >= 3]
    assert segs, a.tiling("fluid")                   # the case exercises the segment kernel
    assert not any(t[6] for t in b.tiling("fluid").values())
    sa, sb = a.state(), b.state()
    tol = 1e-13 if precision == "fp64" else 1e-6
    for k in sa:
        rel = float(np.abs(sa[k] - sb[k]).sum() / max(np.abs(sb[k]).sum(), 1e-300))
        assert rel <= tol, (k, rel)
    assert abs(a.time.time - b.time.time) <= tol * b.time.time
    a.close()
    b.close()


def test_segment_kernel_in_a_batch(monkeypatch):
    monkeypatch.delenv("IMOGEN_B200_TILE_KERNELS", raising=False)
    cases = [problems.orszag_tang(n) for n in (64, 128, 64)]
    alone, together = [], []
    for s, st in cases:
        for lst in (alone, together):
            r = ImogenRun(precision="mixed", **dict(s, time_max=1e5, iter_max=10 ** 6))
            r.set_state(*st)
            lst.append(r)
    b = ImogenBatch(together)
    for _ in range(8):
        b.step()
        for r in alone:
            r.iterate()
    for r in alone:
        r.sync()
    for x, y in zip(alone, together):
        sx, sy = x.state(), y.state()
        for k in sx:
            assert np.array_equal(sx[k], sy[k]), k
    b.close()
    for r in alone + together:
        r.close()
