"""The oracle itself: pinned against SciPy's pchip, the documented perms order, an exact Riemann
solution, and the conservation / div B invariants; the NumPy and C++ restatements must agree bit
for bit (CPU only)."""
import itertools

import numpy as np
import pytest

from imogen_b200 import problems
from oracle import cpp_oracle, np_oracle
from tests.parity import smooth_state
from tests.riemann import sample


def test_pchip_matches_scipy():
    from scipy.interpolate import PchipInterpolator
    rng = np.random.default_rng(0)
    for inf in (5, 20, 37):
        x = np.array([1, 2, 3, inf, inf + 1], float)
        for _ in range(200):
            y = rng.standard_normal(5) * 10 ** rng.uniform(-6, 3)
            if rng.random() < 0.3:
                y[3] = y[4]          # the shape transparent_shift.m feeds (edge repeated)
            xi = np.array([4.0, 5.0])
            ref = PchipInterpolator(x, y)(xi)
            a = np_oracle.pchip(x, y, xi)
            b = cpp_oracle.pchip(x, y, xi)[0]
            assert np.allclose(a, ref, rtol=1e-12, atol=1e-14 * np.abs(y).max())
            assert np.array_equal(a, b)


def test_fade_coefficients_match_scipy():
    from scipy.interpolate import PchipInterpolator
    for f in (20, 24, 31):
        ref = PchipInterpolator([0, np.ceil(f / 4), np.floor(f / 2 + 0.5), f - 1, f],
                                [1, 1, 0.01, 0, 0])(np.arange(1, f + 1))
        assert np.allclose(np_oracle.fade_coefficients(f), ref, rtol=1e-12, atol=1e-15)


def test_perms_order():
    # MATLAB perms returns rows in reverse lexicographic order (flux.m:19,25)
    assert np_oracle.FORWARD_ORDER == tuple(sorted(itertools.permutations((1, 2, 3)), reverse=True))
    assert all(b == tuple(reversed(f)) for f, b in zip(np_oracle.FORWARD_ORDER, np_oracle.BACKWARD_ORDER))


@pytest.mark.parametrize("bc", ["circ", "const", "mirror", "trans", "wall", "fade"])
@pytest.mark.parametrize("grid,mhd", [((30, 1, 1), False), ((24, 22, 1), True), ((21, 20, 20), True)])
def test_numpy_and_cpp_oracles_bitwise(bc, grid, mhd):
    spec = {f: (bc if not ((bc == "mirror" and grid[d] < 2) or (bc == "fade" and grid[d] < 20)) else "circ")
            for d, f in enumerate("xyz")}
    s = dict(grid=grid, dgrid=tuple(1 / g for g in grid), gamma=5 / 3, cfl=0.35, bc=spec,
             limiter=("vanleer", "minmod", "superbee"), magnet=mhd, iter_max=3)
    kw = problems.oracle_kwargs(s)
    st = smooth_state(grid, seed=5, mhd=mhd)
    a = np_oracle.Sim(**kw)
    a.set_state(*st)
    b = cpp_oracle.Sim(**kw)
    b.set_state(*st)
    a.run()
    b.run()
    sa, sb = a.state(), b.state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
    assert a.time == b.time


def test_conservation_and_divb_periodic():
    grid = (32, 24, 1)
    s = dict(grid=grid, dgrid=(1 / 32, 1 / 24, 1.0), gamma=5 / 3, cfl=0.35, bc="circ", magnet=True, iter_max=20)
    st = smooth_state(grid, seed=7, mhd=False)
    nx, ny = 32, 24
    rng = np.random.default_rng(1)
    Az = 0.05 * rng.standard_normal((nx, ny))          # corner vector potential -> div-free faces
    mag = np.zeros((3, nx, ny, 1))
    mag[0, :, :, 0] = (np.roll(Az, -1, 1) - Az) * ny
    mag[1, :, :, 0] = -(np.roll(Az, -1, 0) - Az) * nx
    o = cpp_oracle.Sim(**problems.oracle_kwargs(s))
    o.set_state(st[0], st[1], st[2] + 0.5 * (mag ** 2).sum(0), mag)
    s0 = o.state()
    o.run()
    s1 = o.state()
    for k in ("mass", "ener"):
        assert abs(s1[k].sum() - s0[k].sum()) <= 1e-12 * abs(s0[k]).sum()
    for c in range(3):
        assert abs(s1["mom"][c].sum() - s0["mom"][c].sum()) <= 1e-12 * abs(s0["mom"]).sum()
    div = lambda b: (np.roll(b[0], -1, 0) - b[0]) * nx + (np.roll(b[1], -1, 1) - b[1]) * ny
    assert np.abs(div(s1["mag"])).max() <= 1e-11 * np.abs(s1["mag"]).max() * nx


def test_sod_against_exact_riemann_solution():
    s, st = problems.sod(400, time_max=0.2)
    o = cpp_oracle.Sim(**problems.oracle_kwargs(s))
    o.set_state(*st)
    o.run()
    assert o.time == pytest.approx(0.2, abs=1e-15)
    rho = o.state()["mass"][:, 0, 0]
    x = (np.arange(400) + 0.5) / 400
    ex = sample(x, 0.2, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 5 / 3)
    l1 = np.abs(rho - ex[0]).mean()
    assert l1 < 6e-3, l1            # first order at discontinuities on 400 cells


def test_bc_validation_matches_reference_index_errors():
    with pytest.raises(ValueError):
        np_oracle.Sim((32, 1, 1), (1, 1, 1), bc="mirror")
    with pytest.raises(ValueError):
        cpp_oracle.Sim((32, 1, 1), (1, 1, 1), bc="mirror")
    with pytest.raises(ValueError):
        np_oracle.Sim((19, 32, 1), (1, 1, 1), bc="fade")
