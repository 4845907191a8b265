"""A point fade (classes/PointFade.m via ImogenManager.addFades) on the GPU against the C++ oracle (GPU
required).

Every assignment to a primary in the fade's active list multiplies it by 1 - 0.05 A (A the PointFade map):
the sweeps' updates and relaxingFluid's MINMASS clamp, the radiation sink, the treadmill's shift, and host
assignments (img_upload); the initial arrays are not faded.  Tolerances as for the other FP64 parity tests
(relative L1 per variable): 1e-12 after single sweeps, 1e-10 after 100 iterations; mixed form 2e-5.
"""
import numpy as np
import pytest

from imogen_b200 import ImogenBatch, ImogenError, ImogenRun
from tests.parity import errors, errors_vector, make_pair, smooth_state
from tests.test_oracle import _shock_tube

pytestmark = pytest.mark.gpu


def _settings(grid, bc="circ", active=("mass", "mom", "ener"), **kw):
    s = dict(grid=grid, dgrid=tuple(1 / g for g in grid), cfl=0.35, bc=bc, magnet=True, time_max=1e5,
             iter_max=10 ** 6, fade_location=(grid[0] // 2, grid[1] // 3, max(1, grid[2] // 2)), fade_size=3.0,
             fade_active=active)
    s.update(kw)
    return s


def _check(o, g, tol, what, vector=False):
    e = (errors_vector if vector else errors)(g.state(), o.state())
    bad = {k: v for k, v in e.items() if not (v <= tol)}
    assert not bad, f"{what}: relative L1 above {tol}: {bad}"


@pytest.mark.parametrize("grid,bc", [((48, 40, 1), "circ"), ((48, 40, 1), "trans"), ((20, 18, 16), "const")])
def test_fade_single_sweeps(grid, bc):
    o, g = make_pair(_settings(grid, bc), smooth_state(grid, seed=3, mhd=True))
    o.time_update(1)
    g.time.update(1, sync=True)
    mi = {1: (2, 3), 2: (1, 3), 3: (1, 2)}
    for X in (1, 2, 3):
        if grid[X - 1] < 3:
            continue
        o.relaxing_fluid(X)
        g.relaxing_fluid(X)
        _check(o, g, 1e-12, f"{bc} {grid} after the fluid sweep along {X}")
        o.magnet_flux(X, mi[X])
        g.magnet_flux(X, mi[X])
        _check(o, g, 1e-12, f"{bc} {grid} after the magnet sweep along {X}")
    g.close()


@pytest.mark.parametrize("active", [("mass", "mom", "ener"), ("mass",), ("mom", "ener", "mag")])
def test_fade_100_iterations(active):
    grid = (48, 40, 1)
    st = smooth_state(grid, seed=4, mhd=True)
    o, g = make_pair(_settings(grid, active=active), st)
    assert o.run(100) == 100 and g.run(100) == 100
    _check(o, g, 1e-10, f"fade {active} after 100 iterations")
    plain = ImogenRun(**_settings(grid, active=()))
    plain.set_state(*st)
    plain.run(100)
    d = errors(g.state(), plain.state())
    assert max(d.values()) > 1e-6, d                                   # the fade acts
    g.close()
    plain.close()


def test_fade_with_radiation_and_mixed_form():
    grid = (48, 40, 1)
    s = _settings(grid, radiation="optically_thin", rad_initial_maximum=0.1)
    for precision, tol in (("fp64", 1e-10), ("mixed", 2e-5)):
        o, g = make_pair(s, smooth_state(grid, seed=5, mhd=True), precision=precision)
        o.run(50)
        g.run(50)
        _check(o, g, tol, f"fade + radiation, {precision}")
        g.close()


def test_fade_with_treadmill():
    grid = (40, 6, 1)
    s = _settings(grid, {"x": "fade", "y": "circ", "z": "circ"}, active=("mass", "ener"), treadmill=1)
    o, g = make_pair(s, _shock_tube(grid))
    o.run(20)
    g.run(20)
    assert g.treadmill_history == (o.treadmill_history, o.treadmill_last)
    _check(o, g, 1e-12, "fade + treadmill", vector=True)
    g.close()


def test_host_assignment_is_faded_and_the_initial_state_is_not():
    grid = (32, 24, 1)
    st = smooth_state(grid, seed=6, mhd=True)
    r = ImogenRun(**_settings(grid, active=("mass", "ener")))
    r.set_state(*st)
    assert np.array_equal(r.download("mass"), np.asarray(st[0], dtype=float))
    from oracle import np_oracle
    A = np_oracle.point_fade_array(grid, (grid[0] // 2, grid[1] // 3, 1), 3.0)   # the oracle's map
    r.upload("mass", st[0])
    r.upload("momx", st[1][0])                                         # mom is not in the list
    want = 0.95 * st[0] * A + st[0] * (1 - A)
    assert np.abs(r.download("mass") - want).max() <= 1e-15 * np.abs(want).max()
    assert np.array_equal(r.download("momx"), np.asarray(st[1][0], dtype=float))
    r.close()


def test_fade_contexts_do_not_join_batches():
    grid = (32, 24, 1)
    r = ImogenRun(**_settings(grid))
    r.set_state(*smooth_state(grid, seed=1, mhd=True))
    with pytest.raises(ImogenError):
        ImogenBatch([r])
    r.close()
