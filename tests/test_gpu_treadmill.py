"""treadmillGrid (treadmill/treadmillGrid.m) on the GPU against the C++ oracle (GPU required).

From iteration 10 on, after each flux, the grid is shifted along the treadmill direction so that the
steepest density rise stays where it was first seen; the shift of every primary array uses that
array's own boundary conditions (any shift distance).  The shift decisions (TreadmillManager.history
and .last) must match the oracle's exactly, and the state to 1e-12 (FP64, relative L1 of rho and E,
and of momentum and B as vectors).
"""
import numpy as np
import pytest

from imogen_b200 import ImogenBatch, ImogenError, ImogenRun
from tests.parity import errors_vector, make_pair, smooth_state
from tests.test_oracle import _shock_tube

pytestmark = pytest.mark.gpu


def _settings(grid, bc, treadmill=1, **kw):
    s = dict(grid=grid, dgrid=tuple(1 / g for g in grid), cfl=0.35, bc=bc, magnet=True, time_max=1e5,
             iter_max=10 ** 6, treadmill=treadmill)
    s.update(kw)
    return s


def _check(o, g, tol, what):
    # momentum and B as vectors: after a long const shift the transverse momentum is round-off (1e-12
    # of the total), and a per-component ratio of such sums says nothing
    e = errors_vector(g.state(), o.state())
    bad = {k: v for k, v in e.items() if not (v <= tol)}
    assert not bad, f"{what}: relative L1 above {tol}: {bad}"


@pytest.mark.parametrize("bc", ["fade", "circ", "const", "trans", "wall", "mirror", "flip"])
def test_treadmill_follows_the_shock_like_the_oracle(bc):
    grid = (40, 6, 1)
    s = _settings(grid, {"x": bc, "y": "circ", "z": "circ"})
    o, g = make_pair(s, _shock_tube(grid))
    for it in range(25):
        o.iterate()
        g.iterate()
    hist, last = g.treadmill_history
    assert (hist, last) == (o.treadmill_history, o.treadmill_last)
    _check(o, g, 1e-12, f"treadmill along x with {bc} ends after 25 iterations")
    g.close()


def test_treadmill_along_y_in_3d():
    grid = (6, 48, 8)
    rho, mom, ener, mag = _shock_tube((48, 6, 8))
    swap = lambda a: np.swapaxes(a, 0, 1)                   # the tube along y
    state = (swap(rho), np.stack([swap(mom[1]), swap(mom[0]), swap(mom[2])]), swap(ener),
             np.stack([swap(mag[1]), swap(mag[0]), swap(mag[2])]))
    s = _settings(grid, {"x": "circ", "y": "const", "z": "circ"}, treadmill=2)
    o, g = make_pair(s, state)
    o.run(20)
    g.run(20)
    assert g.treadmill_history == (o.treadmill_history, o.treadmill_last)
    _check(o, g, 1e-12, "treadmill along y, 3-D")
    g.close()


def test_treadmill_mixed_form_takes_the_same_decisions():
    grid = (40, 6, 1)
    s = _settings(grid, {"x": "fade", "y": "circ", "z": "circ"})
    o, g = make_pair(s, _shock_tube(grid), precision="mixed")
    o.run(25)
    g.run(25)
    assert g.treadmill_history == (o.treadmill_history, o.treadmill_last)
    _check(o, g, 2e-5, "treadmill, mixed form")
    g.close()


def test_step_by_step_treadmill_call():
    """time.update, flux, treadmillGrid one at a time (imogen.m:62-64) from iteration 10."""
    grid = (40, 6, 1)
    s = _settings(grid, {"x": "const", "y": "circ", "z": "circ"})
    o, g = make_pair(s, _shock_tube(grid))
    o.run(12)
    g.run(12)
    for i, order in ((1, 1), (2, -1)):
        o.time_update(i)
        g.time.update(i, sync=True)
        o.flux(order)
        g.flux(order)
        o.treadmill()
        g.treadmill()
        _check(o, g, 1e-12, f"after treadmillGrid of timestep {i}")
    assert g.treadmill_history == (o.treadmill_history, o.treadmill_last)
    g.close()


def test_treadmill_contexts_do_not_join_batches():
    grid = (40, 6, 1)
    r = ImogenRun(**_settings(grid, {"x": "const", "y": "circ", "z": "circ"}))
    r.set_state(*smooth_state(grid, seed=1, mhd=True))
    with pytest.raises(ImogenError):
        ImogenBatch([r])
    r.close()
