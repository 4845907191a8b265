"""Pencils of a few cells held whole by one thread (GPU required): the segment fluid kernel and the
window magnet kernels with one segment per pencil (S = 1, C = N cells per thread, many pencils side by
side) take the y and z sweeps of N x 3 x 3 tubes and other grids with 3- or 4-cell dimensions.

Against the C++ oracle, relative L1 per variable: FP64 1e-11 after 10 iterations (the first iteration
captures stored edges on the tile kernels, the later ones run these), the mixed form 2e-5.
"""
import numpy as np
import pytest

from imogen_b200 import ImogenRun
from tests.parity import errors, make_pair

pytestmark = pytest.mark.gpu

GRIDS = [(40, 3, 3), (36, 4, 3), (28, 3, 4)]


def _settings(grid, bc):
    n = grid[0]
    return dict(grid=grid, dgrid=(1.0 / n,) * 3, gamma=2.0, cfl=0.35, bc={"x": "const", "y": bc, "z": bc},
                limiter=("vanleer", "minmod", "superbee"), magnet=True, time_max=1e5, iter_max=10 ** 6)


def _tube(grid, seed):
    """A Brio-Wu-type tube (the batched ensemble's members) with seeded transverse perturbations of
    rho, the transverse momenta and B_z, so that the y and z sweeps move something."""
    rng = np.random.default_rng(seed)
    x = (np.arange(grid[0]) + 0.5)[:, None, None] / grid[0] * np.ones(grid)
    left = x < 0.5
    rho = np.where(left, 1.0, 0.125) * (1 + 0.02 * rng.random(grid))
    P = np.where(left, 1.0, 0.1)
    mom = np.zeros((3,) + grid)
    mom[1:] = 0.02 * (rng.random((2,) + grid) - 0.5) * rho
    mag = np.stack([np.full(grid, 0.75), np.where(left, 1.0, -1.0), 0.02 * (rng.random(grid) - 0.5)])
    ener = P / (2.0 - 1) + 0.5 * (mom ** 2).sum(0) / rho + 0.5 * (mag ** 2).sum(0)
    return rho, mom, ener, mag


def _assert_close(o, g, tol, what):
    e = errors(g.state(), o.state())
    bad = {k: v for k, v in e.items() if not (v <= tol)}
    assert not bad, f"{what}: relative L1 above {tol}: {bad}"


def _one_thread_pencils(run, kind, dims):
    t = run.tiling(kind)
    for d in dims:
        wb, g, cl, nt, cpt, nqc, seg = t[d]
        assert (g, cl, cpt, seg) == (1, 1, run.grid[d - 1], 1) and wb == nt, (kind, d, t[d])


@pytest.mark.parametrize("bc", ["circ", "const"])
@pytest.mark.parametrize("grid", GRIDS)
def test_short_pencils_mixed_default(grid, bc):
    s = _settings(grid, bc)
    o, g = make_pair(s, _tube(grid, 5), precision="mixed")
    short = [d for d in (2, 3) if grid[d - 1] in (3, 4)]
    _one_thread_pencils(g, "fluid", short)
    _one_thread_pencils(g, "magnet", short)
    o.run(10)
    g.run(10)
    _assert_close(o, g, 2e-5, f"mixed {grid} {bc}")
    g.close()


@pytest.mark.parametrize("bc", ["circ", "const"])
@pytest.mark.parametrize("grid", GRIDS)
def test_short_pencils_fp64(grid, bc):
    s = _settings(grid, bc)
    o, g = make_pair(s, _tube(grid, 6))
    # FP64 fluid sweeps default to the tile kernels: ask for the one-thread segment tiling
    for d in (2, 3):
        n = grid[d - 1]
        g.set_tiling(d, (64, 1, 1, 64, n, 1, 1))
    _one_thread_pencils(g, "fluid", (2, 3))
    _one_thread_pencils(g, "magnet", (2, 3))
    o.run(10)
    g.run(10)
    assert abs(g.time.time - o.time) <= 1e-12 * max(1.0, o.time)
    _assert_close(o, g, 1e-11, f"fp64 {grid} {bc}")
    g.close()


def test_short_pencils_and_tile_kernels_agree():
    """The same mixed run on the one-thread tilings and on the pencil-tile kernels: round-off apart."""
    grid = (48, 3, 3)
    st = _tube(grid, 7)
    a = ImogenRun(precision="mixed", **_settings(grid, "circ"))
    a.set_state(*st)
    b = ImogenRun(precision="mixed", **_settings(grid, "circ"))
    b.set_state(*st)
    for d in (2, 3):   # along y and z the pencil-tile kernels instead
        b.set_tiling(d, (128, 4, 1, 512, 1, 1, 0))
        b.set_tiling(d, (128, 4, 1, 512, 1, 1, 0), kind="magnet")
    assert b.tiling("fluid")[2][6] == 0 and b.tiling("magnet")[2][6] == 0, (b.tiling("fluid"), b.tiling("magnet"))
    a.run(20)
    b.run(20)
    e = errors(a.state(), b.state())
    assert max(e.values()) < 1e-5, e
    a.close()
    b.close()
