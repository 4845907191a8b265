"""Segment fluid and window magnet kernels along x for pencils of any length (GPU required): a length
that is not a multiple of the cells per thread leaves the last segment ragged and the threads past it
idle, and a pencil of more segments than one CTA holds spans the CTAs of a thread-block cluster (the
fluid kernel exchanges segment ends and pencil maxima through DSMEM; the window kernels need only the
cluster barrier between reads and in-place writes).

Against the C++ oracle, relative L1 per variable: FP64 1e-11 after 4 to 6 iterations, the mixed form
2e-5.
"""
import numpy as np
import pytest

from imogen_b200 import problems
from tests.parity import errors, make_pair, smooth_state

pytestmark = pytest.mark.gpu


def _assert_close(o, g, tol, what):
    e = errors(g.state(), o.state())
    bad = {k: v for k, v in e.items() if not (v <= tol)}
    assert not bad, f"{what}: relative L1 above {tol}: {bad}"


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 2e-5)])
@pytest.mark.parametrize("n", [1001, 2998, 5003])
def test_window_magnet_on_ragged_and_cluster_pencils(n, precision, tol):
    s, st = problems.brio_wu_tube(n, 1.0, 0.125, 1.0, 0.1)
    s = dict(s, iter_max=6, time_max=1e5)
    o, g = make_pair(s, st, precision=precision)
    kinds = ("magnet", "fluid") if precision == "mixed" else ("magnet",)   # FP64 fluid: the tile kernels
    for kind in kinds:
        wb, S, cl, nt, cpt, nqc, seg = g.tiling(kind)[1]
        assert seg == 1 and S == -(-n // cpt) and cl * nt >= S, (kind, g.tiling(kind))
        if n > 4 * 512:
            assert cl > 1, (kind, g.tiling(kind))
    o.run()
    g.run()
    _assert_close(o, g, tol, f"brio-wu {n} x 3 x 3 {precision}")
    g.close()


@pytest.mark.parametrize("tiling", [(1, 1251, 5, 256, 4, 1, 1), (1, 1251, 3, 448, 4, 1, 1), (1, 626, 3, 224, 8, 1, 1)])
def test_window_cluster_tilings_agree(tiling):
    """Every cluster split of one 5003-cell pencil gives the oracle's result."""
    s, st = problems.brio_wu_tube(5003, 1.0, 0.125, 1.0, 0.1)
    s = dict(s, iter_max=4, time_max=1e5)
    o, g = make_pair(s, st)
    g.set_tiling(1, tiling, kind="magnet")
    o.run()
    g.run()
    _assert_close(o, g, 1e-11, f"tiling {tiling}")
    g.close()


@pytest.mark.parametrize("n,tiling", [(5003, (1, 1251, 5, 256, 4, 1, 1)), (2998, (1, 750, 3, 256, 4, 1, 1)),
                                      (1001, (1, 251, 1, 256, 4, 1, 1)), (1001, (1, 501, 2, 256, 2, 1, 1))])
def test_segment_fluid_cluster_tilings_fp64(n, tiling):
    """The cluster forms of the segment fluid kernel in FP64 (whole pencil per CTA with a ragged end, or
    over 2 to 5 CTAs; FP64 CTAs of more than 256 threads exceed the shared-memory limit), each against
    the oracle."""
    s, st = problems.brio_wu_tube(n, 1.0, 0.125, 1.0, 0.1)
    s = dict(s, iter_max=4, time_max=1e5)
    o, g = make_pair(s, st)
    g.set_tiling(1, tiling)
    o.run()
    g.run()
    _assert_close(o, g, 1e-11, f"fluid tiling {tiling}")
    g.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 2e-5)])
def test_segment_fluid_cluster_periodic(precision, tol):
    """A periodic x pencil over a 5-CTA cluster: the first segment's left neighbour and the last one's
    right neighbour live in other ranks' shared memory."""
    grid = (4800, 3, 3)
    s = dict(grid=grid, dgrid=(1.0 / 4800,) * 3, gamma=5 / 3, cfl=0.35, bc="circ", limiter="vanleer",
             magnet=True, time_max=1e5, iter_max=5)
    o, g = make_pair(s, smooth_state(grid, seed=11, mhd=True), precision=precision)
    g.set_tiling(1, (1, 1200, 5, 256, 4, 1, 1))
    o.run()
    g.run()
    _assert_close(o, g, tol, f"periodic 4800 {precision}")
    g.close()


def _wavy_tube(n, width=3):
    """An MHD tube with no uniform stretch anywhere (the const ends see every stage's own end value)."""
    x = (np.arange(n) + 0.5)[:, None, None] / n * np.ones((n, width, width))
    rho = 1 + 0.2 * np.sin(6 * np.pi * x + 0.3)
    P = 1 + 0.1 * np.cos(4 * np.pi * x)
    mom = np.stack([0.1 * np.sin(2 * np.pi * x), 0.05 * np.cos(2 * np.pi * x), 0 * x]) * rho
    mag = np.stack([np.full(x.shape, 0.75), 0.5 + 0.1 * np.cos(2 * np.pi * x), 0.05 * np.sin(4 * np.pi * x)])
    ener = P / (5 / 3 - 1) + 0.5 * (mom ** 2).sum(0) / rho + 0.5 * (mag ** 2).sum(0)
    return rho, mom, ener, mag


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 2e-5)])
@pytest.mark.parametrize("n", [22, 1001, 2998])
def test_ragged_const_ends_on_a_wavy_tube(n, precision, tol):
    """Ragged last segments next to const ends, where the end cells' stage values differ from their
    neighbours' (22 cells: windows of 6 segments, 32 pencils per CTA; 1001 and 2998: the segment fluid
    kernel's cluster forms too, chosen for the mixed form and set for FP64)."""
    grid = (n, 3, 3)
    s = dict(grid=grid, dgrid=(1.0 / n,) * 3, gamma=5 / 3, cfl=0.35, bc={"x": "const", "y": "circ", "z": "circ"},
             limiter=("vanleer", "minmod", "superbee"), magnet=True, time_max=1e5, iter_max=6)
    o, g = make_pair(s, _wavy_tube(n), precision=precision)
    if n > 64:
        if precision == "fp64":
            g.set_tiling(1, (1, -(-n // 4), -(-n // 1024), 256, 4, 1, 1))
        assert g.tiling("fluid")[1][6] == 1 and g.tiling("fluid")[1][1] == -(-n // 4), g.tiling("fluid")
    assert g.tiling("magnet")[1][6] == 1 and n % g.tiling("magnet")[1][4] != 0, g.tiling("magnet")
    o.run()
    g.run()
    _assert_close(o, g, tol, f"wavy tube {n} {precision}")
    g.close()


@pytest.mark.parametrize("tiling", [(1, 32, 1, 32, 2, 1, 1), (4, 16, 1, 64, 4, 1, 1)])
def test_window_segments_near_const_ends(tiling):
    """Windows reach 4 cells past their segment: with 2 cells per thread the two segments next to each
    const end see past it, and take that end's value at every stage as the last segment does."""
    n = 64
    grid = (n, 3, 3)
    s = dict(grid=grid, dgrid=(1.0 / n,) * 3, gamma=5 / 3, cfl=0.35, bc={"x": "const", "y": "circ", "z": "circ"},
             limiter=("vanleer", "minmod", "superbee"), magnet=True, time_max=1e5, iter_max=6)
    o, g = make_pair(s, _wavy_tube(n))
    g.set_tiling(1, tiling, kind="magnet")
    o.run()
    g.run()
    _assert_close(o, g, 1e-11, f"window tiling {tiling}")
    g.close()


@pytest.mark.parametrize("bc", ["circ", "const"])
@pytest.mark.parametrize("n", [5, 7, 8, 13])
def test_window_rows_at_the_one_wrap_threshold(n, bc):
    """The window kernels wrap (circ) or clamp (const) their rows with selects where one wrap reaches
    every row -- N >= C + 4 for the chain, N >= C + 1 for CT -- and with loops below that.  With C = 4:
    n = 5 and 7 take the loops in the chain (5 takes the selects in CT), 8 sits at the chain's threshold,
    13 leaves a ragged one-cell last segment; 16 pencils per CTA on 9 pencils leave idle threads."""
    grid = (n, 3, 3)
    s = dict(grid=grid, dgrid=(1.0 / n,) * 3, gamma=5 / 3, cfl=0.35, bc={"x": bc, "y": "circ", "z": "circ"},
             limiter=("vanleer", "minmod", "superbee"), magnet=True, time_max=1e5, iter_max=6)
    o, g = make_pair(s, _wavy_tube(n))
    seg = -(-n // 4)
    g.set_tiling(1, (32 // seg, seg, 1, 32, 4, 1, 1), kind="magnet")
    o.run()
    g.run()
    _assert_close(o, g, 1e-11, f"n={n} {bc}")
    g.close()
