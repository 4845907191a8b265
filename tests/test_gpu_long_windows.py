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
