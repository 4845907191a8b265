"""Window magnet kernels along x for pencils of any length (GPU required): a length that is not a
multiple of the cells per thread leaves the last segment ragged and the threads past it idle, and a
pencil of more segments than one CTA holds spans the CTAs of a thread-block cluster, whose barrier
separates the reads from the in-place writes.

Against the C++ oracle, relative L1 per variable: FP64 1e-11 after 6 iterations, the mixed form 2e-5.
"""
import pytest

from imogen_b200 import problems
from tests.parity import errors, make_pair

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
    wb, S, cl, nt, cpt, nqc, seg = g.tiling("magnet")[1]
    assert seg == 1 and S == -(-n // cpt) and cl * nt >= S, g.tiling("magnet")
    if n > 4 * 512:
        assert cl > 1, g.tiling("magnet")
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
