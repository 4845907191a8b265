"""img_totals_static (totals in static device scratch, no allocation) against img_totals.

Collected last on purpose (file name): it must pass both alone and after every other GPU test, so
it relies on no state that an earlier test leaves behind, and it checks that a call after a call on
another grid (other sizes, other precision) reads nothing stale from the shared scratch.
"""
import numpy as np
import pytest

from imogen_b200 import ImogenRun, problems

pytestmark = pytest.mark.gpu


def _run(n, precision, iters):
    s, st = problems.orszag_tang(n)
    g = ImogenRun(precision=precision, **dict(s, iter_max=iters, time_max=1e5))
    g.set_state(*st)
    g.run()
    return g


# 48^2 fits in one pass of the fixed 1023 x 256-thread grid; 528^2 = 278784 cells does not, so the
# grid-stride loop and every block's partials carry data
@pytest.mark.parametrize("n", [48, 528])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_static_totals_match_two_calls_in_a_row(precision, n):
    g = _run(n, precision, 3)
    try:
        ref1, ref2 = g.totals(), g.totals()
        got1, got2 = g.totals_static(), g.totals_static()
        np.testing.assert_array_equal(ref1, ref2)
        np.testing.assert_array_equal(got1, ref1)
        np.testing.assert_array_equal(got2, ref1)
        assert np.all(np.isfinite(got1))
        assert got1[0] > 0  # total mass
    finally:
        g.close()


def test_static_totals_alternating_contexts():
    a = _run(64, "fp64", 2)
    b = _run(24, "mixed", 1)
    try:
        ra, rb = a.totals(), b.totals()
        for _ in range(2):
            np.testing.assert_array_equal(a.totals_static(), ra)
            np.testing.assert_array_equal(b.totals_static(), rb)
        # the state moves on; the static path follows it
        a.iterate()
        a.sync()
        np.testing.assert_array_equal(a.totals_static(), a.totals())
    finally:
        a.close()
        b.close()


def test_static_totals_refuse_a_capturing_stream():
    """The call copies from host memory and synchronises, which a graph capture cannot hold: while
    the context's stream captures it fails with IMG_ERR_STATE and enqueues nothing."""
    from cuda.bindings import runtime as rt
    from imogen_b200 import ImogenError
    g = _run(24, "fp64", 1)
    try:
        want = g.totals()
        st = rt.cudaStream_t(g.stream)
        err, = rt.cudaStreamBeginCapture(st, rt.cudaStreamCaptureMode.cudaStreamCaptureModeThreadLocal)
        assert err == rt.cudaError_t.cudaSuccess
        try:
            with pytest.raises(ImogenError, match="captured"):
                g.totals_static()
        finally:
            err, graph = rt.cudaStreamEndCapture(st)
            assert err == rt.cudaError_t.cudaSuccess
            rt.cudaGraphDestroy(graph)
        np.testing.assert_array_equal(g.totals_static(), want)
    finally:
        g.close()
