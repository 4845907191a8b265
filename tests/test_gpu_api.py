"""C-ABI behaviour beyond the sweeps (GPU required): bulk transfers, the progress counter, and the
limits the library rejects cleanly."""
import numpy as np
import pytest

from imogen_b200 import ImogenError, ImogenRun, problems

pytestmark = pytest.mark.gpu

NAMES = ("mass", "momx", "momy", "momz", "ener", "magx", "magy", "magz")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bulk_transfers_match_single_ones(precision):
    s, st = problems.orszag_tang(40)
    r = ImogenRun(precision=precision, **dict(s, time_max=1e5, iter_max=100))
    r.set_state(*st)
    r.iterate()
    rng = np.random.default_rng(4)
    new = {k: np.ascontiguousarray(1.0 + 0.1 * rng.random(r.ncell)) for k in NAMES}
    r.upload_many(new)
    outs = {k: np.empty(r.ncell) for k in NAMES}
    r.download_many(outs)
    for k in NAMES:
        single = r.download(k).reshape(-1, order="F")
        assert np.array_equal(outs[k], single), k
        expect = new[k] if precision == "fp64" else new[k].astype(np.float32).astype(np.float64)
        assert np.array_equal(outs[k], expect), k
    r.iterate()                                  # the uploaded state steps (CFL recomputed)
    t, n, stopped = r.progress()
    assert n == 2 and not stopped and t > 0
    r.close()


def test_pencils_longer_than_four_ctas_hold_are_rejected():
    with pytest.raises(ImogenError) as e:
        ImogenRun(grid=(20000, 1, 1), precision="fp64")
    assert "cannot be scheduled" in str(e.value) or "UNSUPPORTED" in str(e.value)
