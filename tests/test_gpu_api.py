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


def test_bulk_transfers_from_pinned_buffers_match_pageable_ones():
    """Mixed form: page-locked and pageable caller buffers (the staged copies do not depend on the
    caller's pinning) leave the same bits in the state and return the same values."""
    import torch
    s, st = problems.orszag_tang(48)
    rng = np.random.default_rng(7)
    # positive density and pressure, and no z momentum: on this 2-D grid dz = 1, and a z speed that
    # wins the CFL argmax would take dt from dz (TimeManager.m), 48 times too long for the x and y sweeps
    base = {"mass": 1.0, "ener": 2.0}
    amp = {"momz": 0.0}
    new = {k: np.ascontiguousarray(base.get(k, 0.0) + amp.get(k, 0.1) * (rng.random(48 * 48) - 0.5)) for k in NAMES}
    got = {}
    for kind in ("pageable", "pinned"):
        r = ImogenRun(precision="mixed", **dict(s, time_max=1e5, iter_max=100))
        r.set_state(*st)
        if kind == "pinned":
            ins = {k: torch.from_numpy(v.copy()).pin_memory().numpy() for k, v in new.items()}
            outs = {k: torch.zeros(r.ncell, dtype=torch.float64).pin_memory().numpy() for k in NAMES}
        else:
            ins = {k: v.copy() for k, v in new.items()}
            outs = {k: np.zeros(r.ncell) for k in NAMES}
        for _ in range(2):                       # two rounds: the second reuses what the first set up
            r.upload_many(ins)
            r.iterate()
            r.download_many(outs)
        got[kind] = {k: v.copy() for k, v in outs.items()}
        got[kind]["single"] = r.download("mass").reshape(-1, order="F")
        r.close()
    for k in got["pageable"]:
        assert np.all(np.isfinite(got["pinned"][k])), k
        assert np.array_equal(got["pinned"][k], got["pageable"][k]), k
    assert np.array_equal(got["pinned"]["mass"], got["pinned"]["single"])


def test_pencils_longer_than_four_ctas_hold_are_rejected():
    with pytest.raises(ImogenError) as e:
        ImogenRun(grid=(20000, 1, 1), precision="fp64")
    assert "cannot be scheduled" in str(e.value) or "UNSUPPORTED" in str(e.value)
