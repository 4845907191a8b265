"""Batched execution (img_batch_*) against the same runs advanced one at a time (GPU required).

A batch issues each kernel of an iteration as one launch over all members; every member's kernel
arguments are the ones its own launches would use, so a member's state must be bitwise identical
to the same run stepped alone, whatever else is in the batch.
"""
import numpy as np
import pytest

from imogen_b200 import ImogenBatch, ImogenError, ImogenRun, problems

pytestmark = pytest.mark.gpu


def _make(settings, state, precision):
    r = ImogenRun(precision=precision, **settings)
    r.set_state(*state)
    return r


def _same(a, b, what):
    sa, sb = a.state(), b.state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), f"{what}: {k} differs (max |d| {np.abs(sa[k] - sb[k]).max():.3e})"


def _ot(n, time_max=1e5, cfl=0.35):
    s, st = problems.orszag_tang(n)
    return dict(s, time_max=time_max, iter_max=10 ** 6, cfl=cfl), st


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_of_uneven_grids_matches_runs_alone(precision):
    cases = [_ot(32), _ot(48, cfl=0.3), _ot(64), _ot(40)]
    alone = [_make(s, st, precision) for s, st in cases]
    together = [_make(s, st, precision) for s, st in cases]
    with ImogenBatch(together) as b:
        for _ in range(7):                     # first (edge-capture) iteration, then graph replays
            b.step()
            for r in alone:
                r.iterate()
        for r in alone:
            r.sync()
        for i, (x, y) in enumerate(zip(alone, together)):
            _same(x, y, f"member {i}")
            assert x.time.iteration == y.time.iteration
            assert x.time.time == y.time.time and x.time.dTime == y.time.dTime
        assert b.launches > 0
    for r in alone + together:
        r.close()


def test_brio_wu_tubes_batch_matches_alone():
    tubes = problems.brio_wu_ensemble(count=6, seed=3, nmin=64, nmax=700)
    alone = [_make(dict(s, time_max=1e5), st, "mixed") for s, st in tubes]
    together = [_make(dict(s, time_max=1e5), st, "mixed") for s, st in tubes]
    b = ImogenBatch(together)
    for _ in range(5):
        b.step()
        for r in alone:
            r.iterate()
    for r in alone:
        r.sync()
    for i, (x, y) in enumerate(zip(alone, together)):
        _same(x, y, f"tube {i} (n={x.grid[0]})")
    b.close()


def test_members_stop_at_their_own_time_max():
    # the smallest grid takes the largest steps: it reaches its TIMEMAX first and then stays put
    cases = [_ot(24, time_max=0.02), _ot(48, time_max=0.05), _ot(32, time_max=1e5)]
    alone = [_make(s, st, "fp64") for s, st in cases]
    together = [_make(s, st, "fp64") for s, st in cases]
    b = ImogenBatch(together)
    for _ in range(12):
        b.step()
    flags = b.status()
    for r in alone[:2]:
        r.run()                                # until TIMEMAX
    for _ in range(12):
        alone[2].iterate()
    alone[2].sync()
    assert flags[0] & 1 and flags[1] & 1 and not flags[2] & 1, flags
    for i, (x, y) in enumerate(zip(alone, together)):
        _same(x, y, f"member {i}")
    assert together[0].time.time == pytest.approx(0.02, rel=0, abs=1e-15)
    b.close()


def test_batch_with_stateful_boundaries():
    s, st = problems.sedov(40, dims=2, bc="trans")
    s = dict(s, time_max=1e5)
    s2, st2 = problems.sedov(48, dims=2, bc="trans")
    s2 = dict(s2, time_max=1e5)
    alone = [_make(s, st, "fp64"), _make(s2, st2, "fp64")]
    together = [_make(s, st, "fp64"), _make(s2, st2, "fp64")]
    b = ImogenBatch(together)
    for _ in range(6):
        b.step()
        for r in alone:
            r.iterate()
    for r in alone:
        r.sync()
    for i, (x, y) in enumerate(zip(alone, together)):
        _same(x, y, f"member {i}")
    b.close()


def test_batch_rejects_members_with_another_launch_sequence():
    s2, st2 = _ot(32)
    s3, st3 = problems.kelvin_helmholtz(16)
    a = _make(s2, st2, "mixed")
    c = _make(dict(s3, time_max=1e5), st3, "mixed")
    f = _make(s2, st2, "fp64")
    b = ImogenBatch([a])
    with pytest.raises(ImogenError):
        b.add(c)                               # 3-D member in a 2-D batch
    with pytest.raises(ImogenError):
        b.add(f)                               # other precision
    a.iterate()                                # a member stepped on its own ...
    a.sync()
    b.close()
    for r in (a, c, f):
        r.close()


def test_long_cluster_members_with_fade_match_alone():
    """Members whose x pencils span a 4-CTA cluster at 4 cells per thread (N > 4096), fade ends: the
    batched launches run the same cluster barriers and DSMEM exchanges as the launches alone."""
    tubes = [problems.brio_wu_ensemble(xbc="fade")[i] for i in (4, 5, 9, 1)]      # N = 4288, 6054, 6541, 652
    alone = [_make(dict(s, time_max=1e5), st, "mixed") for s, st in tubes]
    together = [_make(dict(s, time_max=1e5), st, "mixed") for s, st in tubes]
    b = ImogenBatch(together)
    for _ in range(8):
        b.step()
        for r in alone:
            r.iterate()
    for r in alone:
        r.sync()
    for i, (x, y) in enumerate(zip(alone, together)):
        _same(x, y, f"tube {i} (n={x.grid[0]})")
    b.close()
    for r in alone + together:
        r.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fresh_member_joins_a_running_batch(precision):
    """A new member takes its first (edge-capturing, CFL-reducing) iteration inside a batch whose
    members are mid-run (other sweep-order phases): everyone stays bitwise equal to running alone."""
    s, st = _ot(40)
    first = [_ot(32), _ot(48)]
    alone = [_make(c, x, precision) for c, x in first] + [_make(s, st, precision)]
    together = [_make(c, x, precision) for c, x in first]
    b = ImogenBatch(together)
    for _ in range(4):
        b.step()
        alone[0].iterate()
        alone[1].iterate()
    late = _make(s, st, precision)
    b.add(late)
    together.append(late)
    for _ in range(9):
        b.step()
        for r in alone:
            r.iterate()
    for r in alone:
        r.sync()
    for i, (x, y) in enumerate(zip(alone, together)):
        _same(x, y, f"member {i}")
    b.close()
    for r in alone + together:
        r.close()
