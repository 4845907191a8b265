"""Failure paths, injected on the host only (GPU required; nothing here faults, traps or hangs a GPU).

* TimeManager.m:79-86: a state whose every speed is below the 1e-2 floor is a CFL error.
* A NaN in a job's host initial state: with the default non-finite check the first CFL pass flags it
  and the run stops with IMG_ERR_NONFINITE before any sweep touches the state; with the check off the
  run follows the reference (its max ignores NaN, TimeManager.m:70-76 and wFluidFlux.m:20, and
  MINMASS replaces a NaN density, relaxingFluid.m:39,71), compared with the oracle.
* One such faulty job inside a batch and inside the serving loop: it stops with its error flag while
  every other member finishes bitwise equal to its run alone, and its memory returns to the budget.
"""
import numpy as np
import pytest

from imogen_b200 import ImogenBatch, ImogenError, ImogenRun, problems, serve
from oracle import cpp_oracle, np_oracle
from tests.parity import rel_l1

pytestmark = pytest.mark.gpu

IMG_ERR_CFL, IMG_ERR_NONFINITE = -5, -6


def _ot(n=32, **kw):
    s, st = problems.orszag_tang(n)
    s = dict(s, time_max=1e5, iter_max=6)
    s.update(kw)
    return s, st


def _with_nan(st, var="ener", cell=(5, 7, 0)):
    rho, mom, ener, mag = (np.array(a, copy=True) for a in st)
    {"mass": rho, "ener": ener}[var][cell] = np.nan
    return rho, mom, ener, mag


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cfl_error_when_every_speed_is_below_the_floor(precision):
    grid = (32, 32, 1)
    rho = np.ones(grid)
    mom = np.zeros((3,) + grid)
    mag = np.zeros((3,) + grid)
    ener = np.full(grid, 1e-8 / (2 / 3))          # P = 1e-8: c_s ~ 1.3e-4 < 1e-2
    s = dict(grid=grid, dgrid=(1 / 32, 1 / 32, 1.0), gamma=5 / 3, cfl=0.7, bc="circ", magnet=False,
             time_max=1e5, iter_max=3)
    o = np_oracle.Sim(**problems.oracle_kwargs(s))
    o.set_state(rho, mom, ener, mag)
    with pytest.raises(FloatingPointError):
        o.run()
    g = ImogenRun(precision=precision, **s)
    g.set_state(rho, mom, ener, mag)
    with pytest.raises(ImogenError) as e:
        g.run()
    assert e.value.code == IMG_ERR_CFL
    g.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("var", ["mass", "ener"])
def test_nan_in_host_initial_state_stops_the_run(precision, var):
    s, st = _ot()
    bad = _with_nan(st, var)
    g = ImogenRun(precision=precision, **s)
    g.set_state(*bad)
    with pytest.raises(ImogenError) as e:
        g.run()
    assert e.value.code == IMG_ERR_NONFINITE
    # flagged by the first CFL pass, before any sweep: the state is the initial one
    sa = g.state()
    ref = {"mass": bad[0], "ener": bad[2]}[var]
    got = sa[var]
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    fin = ~np.isnan(ref)
    tol = 0 if precision == "fp64" else 1e-7
    assert np.all(np.abs(got[fin] - ref[fin]) <= tol * np.abs(ref[fin]))
    g.close()


def test_nan_density_follows_the_reference_without_the_check():
    """max(rho, MINMASS) replaces a NaN density (MATLAB's max ignores NaN) and the pencil and CFL
    maxima skip NaN cells: the run goes on, and GPU and oracle agree cell for cell."""
    s, st = _ot(iter_max=2)
    bad = _with_nan(st, "mass")
    o = cpp_oracle.Sim(**problems.oracle_kwargs(s))
    o.set_state(*bad)
    assert o.run() == 2
    g = ImogenRun(precision="fp64", nonfinite_check=False, **s)
    g.set_state(*bad)
    assert g.run() == 2
    assert abs(g.time.time - o.time) <= 1e-12 * o.time
    a, b = g.state(), o.state()
    rho = a["mass"]
    assert not np.isnan(rho).any() and rho.min() == pytest.approx(1e-5)   # the NaN cell is MINMASS
    for k in ("mass", "ener", "mom", "mag"):
        na, nb = np.isnan(a[k]), np.isnan(b[k])
        assert np.array_equal(na, nb), k
        assert rel_l1(np.where(na, 0, a[k]), np.where(nb, 0, b[k])) <= 1e-12, k
    g.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_faulty_member_stops_alone_in_a_batch(precision):
    cases = [_ot(32), _ot(48), _ot(40)]
    states = [st for _, st in cases]
    states[1] = _with_nan(states[1], "ener", (10, 3, 0))
    alone = []
    for k in (0, 2):
        r = ImogenRun(precision=precision, **cases[k][0])
        r.set_state(*states[k])
        r.run()
        alone.append(r)
    members = []
    for (s, _), st in zip(cases, states):
        r = ImogenRun(precision=precision, **s)
        r.set_state(*st)
        members.append(r)
    b = ImogenBatch(members)
    with pytest.raises(ImogenError) as e:      # the batch runs every member to its end, then reports
        b.run()
    assert e.value.code == IMG_ERR_NONFINITE
    flags = b.status()
    assert flags[1] & 2 and not flags[0] & 2 and not flags[2] & 2, flags
    for x, y in zip(alone, (members[0], members[2])):
        sa, sb = x.state(), y.state()
        for k in sa:
            assert np.array_equal(sa[k], sb[k]), k
    with pytest.raises(ImogenError) as e:
        members[1].sync()
    assert e.value.code == IMG_ERR_NONFINITE
    b.close()
    for r in alone + members:
        r.close()


def test_faulty_job_in_the_serving_mix():
    def stream():
        return serve.sedov_stream(6, rate=400.0, seed=3, sizes2=(24, 40), sizes3=(20, 24), precision="mixed",
                                  time_max=1e-2)
    jobs = stream()
    faulty = jobs[2]
    rho, mom, ener, mag = (np.array(a, copy=True) for a in faulty.state)
    ener.flat[3] = np.nan
    faulty.state = (rho, mom, ener, mag)
    srv = serve.Server(hbm_budget=1 << 34, check_every=1, keep="state")
    done = {j.id: j for j in srv.serve(jobs)}
    assert srv.used == 0 and len(done) == len(jobs)
    assert done[faulty.id].result["code"] == IMG_ERR_NONFINITE
    assert srv.poll(faulty.id)["state"] == "failed"
    alone = {j.id: j for j in serve.one_at_a_time([j for j in stream() if j.id != faulty.id], precision="mixed",
                                                  keep="state")}
    for jid, ref in alone.items():
        got = done[jid]
        assert srv.poll(jid)["state"] == "done"
        assert got.iterations == ref.iterations
        for k in ("mass", "mom", "ener"):
            assert np.array_equal(got.result[k], ref.result[k]), (jid, k)
