"""The configurations the path is specified on, at their stated sizes (GPU required).

* Sod shock tube, N = 1024, transparent ends, CFL 0.7, vanleer, FP64, run to t = 0.2: the CUDA path
  against the C++ oracle (1e-10 relative L1) and against the exact Riemann solution at gamma = 5/3.
* Orszag-Tang 512^2, FP64, 100 iterations: against the oracle at 1e-10 relative L1.
* 3-D MHD Kelvin-Helmholtz 256^3, 200 iterations: the mixed form (FP32 state) against the plain FP64
  form on the GPU, per variable (rho, E; momentum and B as vectors) within 1e-5 relative L1, with
  the discrete div B of both forms and their compensated totals.
* Brio-Wu ensemble: 16 members of the seeded 512-member ensemble advanced in one batch, each against
  the oracle (FP64 batch at 1e-10; mixed batch at 2e-5).
"""
import math

import numpy as np
import pytest

from imogen_b200 import ImogenBatch, ImogenRun, problems
from oracle import cpp_oracle
from tests.parity import errors, errors_vector, make_pair, rel_l1
from tests.riemann import sample

pytestmark = pytest.mark.gpu


def _assert_close(o, g, tol, what):
    e = errors(g.state(), o.state())
    bad = {k: v for k, v in e.items() if not (v <= tol)}
    assert not bad, f"{what}: relative L1 above {tol}: {bad}"


def div_b(mag, dgrid, periodic=(True, True, True)):
    """Discrete divergence of the face-centred field (B_d(i) on face i-1/2, MagnetArray.m:36-38):
    sum_d (B_d(i+1) - B_d(i)) / dgrid_d, over cells whose upper face is inside the grid."""
    out = np.zeros(mag.shape[1:])
    for d in range(3):
        if mag.shape[1 + d] < 2:
            continue
        out += (np.roll(mag[d], -1, axis=d) - mag[d]) / dgrid[d]
    keep = [slice(None) if periodic[d] or mag.shape[1 + d] < 2 else slice(0, -1) for d in range(3)]
    return out[tuple(keep)]


def test_sod_1024_to_t_0_2():
    s, st = problems.sod(1024, time_max=0.2)
    o, g = make_pair(s, st)
    no = o.run()
    ng = g.run()
    assert no == ng
    assert g.time.time == pytest.approx(0.2, abs=1e-14) and o.time == pytest.approx(0.2, abs=1e-14)
    _assert_close(o, g, 1e-10, "Sod 1024 to t=0.2")
    rho = g.state()["mass"][:, 0, 0]
    x = (np.arange(1024) + 0.5) / 1024
    ex = sample(x, 0.2, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 5 / 3)
    l1 = np.abs(rho - ex[0]).mean()
    assert l1 < 3e-3, l1     # first order at the contact and shock on 1024 cells
    g.close()


def test_orszag_tang_512_fp64_100_iterations():
    s, st = problems.orszag_tang(512)
    s = dict(s, iter_max=100)
    o, g = make_pair(s, st)
    cpp_oracle.set_threads(cpp_oracle.max_threads())
    assert o.run() == g.run() == 100
    assert abs(g.time.time - o.time) <= 1e-12 * o.time
    _assert_close(o, g, 1e-10, "Orszag-Tang 512^2, 100 iterations")
    g.close()


def test_kelvin_helmholtz_256_mixed_vs_fp64_200_iterations():
    s, st = problems.kelvin_helmholtz(256)
    assert s["iter_max"] == 200
    runs = {}
    for precision in ("fp64", "mixed"):
        g = ImogenRun(precision=precision, **s)
        g.set_state(*st)
        assert g.run() == 200
        runs[precision] = g
    a, b = runs["mixed"].state(), runs["fp64"].state()
    e = errors_vector(a, b)
    assert max(e.values()) <= 1e-5, e
    dx = s["dgrid"]
    db64 = np.abs(div_b(b["mag"], dx)).max() * dx[0] / np.abs(b["mag"]).max()
    db32 = np.abs(div_b(a["mag"], dx)).max() * dx[0] / np.abs(a["mag"]).max()
    assert db64 < 1e-12 and db32 < 1e-5, (db64, db32)
    t64, t32 = runs["fp64"].totals(), runs["mixed"].totals()
    # mass and energy are conserved under periodic boundaries up to round-off
    assert abs(t64[0] - st[0].sum()) <= 1e-12 * st[0].sum()
    assert abs(t32[0] - t64[0]) <= 1e-6 * t64[0] and abs(t32[4] - t64[4]) <= 1e-6 * t64[4]
    for g in runs.values():
        g.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 2e-5)])
def test_brio_wu_ensemble_members_against_oracle(precision, tol):
    # the FP64 form holds pencils of up to about 5000 cells on one cluster of 4 CTAs (longer ones are
    # rejected at img_create); the mixed form takes the ensemble's whole range (up to 8192)
    tubes = [t for t in problems.brio_wu_ensemble() if precision == "mixed" or t[0]["grid"][0] <= 4096][:16]
    iters = 40
    runs = []
    for s, st in tubes:
        r = ImogenRun(precision=precision, **dict(s, iter_max=iters, time_max=1e5))
        r.set_state(*st)
        runs.append(r)
    b = ImogenBatch(runs)
    b.run()
    assert all(f & 1 and not f & 2 for f in b.status())
    cpp_oracle.set_threads(cpp_oracle.max_threads())
    for k, ((s, st), r) in enumerate(zip(tubes, runs)):
        o = cpp_oracle.Sim(**problems.oracle_kwargs(dict(s, iter_max=iters, time_max=1e5)))
        o.set_state(*st)
        assert o.run() == iters
        assert abs(r.time.time - o.time) <= (1e-12 if precision == "fp64" else 1e-5) * o.time
        _assert_close(o, r, tol, f"member {k} (n={s['grid'][0]}, {precision})")
    b.close()
    for r in runs:
        r.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_totals_equal_exact_sums(precision):
    """img_totals and img_totals_static (compensated FP64 sums on the device) against math.fsum of the
    downloaded arrays (the correctly rounded sum): within one ulp of the total, or, for totals that
    cancel to near zero (momentum), within the compensated sum's n*eps^2*sum|x| term."""
    s, st = problems.orszag_tang(528)
    g = ImogenRun(precision=precision, **dict(s, iter_max=5, time_max=1e5))
    g.set_state(*st)
    g.run()
    sa = g.state()
    arrays = [sa["mass"], sa["mom"][0], sa["mom"][1], sa["mom"][2], sa["ener"], sa["mag"][0], sa["mag"][1],
              sa["mag"][2]]
    for tot in (g.totals(), g.totals_static()):
        for v, arr in enumerate(arrays):
            flat = arr.ravel()
            exact = math.fsum(flat)
            bound = max(math.ulp(exact), 16 * flat.size * 2.0 ** -106 * float(np.abs(flat).sum()))
            assert abs(tot[v] - exact) <= bound, (v, tot[v], exact, bound)
    g.close()
