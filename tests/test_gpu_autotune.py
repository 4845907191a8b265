"""Autotuner (img_autotune): it leaves the state untouched, every tiling it may pick gives the same
results (bit for bit within one kernel family; within round-off between the pencil-tile and the
segment fluid kernels, whose compiled arithmetic may contract differently into FMAs), and later
contexts of the same shape start from the tuned tiling (GPU required)."""
import numpy as np
import pytest

from imogen_b200 import ImogenRun, problems

pytestmark = pytest.mark.gpu


def _run(s, st, precision):
    r = ImogenRun(precision=precision, **s)
    r.set_state(*st)
    return r


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["ot", "kh", "tube"])
def test_autotune_keeps_state_and_results(precision, case):
    if case == "ot":
        s, st = problems.orszag_tang(96)
    elif case == "kh":
        s, st = problems.kelvin_helmholtz(24)
    else:
        s, st = problems.brio_wu_tube(1500, 1.0, 0.125, 1.0, 0.1)
    s = dict(s, time_max=1e5, iter_max=10 ** 6)
    tuned, plain = _run(s, st, precision), _run(s, st, precision)
    for r in (tuned, plain):                     # past the first (edge-capture) iteration
        r.iterate()
    before = tuned.state()
    t0 = tuned.time.time
    tuned.autotune(trials=2)
    after = tuned.state()
    for k in before:
        assert np.array_equal(before[k], after[k]), k
    assert tuned.time.time == t0
    for _ in range(4):
        tuned.iterate()
        plain.iterate()
    a, b = tuned.state(), plain.state()
    # bit for bit where both runs use the same kernel instantiations (family and cells per thread, fluid
    # and magnet); other instantiations may contract their sums into FMAs differently
    same_kernels = all(x[4] == y[4] and x[6] == y[6] for kind in ("fluid", "magnet")
                       for x, y in zip(tuned.tiling(kind).values(), plain.tiling(kind).values()))
    tol = 0.0 if same_kernels else (1e-13 if precision == "fp64" else 1e-6)
    for k in a:
        rel = float(np.abs(a[k] - b[k]).sum() / max(np.abs(b[k]).sum(), 1e-300))
        assert rel <= tol, (k, rel, tuned.tiling(), plain.tiling())
    again = _run(s, st, precision)
    assert again.tiling("fluid") == tuned.tiling("fluid") and again.tiling("magnet") == tuned.tiling("magnet")
    for r in (tuned, plain, again):
        r.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chain_with_both_components_per_cta_matches(precision):
    """The magnet chain tiling that carries both transverse components in one CTA (a choice the
    autotuner may make) gives bitwise the same results as one component per CTA."""
    for case in ("ot", "kh"):
        s, st = problems.orszag_tang(64) if case == "ot" else problems.kelvin_helmholtz(20)
        s = dict(s, time_max=1e5, iter_max=10 ** 6)
        a, b = _run(s, st, precision), _run(s, st, precision)
        for dim, t in a.tiling("magnet").items():
            if s["grid"][dim - 1] < 3 or t[4] > 2:
                continue
            a.set_tiling(dim, tuple(t[:5]) + (2,), kind="magnet")
            assert a.tiling("magnet")[dim][5] == 2
        for _ in range(4):
            a.iterate()
            b.iterate()
        x, y = a.state(), b.state()
        for k in x:
            assert np.array_equal(x[k], y[k]), (case, k)
        a.close()
        b.close()
