"""Serving loop (imogen_b200.serve) on the GPU: results in the mix equal results alone, the HBM
budget holds, and the mixed form stays within its tolerance of FP64 (GPU required)."""
import numpy as np
import pytest

from imogen_b200 import serve

pytestmark = pytest.mark.gpu


def _stream(precision, count=8, seed=5):
    # small Sedov blasts (2-D 24^2..48^2, 3-D 20^3..28^3), short end time, dense arrivals
    return serve.sedov_stream(count, rate=400.0, seed=seed, sizes2=(24, 48), sizes3=(20, 28), precision=precision,
                              time_max=1e-2)


def _rel_l1(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_results_in_the_mix_equal_results_alone(precision):
    jobs = _stream(precision)
    served = serve.Server(hbm_budget=1 << 34, check_every=2, keep="state").serve(jobs)
    alone = serve.one_at_a_time(_stream(precision), precision=precision, keep="state")
    by_id = {j.id: j for j in alone}
    assert len(served) == len(jobs)
    for j in served:
        ref = by_id[j.id]
        assert j.iterations == ref.iterations >= 1, (j.id, j.iterations, ref.iterations)
        assert j.result["time"] == ref.result["time"] == pytest.approx(1e-2)
        for k in ("mass", "mom", "ener"):
            assert np.array_equal(j.result[k], ref.result[k]), (j.id, k)
    assert sum(j.iterations > 4 for j in served) >= len(jobs) // 2   # most jobs ran inside the batch
    s = serve.latency_summary(served)
    assert s["jobs"] == len(jobs) and s["p99_s"] >= s["p50_s"] > 0


def test_hbm_budget_bounds_the_jobs_on_the_device():
    jobs = _stream("mixed", count=10, seed=7)
    need = [serve.bytes_required(**dict(j.settings, precision="mixed")) for j in jobs]
    budget = 2 * max(need)
    srv = serve.Server(hbm_budget=budget, check_every=1, keep="totals")
    peak = [0]
    admit = srv._admit

    def watched():
        admit()
        peak[0] = max(peak[0], srv.used)
        assert srv.used <= budget

    srv._admit = watched
    done = srv.serve(jobs)
    assert len(done) == len(jobs) and srv.used == 0
    assert 0 < peak[0] <= budget


def test_mixed_form_within_tolerance_of_fp64():
    mixed = {j.id: j for j in serve.Server(hbm_budget=1 << 34, keep="state").serve(_stream("mixed", count=4, seed=9))}
    fp64 = {j.id: j for j in serve.one_at_a_time(_stream("fp64", count=4, seed=9), precision="fp64", keep="state")}
    for i, j in mixed.items():
        for k in ("mass", "ener"):
            assert _rel_l1(j.result[k], fp64[i].result[k]) < 1e-5, (i, k)


def test_poll_and_cancel():
    jobs = serve.sedov_stream(6, rate=400.0, seed=13, sizes2=(48, 64), sizes3=(24, 32), precision="mixed",
                              time_max=0.05)
    srv = serve.Server(hbm_budget=1 << 34, check_every=1, keep="totals")
    for j in jobs:
        srv.submit(j)
    srv.start()
    while not srv.running and srv.tick():                # until a job is on the device
        pass
    running = list(srv.running)
    assert running, "nothing running to cancel"
    victim = running[0]
    assert srv.poll(victim)["state"] == "running"
    assert srv.cancel(victim) and not srv.cancel(victim)
    assert srv.poll(victim)["state"] == "cancelled"
    while srv.tick():
        pass
    srv.close()
    states = {j.id: srv.poll(j.id)["state"] for j in jobs}
    assert states[victim] == "cancelled" and sum(s == "done" for s in states.values()) == len(jobs) - 1
    assert srv.used == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_checkpoint_resumes_bit_for_bit(precision):
    from imogen_b200 import ImogenRun, problems
    for s, st in (problems.orszag_tang(48), problems.sedov(40, dims=2, bc="trans")):
        s = dict(s, time_max=1e5, iter_max=10 ** 6)
        a = ImogenRun(precision=precision, **s)
        a.set_state(*st)
        for _ in range(3):
            a.iterate()
        ck = a.checkpoint()
        for _ in range(4):
            a.iterate()
        b = ImogenRun(precision=precision, **s)
        b.restore(ck)
        for _ in range(4):
            b.iterate()
        x, y = a.state(), b.state()
        for k in x:
            assert np.array_equal(x[k], y[k]), k
        assert a.time.time == b.time.time and a.time.iteration == b.time.iteration
        a.close()
        b.close()
