"""Serving (imogen_b200.serve over the native job server) on the GPU: results in the mix equal results
alone, the HBM budget holds, the mixed form stays within its tolerance of FP64, jobs can be polled and
cancelled, and the C ABI's img_batch_submit / poll / cancel work directly (GPU required)."""
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
    done = srv.serve(jobs)
    st = srv.stats()                                     # the native server's own accounting
    assert len(done) == len(jobs) and st["used"] == 0 and st["finished"] == len(jobs)
    assert max(need) <= st["peak"] <= budget
    assert all("totals" in j.result for j in done)


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


def test_job_api_through_the_c_abi():
    """img_server_create / img_batch_submit / img_batch_poll / img_batch_cancel / img_batch_result as a
    MEX gateway would call them (ctypes, no Python scheduler), including a job that fails at admission
    (an unsupported boundary) next to jobs that finish."""
    import ctypes
    from imogen_b200 import _lib
    from imogen_b200.run import make_config
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.img_server_create(ctypes.byref(h), 1 << 34, 2, 1) == 0
    dp = ctypes.POINTER(ctypes.c_double)
    ids = []
    jobs = _stream("mixed", count=5, seed=21)
    bad = dict(jobs[0].settings, bc="linear")
    for settings in [j.settings for j in jobs] + [bad]:
        st = [j for j in jobs if j.settings is settings] or [jobs[0]]
        rho, mom, ener, mag = st[0].state
        cfg = make_config(precision="mixed", **settings)
        f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
        arrs = [f(rho), np.concatenate([f(m) for m in mom]), f(ener), np.concatenate([f(b) for b in mag])]
        jid = ctypes.c_int()
        assert L.img_batch_submit(h, ctypes.byref(cfg), *[a.ctypes.data_as(dp) for a in arrs], ctypes.byref(jid)) == 0
        ids.append(jid.value)
    victim = ids[2]
    assert L.img_batch_cancel(h, victim) == 0
    info = _lib.ImgJobInfo()
    import time
    t0 = time.time()
    while True:
        states = []
        for j in ids:
            assert L.img_batch_poll(h, j, ctypes.byref(info)) == 0
            states.append(info.status)
        if all(s >= 2 for s in states) or time.time() - t0 > 120:
            break
        time.sleep(0.01)
    assert states[2] == 4                                # cancelled
    assert states[-1] == 3                               # failed: the linear BC is rejected at creation
    L.img_batch_poll(h, ids[-1], ctypes.byref(info))
    assert b"linear" in info.error and info.error_code == -4
    for j, s in zip(ids[:-1], states[:-1]):
        if j == victim:
            continue
        assert s == 2
        tot = np.zeros(8)
        assert L.img_batch_result(h, j, -1, tot.ctypes.data_as(dp), 8) == 0 and tot[0] > 0
    assert L.img_batch_cancel(h, ids[0]) != 0            # already done
    srv_info = _lib.ImgServerInfo()
    assert L.img_server_stats(h, ctypes.byref(srv_info)) == 0 and srv_info.used == 0
    assert L.img_server_destroy(h) == 0
