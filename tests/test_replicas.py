"""The multi-rank path of bench.py on CPU (gloo, world size 2): the path runs one independent replica per
rank with no collective on the data path, and the job's time is the maximum over ranks; the reference
arm runs on rank 0 alone and the other ranks leave without work."""
import importlib.util
import multiprocessing as mp
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        out.put((rank, _bench().max_over_ranks(times[rank], torch.device("cpu"))))
    finally:
        dist.destroy_process_group()


def test_job_time_is_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    times = [0.75, 1.25]
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, times, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 1.25, 1: 1.25}


def test_single_rank_time_is_its_own():
    import torch
    assert _bench().max_over_ranks(0.5, torch.device("cpu")) == 0.5


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, env=env, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
