"""The N > 1 path of the bench on CPU: two ranks over gloo (127.0.0.1); and the
reference arm's line on a small problem.
Replicas only -- the ranks share no data; they meet to time the job (the
slowest rank's time, every rank's units) -- and the reference arm runs on
rank 0 alone."""
import os
import socket
import subprocess
import sys

import pytest

from galpha_b200 import replicas as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        m = R.max_over_ranks(times[rank], dist)
        out.put((rank, m, R.job_throughput(world, 1000, m)))
    finally:
        dist.destroy_process_group()


def test_job_time_is_the_slowest_rank_on_every_rank():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    times = [2.5, 4.0]
    ps = [ctx.Process(target=_rank, args=(r, 2, port, times, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    for _, m, thr in got:
        assert m == 4.0
        assert thr == pytest.approx(2 * 1000 / 4.0e-3)


def test_single_process_and_bad_time():
    assert R.max_over_ranks(3.0) == 3.0
    assert R.job_throughput(1, 500, 2.0) == pytest.approx(250000.0)
    with pytest.raises(ValueError):
        R.job_throughput(2, 1, 0.0)


def test_reference_arm_does_no_work_off_rank_zero():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line_on_a_small_problem():
    """The reference arm's JSON line (oracle port, all host cores busy): the
    fields the comparison reads, on a 20,000-point sample of the workload."""
    import json

    env = dict(os.environ, RANK="0", WORLD_SIZE="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "0", "--n", "20000"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    sys.path.insert(0, ROOT)
    import bench

    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == bench.reference_processes(20000)
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"]["same_config"] is False and line["config"]["points"] == 20000
    assert line["ms_per_step"] == pytest.approx(20000 / (line["value"] * 1e6) * 1e3)


def test_reference_processes_fit_host_memory():
    """One worker per usable core, as many as half the available memory holds
    at 1.5 GB per 4,194,304-point problem."""
    sys.path.insert(0, ROOT)
    import bench

    n = 1 << 22
    assert bench.reference_processes(n, avail_bytes=62e9, cores=16) == 16
    assert bench.reference_processes(n, avail_bytes=64e9, cores=224) == 21
    assert bench.reference_processes(n, avail_bytes=1e9, cores=16) == 1
    assert bench.reference_processes(20000, avail_bytes=8e9, cores=64) == 16  # 0.25 GB floor per worker
    assert bench.reference_processes(n, avail_bytes=None, cores=7) in range(1, 8)
