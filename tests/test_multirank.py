"""The bench's multi-rank host logic on the CPU: two gloo ranks on 127.0.0.1.

bench.py runs one replica per GPU (the meshes are independent, so the data path has no
collective) and reports the whole job's element-updates/s over the slowest rank's
device time.  These tests run that reduction and the reference arm's rank split as
two processes with the gloo backend; no GPU is involved.
"""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist)  # rank 1 is the slow one
        rate = bench.job_rate(1000, 50, world, ms)
        out.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, rate in got:
        assert ms == 15.0  # the slowest rank's time on every rank
        assert rate == pytest.approx(1000 * 50 * 2 / 0.015)


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm's rank 0 alone works and prints; the others
    exit 0 at once (checked here for rank 1, which must print nothing)."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
