"""bench.py's N > 1 path on the host: two ranks over gloo (127.0.0.1) agree on the slowest rank's time
and on the whole-job rate, and the reference arm runs on rank 0 alone (the other ranks exit without
work). The GPU parts (CUDA events, NCCL) are covered by the single-GPU runs."""

import contextlib
import io
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    r, w, local = bench.dist_env()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 10.0 * r  # rank 1 is the slower one
        ms_max = bench.reduce_max(ms, w, local)
        rate = bench.job_rate(1000, 5, ms_max, w)
        q.put((r, w, ms_max, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time_and_the_job_rate():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for r, w, ms_max, rate in got:
        assert w == 2 and ms_max == 110.0
        assert rate == pytest.approx(2 * 1000 * 5 / 0.110)


def test_reference_arm_runs_on_rank_zero_only():
    import bench

    class Args:
        steps, warmup, gpus = 1, 0, 2

    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(Args, rank=1)
    assert buf.getvalue() == ""
