"""bench.py's multi-rank path on CPU: two gloo ranks (replicas only -- no
data-path collective): the job time is the slowest rank's, the job rate counts
every rank's replica, and the reference arm prints on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [120.0, 150.0][rank]
        t = bench.max_over_ranks(ms, dist, device="cpu")
        rate = bench.job_rate(4096 * 4096, 100, world, t)
        out.put((rank, t, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_count_both_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, rate in res:
        assert t == 150.0
        assert rate == pytest.approx(4096 * 4096 * 100 * 2 / 0.150)


def test_one_rank_is_its_own_job():
    import bench
    assert bench.max_over_ranks(42.0) == 42.0
    assert bench.job_rate(100, 10, 1, 1000.0) == pytest.approx(1000.0)


def test_reference_arm_prints_on_rank_zero_only(capsys):
    import bench

    class A:
        steps, warmup, gpus = 1, 0, 2
    bench.run_reference(A(), 1)
    assert capsys.readouterr().out == ""
