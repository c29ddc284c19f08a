"""CPU test of the multi-GPU replica plumbing with two gloo ranks: the job
time is the slowest rank's, the job's rate sums the ranks' work, and only
rank 0 reports (the same code runs with NCCL on GPUs in bench.py)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from alpine_b200 import replicas

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = replicas.world_info()
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        rate, job_ms = replicas.job_rate(1000.0, ms, w, dist, "cpu")
        out.put((r, local, rate, job_ms, replicas.reports(r)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, local, rate, job_ms, reports in res:
        assert local == rank
        assert job_ms == pytest.approx(15.0)                 # the slowest rank
        assert rate == pytest.approx(2 * 1000.0 / 0.015)     # both ranks' work over the job time
        assert reports == (rank == 0)


def test_single_process_defaults(monkeypatch):
    from alpine_b200 import replicas

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.world_info() == (1, 0, 0)
    assert replicas.job_rate(500.0, 20.0, 1) == (pytest.approx(25000.0), 20.0)


def test_reference_arm_other_ranks_are_silent(monkeypatch, capsys):
    """bench.py --impl reference under torchrun: ranks other than 0 exit
    without work or output."""
    import argparse

    import bench

    monkeypatch.setenv("RANK", "1")
    bench.run_reference(argparse.Namespace(gpus=2, steps=1, warmup=0))
    assert capsys.readouterr().out == ""
