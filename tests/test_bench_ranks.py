"""The multi-rank side of bench.py on CPU (gloo, world size 2, 127.0.0.1).

Under torchrun every rank runs its own replica of the solve; the job's time is the
slowest rank's (all-reduce MAX) and its throughput counts the iterations of all ranks.
The reference arm runs on rank 0 alone; the other ranks return without work.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks(times[rank], dist, "cpu")
        out[rank] = got
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    port = _free_port()
    times = [[12.5, 40.0], [11.0, 47.5]]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(2, port, times, out), nprocs=2, join=True,
                       start_method="spawn")
    assert out[0] == [12.5, 47.5] and out[1] == [12.5, 47.5]


def test_job_throughput_counts_every_rank():
    sys.path.insert(0, REPO)
    import bench
    assert bench.job_throughput(1, 200, 500.0) == pytest.approx(400.0)
    assert bench.job_throughput(8, 200, 500.0) == pytest.approx(3200.0)


def test_reference_arm_runs_on_rank0_only(monkeypatch, capsys):
    sys.path.insert(0, REPO)
    import bench
    called = []
    monkeypatch.setattr(bench, "cpu_reference", lambda *a, **k: called.append(1))
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    bench.main()
    assert called == [] and capsys.readouterr().out == ""
