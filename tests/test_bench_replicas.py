"""The replica path of bench.py (--gpus N, one process per GPU, no data-path
collective) on CPU: two gloo ranks on 127.0.0.1.  Each rank times its own
replica; the job's time is the slowest rank's, and its rate counts every
rank's particles over that time."""
import importlib.util
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rank(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b = _bench()
        b.barrier(dist)
        ms = b.reduce_max(dist, times[rank], 0)
        out[rank] = (ms, b.whole_job_rate(1000, 10, world, ms))
        b.barrier(dist)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_replicas_report_the_slowest_time_and_the_whole_job_rate():
    world, times = 2, [120.0, 250.0]
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), times, out), nprocs=world, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1]
    ms, rate = res[0]
    assert ms == 250.0
    assert rate == pytest.approx(1000 * 10 * 2 / 0.25)


def test_single_process_needs_no_collective():
    b = _bench()
    assert b.reduce_max(None, 3.5, 0) == 3.5
    assert b.whole_job_rate(100, 4, 1, 200.0) == pytest.approx(2000.0)
