"""Replica aggregation of bench.py over two gloo ranks on the CPU: the step
time is the max over ranks and the value counts every rank's k-mers."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms = [100.0, 250.0][rank]
        n = [1_000_000, 3_000_000][rank]
        got = bench.replica_totals(ms, n, dist, "cpu")
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_replica_totals_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:  # no fork of a threaded process
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms, value = res[r]
        assert ms == 250.0
        assert value == pytest.approx(4_000_000 / 0.25)


def test_replica_totals_single_process():
    import bench
    ms, value = bench.replica_totals(200.0, 1_000_000)
    assert ms == 200.0 and value == pytest.approx(5e6)
