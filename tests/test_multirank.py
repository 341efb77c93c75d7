"""The N>1 bench path on CPU ranks (gloo, world size 2): every rank steps its
own replica, the job time is the max over ranks, and the value is weak-scaled.
No GPU: the ranks report synthetic per-rank times through the same helpers."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
        m = bench.reduce_max(local_ms, dist, "cpu")
        out[rank] = (m, bench.weak_scaling_value(10, world, m))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_weak_scaling():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert out[0] == out[1]
    m, v = out[0]
    assert m == 150.0
    assert v == pytest.approx(2 * 10 / 0.150)


def test_single_rank_identity():
    assert bench.reduce_max(12.5, None, "cpu") == 12.5
    assert bench.weak_scaling_value(20, 1, 1000.0) == pytest.approx(20.0)
