"""The multi-GPU path of bench.py (independent replicas, one per rank):
max-over-ranks timing and the whole-job value, on CPU with two gloo ranks."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = 100.0 + 25.0 * rank  # rank 1 is the slowest replica
    t_max = bench.max_over_ranks(ms, world)
    out[rank] = (t_max, bench.replica_value(1e9, t_max, world))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_max_and_value():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:  # no fork of a threaded process
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        t_max, value = res[r]
        assert t_max == pytest.approx(125.0)
        assert value == pytest.approx(2 * 1e9 / 0.125)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_value(10.0, 1000.0, 1) == pytest.approx(10.0)
