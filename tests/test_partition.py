"""The multi-GPU partition (elfmmlib3d_b200.partition) on CPU: right-hand-side
column blocks, the greedy n^2 balance of uneven problems, and the
all-gather of column blocks with two gloo ranks."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from elfmmlib3d_b200 import partition as PT  # noqa: E402


@pytest.mark.parametrize("nrhs,world", [(64, 1), (64, 2), (64, 3), (64, 8), (5, 8), (0, 4), (127, 4)])
def test_rhs_columns_cover_once(nrhs, world):
    blocks = [PT.rhs_columns(nrhs, world, r) for r in range(world)]
    seen = np.concatenate([np.arange(a, b) for a, b in blocks]) if nrhs else np.zeros(0)
    assert np.array_equal(seen, np.arange(nrhs))
    sizes = [b - a for a, b in blocks]
    assert max(sizes) - min(sizes) <= 1


def test_rhs_columns_rejects_bad_rank():
    with pytest.raises(ValueError):
        PT.rhs_columns(64, 2, 2)


def test_balance_problems_partition_and_bound():
    rng = np.random.default_rng(7)
    n = np.exp(rng.uniform(np.log(1000), np.log(50000), 256)).astype(int)
    cost = n.astype(float) ** 2
    for world in (1, 2, 3, 8):
        parts = PT.balance_problems(cost, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(n)))
        loads = np.array([cost[p].sum() for p in parts])
        lower = max(cost.sum() / world, cost.max())  # no assignment can beat this
        assert loads.max() <= 4.0 / 3.0 * lower
    # the greedy rule itself on a small case: 5, 4, 3, 3, 3 over two ranks
    assert PT.balance_problems([3, 5, 3, 4, 3], 2) == [[1, 2], [0, 3, 4]]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _gather_worker(rank, world, port, nrhs, out):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from elfmmlib3d_b200 import partition as P
    full = torch.arange(nrhs * 6, dtype=torch.float64).reshape(nrhs, 2, 3)
    a, b = P.rhs_columns(nrhs, world, rank)
    got = P.all_gather_columns(full[a:b].clone(), nrhs)
    out[rank] = bool(torch.equal(got, full))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("nrhs", [64, 7])
def test_all_gather_columns_two_ranks(nrhs):
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_gather_worker, args=(world, port, nrhs, out), nprocs=world, join=True)
        res = dict(out)
    assert res == {0: True, 1: True}
