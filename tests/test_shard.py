"""Scene placement across ranks (host logic of the multi-GPU path), checked
with two gloo ranks on the CPU: the split is complete, disjoint, identical on
every rank and balanced; the time reduction is the maximum over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from diff_fem_b200.shard import assign_scenes, gather_by_scene, max_over_ranks, my_scenes


def test_assign_is_a_balanced_partition():
    rng = np.random.default_rng(7)
    costs = np.exp(rng.uniform(np.log(1e3), np.log(5e4), 256))
    for world in (1, 2, 3, 8):
        parts = assign_scenes(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(costs.size))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max() + 1e-9  # LPT bound
        assert parts == assign_scenes(costs, world)  # deterministic


def test_assign_edge_cases():
    assert assign_scenes([], 4) == [[], [], [], []]
    assert assign_scenes([5.0], 3) == [[0], [], []]
    assert assign_scenes([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        assign_scenes([1.0], 0)
    with pytest.raises(ValueError):
        my_scenes([1.0], 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = my_scenes(costs, world, rank)
        t = max_over_ranks(1.0 + rank)
        vals = gather_by_scene([10.0 * i for i in mine], mine, len(costs))
        out[rank] = (mine, t, list(vals))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_reduce():
    costs = list(np.linspace(1.0, 9.0, 11))
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), costs, out), nprocs=world, join=True)
    mine0, t0, v0 = out[0]
    mine1, t1, v1 = out[1]
    assert sorted(mine0 + mine1) == list(range(len(costs)))
    assert not set(mine0) & set(mine1)
    assert t0 == t1 == 2.0
    assert v0 == v1 == [10.0 * i for i in range(len(costs))]
