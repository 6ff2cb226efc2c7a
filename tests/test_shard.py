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


def _flow_worker(rank, world, port, out):
    """One rank of a sharded job: its scenes by placement, each stepped (the
    oracle stands in for the GPU engine here), results gathered by scene."""
    import torch.distributed as dist
    from diff_fem_b200 import scene as S
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        descs = [S.inverse_stiffness(nx=2 + k, ny=2, nz=2, seed=k) for k in range(5)]
        mine = my_scenes([d.n_tets for d in descs], world, rank)
        vals = []
        for i in mine:
            d = descs[i]
            x = d.x0.reshape(-1).copy()
            r = O.OracleScene(d).forward(x, np.zeros_like(x), n_steps=3)
            vals.append(float(np.abs(r["x"] - x).sum()))
        t = max_over_ranks(float(len(mine)))
        out[rank] = (mine, t, list(gather_by_scene(vals, mine, len(descs))))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_place_step_and_gather_scenes():
    """The multi-GPU flow of a sharded batch on CPU: each rank steps only its
    share, the job time is the maximum over ranks, and the gathered per-scene
    results equal the scenes stepped in one process."""
    from diff_fem_b200 import scene as S
    from oracle import oracle as O
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_flow_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    (m0, t0, v0), (m1, t1, v1) = out[0], out[1]
    assert sorted(m0 + m1) == list(range(5)) and not set(m0) & set(m1) and m0 and m1
    assert t0 == t1 == float(max(len(m0), len(m1)))
    ref = []
    for k in range(5):
        d = S.inverse_stiffness(nx=2 + k, ny=2, nz=2, seed=k)
        x = d.x0.reshape(-1).copy()
        ref.append(float(np.abs(O.OracleScene(d).forward(x, np.zeros_like(x), n_steps=3)["x"] - x).sum()))
    assert v0 == v1 == ref
