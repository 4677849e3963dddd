"""Scene sharding host logic (CPU): the assignment, and a world-size-2 gloo
run in which each rank advances its own share of scenes with the oracle and
the gathered results equal a single-process run."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from mls_mpm_b200 import scenes, shard


def test_assign_balances_and_is_deterministic():
    rng = np.random.default_rng(0)
    costs = [int(x) for x in rng.integers(1, 1000, 50)]
    a = shard.assign(costs, 4)
    assert a == shard.assign(costs, 4)
    loads = [sum(c for c, r in zip(costs, a) if r == k) for k in range(4)]
    # LPT bound: max load <= (4/3 - 1/12) * optimum <= that bound of the mean
    assert max(loads) <= (4 / 3) * (sum(costs) / 4) + max(costs)
    assert sorted(i for k in range(4) for i in shard.my_items(costs, 4, k)) == list(range(50))


def test_assign_respects_capacity():
    assert shard.assign([5, 5, 5, 5], 2, capacity=10) in ([0, 1, 0, 1], [0, 1, 1, 0])
    with pytest.raises(ValueError):
        shard.assign([11, 1], 2, capacity=10)
    with pytest.raises(ValueError):
        shard.assign([6, 6, 6], 2, capacity=10)


def _scene_list():
    return [scenes.small_box(grid=g, n=n, seed=s) for g, n, s in
            (((16, 16, 16), 600, 1), ((20, 16, 18), 900, 2), ((16, 20, 16), 400, 3), ((18, 18, 18), 1200, 4),
             ((16, 16, 20), 300, 5))]


def _digests(indices, substeps=3):
    import oracle as O
    from mls_mpm_b200 import abi
    from mls_mpm_b200.batch import default_params
    out = {}
    for i in indices:
        sc = _scene_list()[i]
        st = O.new_state(sc)
        P = default_params(sc.grid, sc.n)
        for _ in range(substeps):
            O.substep(st, P, abi.WallParams())
        out[i] = O.digest(st)
    return out


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [sc.n for sc in _scene_list()]
        mine = shard.my_items(costs, world, rank)
        got = shard.gather(_digests(mine))
        if rank == 0:
            merged = {}
            for d in got:
                merged.update(d)
            q.put(merged)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_sharded_run_matches_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert merged == _digests(range(len(_scene_list())))
