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


class _FakeBatch:
    """Stands in for the device batch in the host-path test: records what the
    rank built and returns a per-scene result computed on the host."""

    def __init__(self, particles, cells, scenes):
        self.capacity = (particles, cells, scenes)
        self.added = []
        self.steps = 0

    def add_scene(self, scene, params=None):
        self.added.append(scene)
        return len(self.added) - 1

    def step(self, k):
        self.steps += k

    def sync(self):
        pass

    def read(self, sid, name):
        sc = self.added[sid]
        return float(np.float64(sc.pos[:, :3]).sum()) + self.steps


def _sharded_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = _scene_list()
        sb = shard.ShardedBatch(sc, 7, world, rank, make_batch=_FakeBatch)
        b = sb.batch
        # this rank's batch holds exactly its share, sized to it
        assert b.capacity == (sum(sc[i].n for i in sb.mine), sum(sc[i].cells for i in sb.mine), len(sb.mine))
        sb.step(7)
        sb.sync()
        got = sb.gather_results(lambda batch, sid: batch.read(sid, "pos"))
        jobs = [(s, 10 + i) for i, s in enumerate(sc)]
        q.put((rank, sorted(sb.mine), got, shard.shard_jobs(jobs, world, rank)))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharded_batch_host_path():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sc = _scene_list()
    (r0, mine0, got0, jobs0), (r1, mine1, got1, jobs1) = res
    # the two shares partition the scenes, and both ranks gathered every result
    assert sorted(mine0 + mine1) == list(range(len(sc))) and not set(mine0) & set(mine1)
    want = {i: float(np.float64(s.pos[:, :3]).sum()) + 7 for i, s in enumerate(sc)}
    assert got0 == want and got1 == want
    assert sorted(jobs0 + jobs1) == list(range(len(sc))) and not set(jobs0) & set(jobs1)
