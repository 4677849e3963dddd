"""Scene sharding on the device: two ranks (gloo, world size 2) each advance
their share of a scene list as one batch through the CUDA library, and the
results gathered on every rank match the oracle running each scene alone.

Both ranks share the one GPU this suite runs on.  Their kernels never wait
on each other: the only exchange is the host-side gather of results
(all_gather_object over gloo) after each rank has synchronised its batch."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

SUBSTEPS = 20
FIELDS = ("pos", "vel", "density")


def _scene_list():
    from mls_mpm_b200 import scenes
    # uneven counts and grids of the batched mix, kept small for the oracle
    return [scenes.batch_scene(3, i, n_min=2048, n_max=40000) for i in range(6)]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from mls_mpm_b200 import shard
        from mls_mpm_b200.batch import default_params
        sc = _scene_list()
        sb = shard.ShardedBatch(sc, SUBSTEPS, world, rank, params=lambda s: default_params(s.grid, s.n))
        sb.step(SUBSTEPS)
        sb.sync()
        got = sb.gather_results(lambda b, sid: {k: b.read(sid, k) for k in FIELDS})
        q.put((rank, sorted(sb.mine), got if rank == 0 else None))
        sb.batch.close()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_share_the_scene_list_and_match_the_oracle(gpu):
    import oracle as O
    from mls_mpm_b200 import abi
    from mls_mpm_b200.batch import default_params
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    mine = {r: m for r, m, _ in res}
    got = next(g for r, _, g in res if r == 0)
    sc = _scene_list()
    # every scene on exactly one rank, both ranks busy
    assert sorted(mine[0] + mine[1]) == list(range(len(sc))) and mine[0] and mine[1]
    assert sorted(got) == list(range(len(sc)))
    for i, s in enumerate(sc):
        st = O.new_state(s)
        P = default_params(s.grid, s.n)
        for _ in range(SUBSTEPS):
            O.substep(st, P, abi.WallParams(), threads=max(1, os.cpu_count() or 1))
        for k in FIELDS:
            assert np.array_equal(np.ascontiguousarray(got[i][k]).view(np.uint32),
                                  np.ascontiguousarray(st[k]).view(np.uint32)), (i, k)
