"""The serving loop (mpm_server_*): every job's final state is bit-exact
against the oracle running that scene alone, whatever else shared its
substeps; admission follows arrival order and the memory budget; latencies
are consistent with arrival, admission and completion."""
import numpy as np
import pytest

import oracle as O
from mls_mpm_b200 import abi, scenes
from mls_mpm_b200.batch import Batch, default_params
from mls_mpm_b200.server import Server

pytestmark = pytest.mark.gpu


def job_mix(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        g = (int(rng.integers(16, 33)), int(rng.integers(16, 29)), int(rng.integers(16, 33)))
        n = int(rng.integers(200, 2500))
        sc = scenes.small_box(grid=g, n=n, seed=100 + i, name=f"job{i}")
        out.append((sc, int(rng.integers(1, 14))))
    return out


def oracle_final(sc, substeps):
    st = O.new_state(sc)
    P = default_params(sc.grid, sc.n)
    for _ in range(substeps):
        O.substep(st, P, abi.WallParams())
    return st


@pytest.mark.parametrize("budget_scale", [1000.0, 2.2])
def test_served_jobs_match_oracle_alone(gpu, budget_scale):
    jobs = job_mix(12, 3)
    biggest = max(sc.n for sc, _ in jobs)
    biggest_cells = max(sc.cells for sc, _ in jobs)
    # budget_scale 2.2: room for about two of the largest jobs at once, so most wait in the queue
    budget = int(Batch.footprint(int(budget_scale * biggest), int(budget_scale * biggest_cells), 16))
    srv = Server(budget, scene_capacity=16, cells_per_particle=biggest_cells / biggest,
                 flags=abi.SERVER_KEEP_STATE)
    try:
        ids = []
        for i, (sc, steps) in enumerate(jobs):
            P = default_params(sc.grid, sc.n)
            ids.append(srv.submit(P, sc.pos, sc.mass, steps, arrival_s=0.002 * i, vel4=sc.vel))
        st = srv.run()
        assert st.jobs == len(jobs)
        assert st.particle_updates == sum(sc.n * s for sc, s in jobs)
        res = [srv.job(j) for j in ids]
        for r in res:
            assert r.done and r.admit_s >= r.arrival_s and r.finish_s > r.admit_s
        # FIFO admission: admit times follow arrival order
        admits = [r.admit_s for r in res]
        assert admits == sorted(admits)
        assert 1 <= st.max_active <= len(jobs)
        for (sc, steps), j in zip(jobs, ids):
            want = oracle_final(sc, steps)
            for k in ("pos", "vel", "density"):
                got = srv.download(j, k)
                w = want[k]
                assert np.array_equal(got.view(np.uint32), np.ascontiguousarray(w).view(np.uint32)), (sc.name, k)
    finally:
        srv.close()


def test_server_rejects_jobs_that_never_fit(gpu):
    srv = Server(int(Batch.footprint(10_000, 50_000, 4)), scene_capacity=4, cells_per_particle=5.0)
    try:
        sc = scenes.small_box(grid=(64, 64, 64), n=1000)
        with pytest.raises(abi.MpmError) as e:
            srv.submit(default_params(sc.grid, sc.n), sc.pos, sc.mass, 5, 0.0)
        assert e.value.status == 9
        with pytest.raises(abi.MpmError):
            sc2 = scenes.small_box(grid=(16, 16, 16), n=1000)
            srv.submit(default_params(sc2.grid, sc2.n), sc2.pos, sc2.mass, 0, 0.0)
    finally:
        srv.close()
