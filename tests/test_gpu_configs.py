"""The benchmark configurations at their own sizes and lengths, bit-exact
against the oracle (the f32 restatement of the reference's passes,
shaders.js:196-997 in the order of fluid-gpu.js:663-682 and
diffuse-gpu.js:148-166; the oracle itself is pinned to the reference's WGSL in
test_oracle_pin.py):

* 1M-particle dam break (128^3 grid, 262,144 diffuse slots): every array after
  each of the first 50 substeps, then at checkpoints up to all 500 substeps.
* 8M-particle dam break with a falling sphere (256x128x256, 1,048,576 diffuse
  slots): every array after each of the first 3 substeps, and after 10.
* Batched form: 8 scenes of the batched mix (uneven counts, grids 32-128,
  overpacked blocks) in one batch for the full 200 substeps, each scene
  against the oracle running it alone at checkpoints.
* Served form: 8 jobs of the served mix (8k-2M particles, grids 32-192) with
  Poisson arrivals under a budget that holds only part of them at once,
  substep counts cut to 5-40; every job's final state against the oracle alone.

The 64^3 configuration runs its full 200 substeps in test_gpu_parity.py
(every substep, both engines, and the reference pin's golden digests).
"""
import os

import numpy as np
import pytest

import oracle as O
import scenarios as S
from mls_mpm_b200 import abi, scenes
from mls_mpm_b200.batch import Batch, default_params
from mls_mpm_b200.server import Server
from runner import GpuScene, diff_report

pytestmark = pytest.mark.gpu

THREADS = max(1, os.cpu_count() or 1)
FLUID = ("pos", "vel", "affine", "density", "cell_mv", "cell_mass", "cell_mv_f32", "cell_mass_f32")


def _compare_run(lib, scn, every, checkpoints):
    """GPU and oracle side by side; full-state compare after each substep in
    `every` and at `checkpoints`."""
    g = GpuScene(lib, scn.scene, scn.diffuse_max)
    st = O.new_state(scn.scene, scn.diffuse_max)
    checked = 0
    try:
        for s, (P, W, H, dims, gen, adv) in enumerate(scn.frames()):
            g.frame(P, W, H, dims)
            O.substep(st, P, W, H, dims, gen, adv, threads=THREADS)
            if s < every or (s + 1) in checkpoints:
                bad = diff_report(g.state(), st)
                assert not bad, f"{scn.name} substep {s}: {bad}"
                checked += 1
        return g.state(), st, checked
    finally:
        g.close()


def test_dam_break_1m_bit_exact_50_substeps_then_to_500(gpu):
    sc = scenes.dam_break_1m(0)
    scn = S.Scenario("dam_break_1m", sc, 500, diffuse_max=sc.diffuse_max)
    got, want, checked = _compare_run(gpu, scn, 50, (100, 200, 300, 400, 500))
    assert checked == 55
    # the run did spawn and kill diffuse particles
    alive = int((want["diffuse"]["alive"] != 0).sum())
    assert 0 < alive < sc.diffuse_max
    assert int(want["top"][0]) + alive == sc.diffuse_max


def test_dam_break_sphere_8m_bit_exact(gpu):
    sc = scenes.dam_break_sphere_8m(0)
    assert sc.n == 8388608 and sc.grid == (256, 128, 256)
    assert (sc.vel[:, 1] < 0).sum() > 0       # the falling sphere
    scn = S.Scenario("dam_break_sphere_8m", sc, 10, diffuse_max=sc.diffuse_max)
    _compare_run(gpu, scn, 3, (10,))


def _oracle_alone(scn, frames, checkpoints):
    st = O.new_state(scn.scene)
    out = {}
    for i, (P, W, H, d) in enumerate(frames):
        O.substep(st, P, W, H, d, threads=THREADS)
        if i + 1 in checkpoints:
            out[i + 1] = {k: st[k].copy() for k in FLUID}
    return out


def test_batch_mix_draw_each_scene_matches_oracle(gpu):
    substeps, checks = 200, (1, 20, 100, 200)
    scns = [S.Scenario(f"batch_{i}", scenes.batch_scene(0, i), substeps) for i in range(8)]
    frames = [[(P, W, H, d) for P, W, H, d, _, _ in s.frames()] for s in scns]
    b = Batch(sum(s.scene.n for s in scns), sum(s.scene.cells for s in scns), len(scns))
    try:
        ids = [b.add_scene(s.scene, params=frames[i][0][0]) for i, s in enumerate(scns)]
        got = {}
        for t in range(substeps):
            b.step(1)
            if t + 1 in checks:
                got[t + 1] = [{k: b.read(sid, k) for k in FLUID} for sid in ids]
    finally:
        b.close()
    for i, s in enumerate(scns):
        want = _oracle_alone(s, frames[i], checks)
        for c in checks:
            bad = diff_report(want[c], got[c][i])
            assert not bad, (s.name, c, bad)


def test_served_mix_jobs_match_oracle_alone(gpu):
    jobs = [scenes.serve_job(0, i, steps_min=5, steps_max=40) for i in range(8)]
    arrivals = scenes.poisson_arrivals(200.0, len(jobs), 0)
    biggest = max(sc.n for sc, _ in jobs)
    biggest_cells = max(sc.cells for sc, _ in jobs)
    # room for about two of the largest jobs at once: later arrivals wait for memory
    budget = int(Batch.footprint(int(2.2 * biggest), int(2.2 * biggest_cells), 16))
    srv = Server(budget, scene_capacity=16, cells_per_particle=biggest_cells / biggest,
                 flags=abi.SERVER_KEEP_STATE)
    try:
        ids = [srv.submit(default_params(sc.grid, sc.n), sc.pos, sc.mass, steps, arrival_s=float(arrivals[i]),
                          vel4=sc.vel) for i, (sc, steps) in enumerate(jobs)]
        st = srv.run()
        assert st.jobs == len(jobs)
        assert st.particle_updates == sum(sc.n * s for sc, s in jobs)
        assert st.max_active < len(jobs)            # the budget made jobs wait
        for (sc, steps), j in zip(jobs, ids):
            want = O.new_state(sc)
            P = default_params(sc.grid, sc.n)
            for _ in range(steps):
                O.substep(want, P, abi.WallParams(), threads=THREADS)
            for k in ("pos", "vel", "density"):
                got = srv.download(j, k)
                assert np.array_equal(got.view(np.uint32), np.ascontiguousarray(want[k]).view(np.uint32)), \
                    (sc.name, sc.n, k)
    finally:
        srv.close()
