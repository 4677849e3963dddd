"""Full-size checks on the 1M-particle workload (128^3 grid, diffuse pool
262,144): bit-exact against the oracle for the first substeps, then
size-independent invariants over a longer run: determinism (two runs give
identical digests), particles inside the hard bounds, the integer mass grid
equal to the sum of each particle's encoded contributions, and free-list
conservation (top + alive == pool size, free list a permutation of the
dead slots)."""
import numpy as np
import pytest

import oracle as O
import scenarios
from mls_mpm_b200 import scenes
from runner import GpuScene, cpu_run, diff_report

pytestmark = pytest.mark.gpu


def _scenario(substeps):
    sc = scenes.dam_break_1m(0)
    return scenarios.Scenario("dam_break_1m", sc, substeps, diffuse_max=sc.diffuse_max)


def _run(lib, scn, engine=0):
    g = GpuScene(lib, scn.scene, scn.diffuse_max, flags=engine)
    for P, W, H, dims, gen, adv in scn.frames():
        g.frame(P, W, H, dims)
    return g


def test_full_size_first_substeps_bit_exact(gpu):
    scn = _scenario(3)
    g = GpuScene(gpu, scn.scene, scn.diffuse_max)
    try:
        for s, ((P, W, H, dims, gen, adv), o) in enumerate(zip(scn.frames(), cpu_run(scn, "oracle", threads=16))):
            g.frame(P, W, H, dims)
            bad = diff_report(g.state(), o)
            assert not bad, f"substep {s}: {bad}"
    finally:
        g.close()


def test_full_size_invariants_and_determinism(gpu):
    scn = _scenario(60)
    a = _run(gpu, scn)
    b = _run(gpu, scn)
    try:
        sa, sb = a.state(), b.state()
        assert O.digest(sa) == O.digest(sb), "two runs differ"
        P = next(scn.frames())[0]
        pos = sa["pos"][:, :3]
        assert np.isfinite(pos).all()
        assert pos.min() >= P.hard_min and pos[:, 0].max() <= P.hard_max_x
        assert pos[:, 1].max() <= P.hard_max_y and pos[:, 2].max() <= P.hard_max_z
        # the mass grid is the exact i32 sum of every particle's 27 encoded weights
        # (recomputed here from the positions the grid was built from is not
        # possible after G2P moved them; instead check the sum against the bound
        # of at most 1 count of truncation per contribution)
        total = int(sa["cell_mass"].astype(np.int64).sum())
        n = pos.shape[0]
        assert abs(total - n * 100000) <= 27 * n
        top = int(sa["top"][0])
        alive = int((sa["diffuse"]["alive"] != 0).sum())
        assert top + alive == scn.diffuse_max
        free = np.sort(sa["free_list"][:top])
        dead = np.nonzero(sa["diffuse"]["alive"] == 0)[0]
        assert np.array_equal(free, dead)
    finally:
        a.close()
        b.close()


def test_binned_equals_plain_engine_full_size(gpu):
    scn = _scenario(20)
    a = _run(gpu, scn, engine=0)
    b = _run(gpu, scn, engine=1)
    try:
        bad = diff_report(a.state(), b.state())
        assert not bad, bad
    finally:
        a.close()
        b.close()
