"""Overpacked cells: many particles per cell put the lanes of a warp on the
same shared-memory accumulators in P2G_MASS and P2G_MOM, and the integer
grid sums (shaders.js:242-371, one atomicAdd per contribution in the
reference) must stay bit-identical to the oracle however the adds interleave.

* One scene at 150 particles per cell of its block, diffuse on: every array
  after each of 40 substeps.
* A batch of the batched mix's most overpacked scenes (110-560 particles per
  cell) with its two sparsest ones: each scene against the oracle alone.
"""
import os

import numpy as np
import pytest

import oracle as O
import scenarios as S
from mls_mpm_b200 import scenes
from mls_mpm_b200.batch import Batch
from runner import GpuScene, diff_report

pytestmark = pytest.mark.gpu

THREADS = max(1, os.cpu_count() or 1)
FLUID = ("pos", "vel", "affine", "density", "cell_mv", "cell_mass", "cell_mv_f32", "cell_mass_f32")


def dense_block(per_cell=150, edge=48, block=(12, 12, 12), seed=11):
    """A 12^3-cell block from cell 2 filled with `per_cell` particles per cell
    at seeded uniform positions."""
    n = per_cell * block[0] * block[1] * block[2]
    r = scenes.uniform01(seed, 3 * n).reshape(n, 3)
    pos = (2.0 + r * np.asarray(block, np.float64)).astype(np.float32)
    return scenes.Scene((edge, edge, edge), pos, name=f"dense_{per_cell}", substeps=40)


def test_dense_block_bit_exact_every_substep(gpu):
    sc = dense_block()
    scn = S.Scenario(sc.name, sc, 40, diffuse_max=32768)
    g = GpuScene(gpu, sc, scn.diffuse_max)
    st = O.new_state(sc, scn.diffuse_max)
    try:
        for s, (P, W, H, dims, gen, adv) in enumerate(scn.frames()):
            g.frame(P, W, H, dims)
            O.substep(st, P, W, H, dims, gen, adv, threads=THREADS)
            bad = diff_report(g.state(), st)
            assert not bad, f"substep {s}: {bad}"
    finally:
        g.close()


def _densest(count):
    mix = [(i, scenes.batch_scene(0, i)) for i in range(64)]
    mix.sort(key=lambda t: t[1].n / t[1].block_cells)
    return [sc for _, sc in mix[:2]] + [sc for _, sc in mix[-count:]]


def test_dense_batch_scenes_match_oracle_alone(gpu):
    substeps, checks = 30, (1, 10, 30)
    scs = _densest(5)
    assert scs[-1].n / scs[-1].block_cells > 500
    scns = [S.Scenario(s.name, s, substeps) for s in scs]
    frames = [[(P, W, H, d) for P, W, H, d, _, _ in s.frames()] for s in scns]
    b = Batch(sum(s.n for s in scs), sum(s.cells for s in scs), len(scs))
    try:
        ids = [b.add_scene(s, params=frames[i][0][0]) for i, s in enumerate(scs)]
        got = {}
        for t in range(substeps):
            b.step(1)
            if t + 1 in checks:
                got[t + 1] = [{k: b.read(sid, k) for k in FLUID} for sid in ids]
    finally:
        b.close()
    for i, s in enumerate(scs):
        st = O.new_state(s)
        for t, (P, W, H, d) in enumerate(frames[i]):
            O.substep(st, P, W, H, d, threads=THREADS)
            if t + 1 in checks:
                bad = diff_report({k: st[k] for k in FLUID}, got[t + 1][i])
                assert not bad, (s.name, t + 1, bad)
