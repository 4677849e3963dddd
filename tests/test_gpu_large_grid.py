"""A world of more tiles than one block scans (256x128x256 cells = 8,192 tiles
of 16x8x8, eight groups of 1,024): the binning runs its separate grid-list and
two-level scan kernels.  Bit-exact against the oracle for the first substeps
(diffuse on), and the binned engine equal to the plain engine afterwards."""
import pytest

import scenarios
from mls_mpm_b200 import scenes
from runner import GpuScene, cpu_run, diff_report

pytestmark = pytest.mark.gpu


def _scenario(substeps):
    # the 256x128x256 grid with a dam block only (no sphere), 8 particles per
    # cell in a 24 x 48-cell footprint: 524,288 particles.  The full 8M-particle
    # configuration with its falling sphere is in test_gpu_configs.py.
    n = 1 << 19
    nx, ny = 48, 96
    nz = -(-n // (nx * ny))
    sc = scenes.dam_break((256, 128, 256), (2.0, 2.0, 2.0), (nx, ny, nz), n, seed=3, name="large_grid",
                          substeps=substeps, diffuse_max=65536)
    return scenarios.Scenario("large_grid", sc, substeps, diffuse_max=sc.diffuse_max)


def test_large_grid_first_substeps_bit_exact(gpu):
    scn = _scenario(3)
    g = GpuScene(gpu, scn.scene, scn.diffuse_max)
    try:
        for s, ((P, W, H, dims, gen, adv), o) in enumerate(zip(scn.frames(), cpu_run(scn, "oracle", threads=16))):
            g.frame(P, W, H, dims)
            bad = diff_report(g.state(), o)
            assert not bad, f"substep {s}: {bad}"
    finally:
        g.close()


def test_large_grid_binned_equals_plain(gpu):
    scn = _scenario(12)
    a = GpuScene(gpu, scn.scene, scn.diffuse_max, flags=0)
    b = GpuScene(gpu, scn.scene, scn.diffuse_max, flags=1)
    try:
        for P, W, H, dims, gen, adv in scn.frames():
            a.frame(P, W, H, dims)
            b.frame(P, W, H, dims)
        bad = diff_report(a.state(), b.state())
        assert not bad, bad
    finally:
        a.close()
        b.close()
