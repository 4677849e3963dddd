"""CUDA path (through the C ABI) against the oracle, every substep, bit-exact.

Tolerance: integer grids (cell_mv, cell_mass) must be bit-identical; f32
particle and grid state is required to be bit-identical too (the kernels
follow the reference's operation order with no FMA contraction and IEEE
division/sqrt), which is stricter than the 1e-5 relative per-step bound the
path promises; REL_TOL is the documented fallback bound, applied only to the
non-default eos_power != 1 path where CUDA powf replaces libm pow.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
import scenarios
from runner import cpu_run, diff_report, gpu_run

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


@pytest.mark.parametrize("engine", ["binned", "plain"])
@pytest.mark.parametrize("name", sorted(scenarios.SCENARIOS))
def test_gpu_matches_oracle_every_substep(gpu, name, engine):
    sc = scenarios.SCENARIOS[name]()
    for s, (g, o) in enumerate(zip(gpu_run(gpu, sc, engine), cpu_run(sc, "oracle", threads=8))):
        bad = diff_report(g, o)
        assert not bad, f"{name} [{engine}] substep {s}: {bad}"


@pytest.mark.parametrize("engine", ["binned", "plain"])
@pytest.mark.parametrize("name", sorted(scenarios.SCENARIOS))
def test_gpu_matches_reference_golden(gpu, name, engine):
    sc = scenarios.SCENARIOS[name]()
    gold = GOLDEN["scenarios"][name]["steps"]
    for s, g in enumerate(gpu_run(gpu, sc, engine)):
        d = O.digest(g)
        bad = [k for k, v in gold[s]["digest"].items() if d.get(k) != v]
        assert not bad, f"{name} substep {s}: {bad}"


def test_gpu_eos_power_two_within_tolerance(gpu):
    """eos_power != 1 uses CUDA powf; state must stay within REL_TOL per step."""
    sc = scenarios.walls_hand_diffuse()
    sc.substeps = 1
    frames = list(sc.frames())
    P, W, H, dims, gen, adv = frames[0]
    P.eos_power = 2.0
    st = O.new_state(sc.scene, sc.diffuse_max)
    O.substep(st, P, W, H, dims, gen, adv)
    from runner import GpuScene
    g = GpuScene(gpu, sc.scene, sc.diffuse_max)
    try:
        g.frame(P, W, H, dims)
        for k in ("pos", "vel", "density"):
            a, b = g.read(k).astype(np.float64), st[k].astype(np.float64)
            err = np.abs(a - b) / np.maximum(np.abs(b), 1.0)
            assert err.max() <= REL_TOL, (k, err.max())
    finally:
        g.close()


def test_fluidgpu_class_drop_in(gpu):
    """The FluidGPU/DiffuseGPU mirror drives the same path as the raw ABI."""
    from mls_mpm_b200 import DiffuseGPU, FluidGPU
    sc = scenarios.walls_hand_diffuse()
    fl = FluidGPU.from_scene(sc.scene)
    dif = DiffuseGPU(sc.diffuse_max).initGPU(0, fl)
    ref = cpu_run(sc, "oracle")
    for s in range(10):
        scenarios._walls_moving(s, fl._walls)
        pos, vel, r, strength, active, eye = scenarios._hand_sweep(s)
        fl.updateHand(pos, vel, r, strength, active, eye)
        fl.simFrame()
        o = next(ref)
        assert np.array_equal(fl.read("pos"), o["pos"]), s
        assert np.array_equal(fl.read("cell_mass"), o["cell_mass"]), s
    want = sc.diffuse_max - int(o["top"][0])
    assert dif.readAliveCount() == want
    # the asynchronous pair: a readback queued after the step, read once it landed
    dif.requestDebugReadback()
    fl.sync()
    assert dif.pollDebug() == want
    fl.destroy()
