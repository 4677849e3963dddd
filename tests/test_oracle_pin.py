"""The oracle against the reference: golden digests produced by the reference
pin (the reference's WGSL compiled on the host), and — where the reference
checkout exists — the pin itself, substep by substep."""
import json
import os

import numpy as np
import pytest

import oracle as O
import scenarios
from mls_mpm_b200.abi import Params, RayParams
from runner import cpu_run, diff_report

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


@pytest.mark.parametrize("name", sorted(scenarios.SCENARIOS))
def test_oracle_matches_golden(name):
    sc = scenarios.SCENARIOS[name]()
    gold = GOLDEN["scenarios"][name]
    assert gold["n"] == sc.scene.n and gold["substeps"] == sc.substeps
    for s, st in enumerate(cpu_run(sc, "oracle", threads=4)):
        d = O.digest(st)
        bad = [k for k, v in gold["steps"][s]["digest"].items() if d.get(k) != v]
        assert not bad, f"{name} substep {s}: {bad} differ from the reference pin's digests"


@pytest.mark.parametrize("name", ["walls_hand_diffuse", "saturate", "crowded"])
def test_oracle_matches_reference_pin(name):
    if not O.ref_available():
        pytest.skip("reference pin not built here (no reference checkout)")
    sc = scenarios.SCENARIOS[name]()
    for s, (a, b) in enumerate(zip(cpu_run(sc, "oracle"), cpu_run(sc, "ref"))):
        bad = diff_report(a, b)
        assert not bad, f"substep {s}: {bad}"


def test_oracle_threads_bit_identical():
    """Integer-atomic grids make the multi-threaded oracle bit-identical."""
    sc = scenarios.walls_hand_diffuse()
    for s, (a, b) in enumerate(zip(cpu_run(sc, "oracle", threads=1), cpu_run(sc, "oracle", threads=4))):
        assert not diff_report(a, b), f"substep {s}"


def test_f64_drift_reported_and_small():
    """The binary64 evaluation of the same passes (the drift reference):
    after a few substeps the f32 state stays close to it."""
    sc = scenarios.dam_break_64(substeps=5)
    a = O.new_state(sc.scene)
    b = O.to_f64(O.new_state(sc.scene))
    for P, W, H, dims, gen, adv in sc.frames():
        O.substep(a, P, W, H, dims)
        O.substep(b, P, W, H, dims, impl="f64")
    dpos = np.abs(a["pos"][:, :3].astype(np.float64) - b["pos"][:, :3]).max()
    assert np.isfinite(dpos) and dpos < 1e-3, dpos


def _params(n, grid=(16, 16, 16)):
    p = Params()
    p.grid_X, p.grid_Y, p.grid_Z = grid
    p.particle_num = n
    return p


def test_compact_and_raycast_match_reference_pin():
    rng = np.random.default_rng(5)
    n = 500
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(2, 14, (n, 3))
    vel = rng.standard_normal((n, 4)).astype(np.float32)
    mass = np.ones(n, np.float32)
    d = np.array([0.3, -0.2, 0.9])
    d /= np.linalg.norm(d)
    ray = RayParams(8.0, 8.0, 0.0, 2.5, *d.astype(np.float32), 0.0)
    P = _params(n)
    cnt, po, vo, mo = O.compact(P, ray, pos, vel, mass)
    assert 0 < cnt < n
    hit = O.raycast(P, ray, pos)
    assert hit != 0xFFFFFFFF
    if O.ref_available():
        cnt2, po2, vo2, mo2 = O.compact(P, ray, pos, vel, mass, impl="ref")
        assert cnt == cnt2 and np.array_equal(po, po2) and np.array_equal(vo, vo2)
        assert O.raycast(P, ray, pos, impl="ref") == hit
