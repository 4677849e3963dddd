"""Batches of scenes (mpm_batch_*) against the oracle and against the same
scenes run alone: bit-exact per scene, across graph / no-graph / autotuned
launch shapes, and through removals and additions between substeps."""
import ctypes

import numpy as np
import pytest

import oracle as O
import scenarios as S
from mls_mpm_b200 import abi, scenes
from mls_mpm_b200.abi import MpmError
from mls_mpm_b200.batch import Batch
from runner import GpuScene, diff_report

pytestmark = pytest.mark.gpu

FLUID = ("pos", "vel", "affine", "density", "cell_mv", "cell_mass", "cell_mv_f32", "cell_mass_f32")


def _copy(c):
    return None if c is None else type(c).from_buffer_copy(c)


def script(scn, substeps):
    """Per-substep (P, W, H, dims) for `substeps` substeps, repeating the last
    uniforms once the scenario's own script ends."""
    fr = [(_copy(P), _copy(W), _copy(H), None if d is None else list(d)) for P, W, H, d, _, _ in scn.frames()]
    if not fr:
        fr = [(None, None, None, None)]
    return [fr[min(i, len(fr) - 1)] for i in range(substeps)]


def oracle_states(scn, frames, checkpoints):
    st = O.new_state(scn.scene)
    out = {}
    for i, (P, W, H, d) in enumerate(frames):
        O.substep(st, P, W, H, d)
        if i + 1 in checkpoints:
            out[i + 1] = {k: st[k].copy() for k in FLUID}
    return out


def mix():
    return [S.walls_hand_diffuse(), S.saturate(), S.empty(), S.crowded(), S.dam_break_64(10)]


def set_uniforms(b, sid, P, W, H, d):
    b.set_params(sid, P)
    b.set_walls(sid, W)
    if H is not None:
        b.set_hand(sid, H, int(any(d) and H.is_on != 0), d)


def read_all(b, sid):
    return {k: b.read(sid, k) for k in FLUID}


def new_batch(flags=0, scene_capacity=8, particles=100_000, cells=400_000):
    return Batch(particles, cells, scene_capacity, flags=flags)


def run_batch(flags, scns, substeps, checkpoints):
    frames = [script(s, substeps) for s in scns]
    b = new_batch(flags)
    try:
        ids = [b.add_scene(s.scene, params=frames[i][0][0]) for i, s in enumerate(scns)]
        got = {}
        for t in range(substeps):
            for i, sid in enumerate(ids):
                set_uniforms(b, sid, *frames[i][t])
            b.step(1)
            if t + 1 in checkpoints:
                got[t + 1] = [read_all(b, sid) for sid in ids]
        info = b.info()
        return got, frames, info
    finally:
        b.close()


def test_batch_matches_oracle_per_scene(gpu):
    scns = mix()
    substeps, checks = 12, (1, 5, 12)
    got, frames, info = run_batch(0, scns, substeps, checks)
    assert info.scenes == len(scns) and info.particles == sum(s.scene.n for s in scns)
    for i, s in enumerate(scns):
        want = oracle_states(s, frames[i], checks)
        for c in checks:
            assert diff_report(want[c], got[c][i]) == [], (s.name, c)


def test_batch_graph_nograph_autotune_identical(gpu):
    scns = [S.dam_break_64(10), S.crowded(), S.saturate()]
    substeps = 30   # enough substeps for the tuner to finish its trials
    ref, _, _ = run_batch(abi.BATCH_NO_GRAPH, scns, substeps, (substeps,))
    for flags in (0, abi.BATCH_AUTOTUNE):
        got, _, info = run_batch(flags, scns, substeps, (substeps,))
        for i in range(len(scns)):
            assert diff_report(ref[substeps][i], got[substeps][i]) == [], (flags, scns[i].name)


def test_scene_alone_equals_scene_in_mix(gpu):
    scns = [S.walls_hand_diffuse(), S.crowded(), S.dam_break_64(10)]
    substeps = 10
    got, frames, _ = run_batch(0, scns, substeps, (substeps,))
    for i, s in enumerate(scns):
        g = GpuScene(gpu, s.scene)
        try:
            for P, W, H, d in frames[i]:
                g.frame(P, W, H, d)
            alone = {k: g.read(k) for k in FLUID}
        finally:
            g.close()
        assert diff_report(alone, got[substeps][i]) == [], s.name


def test_remove_and_add_between_substeps(gpu):
    a, bb, c = S.crowded(), S.saturate(), S.walls_hand_diffuse()
    d = S.Scenario("late", scenes.small_box(grid=(28, 22, 26), n=4000, seed=21, name="late"), 8)
    fa, fb, fc, fd = script(a, 12), script(bb, 12), script(c, 12), script(d, 8)
    b = new_batch()
    try:
        ia, ib, ic = b.add_scene(a.scene, fa[0][0]), b.add_scene(bb.scene, fb[0][0]), b.add_scene(c.scene, fc[0][0])
        for t in range(4):
            for sid, f in ((ia, fa), (ib, fb), (ic, fc)):
                set_uniforms(b, sid, *f[t])
            b.step(1)
        b.remove(ib)
        # the removed scene's slots stay in the layout until the next substep;
        # with this capacity the new scene still fits behind them
        idd = b.add_scene(d.scene, fd[0][0])
        for t in range(4, 12):
            for sid, f in ((ia, fa), (ic, fc)):
                set_uniforms(b, sid, *f[t])
            set_uniforms(b, idd, *fd[t - 4])
            b.step(1)
        got = {n: read_all(b, sid) for n, sid in (("a", ia), ("c", ic), ("d", idd))}
        assert b.info().scenes == 3
    finally:
        b.close()
    assert diff_report(oracle_states(a, fa, (12,))[12], got["a"]) == []
    assert diff_report(oracle_states(c, fc, (12,))[12], got["c"]) == []
    assert diff_report(oracle_states(d, fd, (8,))[8], got["d"]) == []


def test_batch_capacity_errors(gpu):
    b = Batch(10_000, 100_000, 3)
    try:
        a = scenes.small_box(grid=(16, 16, 16), n=3000, seed=1)
        big = scenes.small_box(grid=(24, 20, 22), n=6000, seed=2)
        tiny = scenes.small_box(grid=(16, 16, 16), n=100, seed=3)
        b.add_scene(a)
        ib = b.add_scene(big)
        b.add_scene(tiny)
        with pytest.raises(MpmError) as e:
            b.add_scene(tiny)        # scene slots exhausted
        assert e.value.status == 9
        with pytest.raises(MpmError) as e:
            b.remove(7)              # unknown scene
        assert e.value.status == 1
        b.step(1)
        b.remove(ib)
        with pytest.raises(MpmError) as e:
            b.add_scene(big)         # fits in particles, but the layout still holds the removed scene
        assert e.value.status == 7
        b.step(1)
        b.add_scene(big)
        b.step(2)
        assert b.info().particles == 9100
    finally:
        b.close()


def test_chunk_size_switch_between_substeps(gpu):
    """A world that grows past the size where 512-particle chunks fill the
    chunk kernels' grid (about 300k particles on 148 SMs) switches from
    one-pass to full-size chunks between substeps, and back after a removal;
    every scene stays bit-exact against the oracle through both switches."""
    a = S.crowded()
    big = S.Scenario("big", scenes.small_box(grid=(96, 64, 96), n=400_000, seed=5, name="big"), 6)
    fa, fb = script(a, 12), script(big, 6)
    b = new_batch(particles=600_000, cells=1_500_000)
    try:
        ia = b.add_scene(a.scene, fa[0][0])
        for t in range(3):                      # a small world: one-pass chunks
            set_uniforms(b, ia, *fa[t])
            b.step(1)
        ib = b.add_scene(big.scene, fb[0][0])   # past the threshold: full-size chunks
        for t in range(3, 9):
            set_uniforms(b, ia, *fa[t])
            set_uniforms(b, ib, *fb[t - 3])
            b.step(1)
        got_b = read_all(b, ib)
        b.remove(ib)                            # small again
        for t in range(9, 12):
            set_uniforms(b, ia, *fa[t])
            b.step(1)
        got_a = read_all(b, ia)
    finally:
        b.close()
    assert diff_report(oracle_states(a, fa, (12,))[12], got_a) == []
    assert diff_report(oracle_states(big, fb, (6,))[6], got_b) == []


def test_scene_churn_keeps_every_survivor_exact(gpu):
    """Scenes added and removed between substeps over many cycles, so cell,
    tile and id ranges are freed and reused while the other scenes keep the
    binning counts G2P left them: every scene alive at the end matches the
    oracle for the substeps it lived through."""
    rng = np.random.default_rng(7)
    b = new_batch(scene_capacity=6, particles=60_000, cells=400_000)
    live = {}   # scene id -> [scenario, frames, substeps done]

    def step_all():
        for sid, (scn, fr, k) in live.items():
            set_uniforms(b, sid, *fr[k])
        b.step(1)
        for sid in live:
            live[sid][2] += 1

    try:
        for cycle in range(18):
            if len(live) < 5:
                grid = tuple(int(x) for x in rng.integers(16, 33, 3))
                sc = scenes.small_box(grid=grid, n=int(rng.integers(500, 4000)), seed=int(rng.integers(1, 1000)),
                                      name=f"c{cycle}")
                scn = S.Scenario(f"c{cycle}", sc, 40)
                fr = script(scn, 40)
                live[b.add_scene(sc, fr[0][0])] = [scn, fr, 0]
            step_all()
            if cycle % 3 == 2 and len(live) > 2:
                victim = sorted(live)[int(rng.integers(0, len(live)))]
                b.remove(victim)
                del live[victim]
                step_all()   # the layout drops the removed scene's slots before the next add
        got = {sid: read_all(b, sid) for sid in live}
    finally:
        b.close()
    assert len(got) >= 3
    for sid, (scn, fr, k) in live.items():
        want = oracle_states(scn, fr[:k], (k,))[k]
        assert diff_report(want, got[sid]) == [], (scn.name, k)
