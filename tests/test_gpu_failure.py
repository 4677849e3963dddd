"""Failure detection and error paths, made on the host (no GPU fault):

* a scene given a NaN position is flagged MPM_HEALTH_NONFINITE by G2P and
  mpm_sync returns MPM_ERR_NAN; in a batch only that scene is flagged and the
  other scenes stay bit-exact against the oracle; a served job carries the
  flag in its result;
* infinite velocities hit encode's clamp: MPM_HEALTH_SATURATED is set, no call
  fails, and the state still follows the oracle bit for bit;
* mpm_wait returns MPM_ERR_TIMEOUT while work runs and MPM_OK after it;
* a device-memory cap makes mpm_create, mpm_batch_create, mpm_batch_add,
  mpm_server_create and mpm_server_run fail with MPM_ERR_OOM and leave their
  objects usable;
* the plain engine (unchecked stencils, as the reference) refuses positions
  whose stencil would leave the grid, before anything reaches the device.

Only the binned engine ever sees a NaN position: its stencils are
bounds-checked on every path."""
import ctypes

import numpy as np
import pytest

import oracle as O
import scenarios as S
from mls_mpm_b200 import abi, scenes
from mls_mpm_b200.abi import HEALTH_NONFINITE, HEALTH_SATURATED, MpmError, check
from mls_mpm_b200.batch import Batch, default_params
from mls_mpm_b200.server import Server
from runner import GpuScene, diff_report

pytestmark = pytest.mark.gpu

FLUID = ("pos", "vel", "affine", "density", "cell_mv", "cell_mass", "cell_mv_f32", "cell_mass_f32")


def _health(lib, h, clear=False):
    f = ctypes.c_uint32()
    check(lib.mpm_get_health(h, ctypes.byref(f), int(clear)), "mpm_get_health")
    return f.value


def _nan_scene(seed=5):
    sc = scenes.small_box(grid=(24, 20, 22), n=2000, seed=seed, name="nan")
    sc.pos[17, 1] = np.nan
    return sc


def test_nan_position_flags_the_scene(gpu):
    sc = _nan_scene()
    scn = S.Scenario("nan", sc, 3)
    g = GpuScene(gpu, sc)
    try:
        assert gpu.mpm_sync(g.h) == 0 and _health(gpu, g.h) == 0
        for P, W, H, dims, _, _ in scn.frames():
            g.frame(P, W, H, dims)
        assert gpu.mpm_sync(g.h) == 5                      # MPM_ERR_NAN
        assert b"NONFINITE" in gpu.mpm_last_error()
        assert _health(gpu, g.h, clear=True) & HEALTH_NONFINITE
        assert _health(gpu, g.h) == 0                      # cleared
        # the NaN never heals: the next substep flags the scene again
        g.frame(*next(scn.frames())[:4])
        assert gpu.mpm_sync(g.h) == 5
    finally:
        g.close()


def test_infinite_velocity_saturates_and_stays_bit_exact(gpu):
    sc = scenes.small_box(grid=(24, 20, 22), n=2000, seed=9, name="inf_vel")
    sc.vel[:5, 0] = np.inf
    sc.vel[5:8, 2] = -np.inf
    # no stencil weight of these particles is exactly 0 (a coordinate on a cell
    # face would give one, and 0 * inf is NaN, whose clamp is not the point here)
    p = sc.pos[:8, :3]
    assert (p != np.floor(p)).all()
    scn = S.Scenario("inf_vel", sc, 4)
    g = GpuScene(gpu, sc)
    st = O.new_state(sc)
    try:
        for s, (P, W, H, dims, gen, adv) in enumerate(scn.frames()):
            g.frame(P, W, H, dims)
            O.substep(st, P, W, H, dims)
            bad = diff_report(g.state(), st)
            assert not bad, f"substep {s}: {bad}"
        assert gpu.mpm_sync(g.h) == 0
        f = _health(gpu, g.h)
        assert f & HEALTH_SATURATED and not f & HEALTH_NONFINITE
    finally:
        g.close()


def test_healthy_scene_reports_nothing(gpu):
    scn = S.walls_hand_diffuse()
    scn.substeps = 10
    g = GpuScene(gpu, scn.scene, scn.diffuse_max)
    try:
        for P, W, H, dims, _, _ in scn.frames():
            g.frame(P, W, H, dims)
        assert gpu.mpm_sync(g.h) == 0 and _health(gpu, g.h) == 0
    finally:
        g.close()


def test_nan_scene_in_a_batch_leaves_the_others_exact(gpu):
    good = [S.crowded(), S.dam_break_64(8)]
    nan = _nan_scene()
    b = Batch(200_000, 600_000, 4)
    try:
        frames = [[(P, W, H, d) for P, W, H, d, _, _ in s.frames()] for s in good]
        ids = [b.add_scene(s.scene, params=frames[i][0][0]) for i, s in enumerate(good)]
        bad_id = b.add_scene(nan)
        for t in range(8):
            for i, sid in enumerate(ids):
                P, W, H, d = frames[i][min(t, len(frames[i]) - 1)]
                b.set_params(sid, P)
                b.set_walls(sid, W)
            b.step(1)
        with pytest.raises(MpmError) as e:
            b.sync()
        assert e.value.status == 5
        assert b.health(bad_id) & HEALTH_NONFINITE
        for i, (s, sid) in enumerate(zip(good, ids)):
            assert b.health(sid) & HEALTH_NONFINITE == 0
            st = O.new_state(s.scene)
            for P, W, H, d in frames[i][:8]:
                O.substep(st, P, W, H, d)
            got = {k: b.read(sid, k) for k in FLUID}
            assert not diff_report(st, got), s.name
    finally:
        b.close()


def test_served_job_reports_its_health(gpu):
    jobs = [(scenes.small_box(grid=(20, 18, 20), n=1500, seed=40 + i, name=f"job{i}"), 6) for i in range(3)]
    jobs[1][0].pos[3, 0] = np.nan
    srv = Server(int(Batch.footprint(20_000, 60_000, 8)), scene_capacity=8, cells_per_particle=10.0)
    try:
        ids = [srv.submit(default_params(sc.grid, sc.n), sc.pos, sc.mass, k, 0.001 * i) for i, (sc, k) in
               enumerate(jobs)]
        srv.run()
        health = [srv.job(j).health for j in ids]
        assert health[1] & HEALTH_NONFINITE
        assert health[0] & HEALTH_NONFINITE == 0 and health[2] & HEALTH_NONFINITE == 0
    finally:
        srv.close()


def test_wait_times_out_while_work_runs(gpu):
    sc = scenes.dam_break_1m(0)
    g = GpuScene(gpu, sc)
    try:
        P = default_params(sc.grid, sc.n)
        check(gpu.mpm_set_params(g.h, ctypes.byref(P)), "mpm_set_params")
        check(gpu.mpm_step(g.h, 200), "mpm_step")     # tens of milliseconds of work
        assert gpu.mpm_wait(g.h, ctypes.c_double(0.0)) == 4       # MPM_ERR_TIMEOUT
        assert gpu.mpm_wait(g.h, ctypes.c_double(120.0)) == 0
        assert gpu.mpm_wait(g.h, ctypes.c_double(0.0)) == 0       # nothing left to wait for
        assert gpu.mpm_wait(g.h, ctypes.c_double(-1.0)) == 1      # MPM_ERR_INVALID_ARG
    finally:
        g.close()


def _in_use(lib):
    b = ctypes.c_uint64()
    check(lib.mpm_device_memory_in_use(ctypes.byref(b)), "mpm_device_memory_in_use")
    return b.value


def test_device_memory_cap_gives_clean_oom(gpu):
    lib = gpu
    base = _in_use(lib)
    try:
        # a scene that does not fit under the cap
        check(lib.mpm_set_device_memory_limit(base + (1 << 20)), "limit")
        sc = scenes.dam_break_64(0)
        with pytest.raises(MpmError) as e:
            GpuScene(lib, sc)
        assert e.value.status == 2                                # MPM_ERR_OOM
        assert _in_use(lib) == base                               # nothing left behind
        with pytest.raises(MpmError) as e:
            Batch(100_000, 300_000, 4)
        assert e.value.status == 2 and _in_use(lib) == base
        # a batch whose first add needs more staging than the cap leaves
        check(lib.mpm_set_device_memory_limit(0), "limit")
        b = Batch(300_000, 300_000, 4)
        try:
            check(lib.mpm_set_device_memory_limit(_in_use(lib) + (1 << 20)), "limit")
            with pytest.raises(MpmError) as e:
                b.add_scene(sc)
            assert e.value.status == 2
            assert b.info().scenes == 0
            check(lib.mpm_set_device_memory_limit(0), "limit")
            sid = b.add_scene(sc)                                 # the batch still works
            b.step(2)
            b.sync()
            assert b.read(sid, "pos").shape == (sc.n, 4)
        finally:
            b.close()
        # a server whose batch does not fit, and one whose staging does not
        check(lib.mpm_set_device_memory_limit(base + (1 << 20)), "limit")
        with pytest.raises(MpmError) as e:
            Server(int(Batch.footprint(50_000, 200_000, 8)), scene_capacity=8, cells_per_particle=4.0)
        assert e.value.status == 2
        check(lib.mpm_set_device_memory_limit(0), "limit")
        srv = Server(int(Batch.footprint(100_000, 400_000, 8)), scene_capacity=8, cells_per_particle=4.0)
        try:
            check(lib.mpm_set_device_memory_limit(_in_use(lib) + (1 << 20)), "limit")
            small = scenes.small_box(grid=(20, 20, 20), n=1000, seed=2)
            srv.submit(default_params(small.grid, small.n), small.pos, small.mass, 3, 0.0)
            with pytest.raises(MpmError) as e:
                srv.run()                                         # its staging (64 MB) is refused
            assert e.value.status == 2
        finally:
            srv.close()
        assert _in_use(lib) == base
    finally:
        lib.mpm_set_device_memory_limit(0)


def test_plain_engine_refuses_positions_outside_its_stencil_band(gpu):
    sc = scenes.small_box(grid=(16, 16, 16), n=100, seed=1)
    bad = sc.pos.copy()
    bad[7, 2] = 0.5                       # stencil would reach cell -1
    from mls_mpm_b200.fluid_gpu import Desc
    desc = Desc(16, 16, 16, sc.n, 0, 1)   # MPM_FLAG_PLAIN
    h = ctypes.c_void_p()
    check(gpu.mpm_create(ctypes.byref(desc), ctypes.byref(h)), "mpm_create")
    try:
        st = gpu.mpm_upload_particles(h, abi.ptr(bad), None, None, abi.ptr(sc.mass), sc.n)
        assert st == 1 and b"outside" in gpu.mpm_last_error()
        bad[7, 2] = np.nan
        assert gpu.mpm_upload_particles(h, abi.ptr(bad), None, None, abi.ptr(sc.mass), sc.n) == 1
        assert gpu.mpm_upload_particles(h, abi.ptr(sc.pos), None, None, abi.ptr(sc.mass), sc.n) == 0
        assert gpu.mpm_upload(h, 0, abi.ptr(bad), bad.nbytes) == 1
    finally:
        gpu.mpm_destroy(h)
