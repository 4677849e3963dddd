"""Host-side logic: grid sizing, uniform packing, walls, hand box, scenes."""
import math

import numpy as np

import scenarios
from mls_mpm_b200 import host, scenes
from mls_mpm_b200.fluid_gpu import FluidGPU


def test_grid_dims_match_constructor():
    # main.js:21 new FluidGPU(2, 2, 3, 0.0125, 400000) -> 40 x 40 x 60
    assert host.grid_dims(2, 2, 3, 0.0125) == (40, 40, 60)
    fl = FluidGPU(2, 2, 3, 0.0125, 1000)
    assert (fl.grid_X_num, fl.grid_Y_num, fl.grid_Z_num) == (40, 40, 60)
    assert (fl.HARD_MIN, fl.HARD_MAX_X, fl.HARD_MAX_Y, fl.HARD_MAX_Z) == (2, 38, 38, 58)


def test_fill_block_counts_and_stacking():
    fl = FluidGPU(1, 1, 1, 1 / 64, 100000, grid=(16, 16, 16))
    import random
    n1 = fl.fillBlock(0.125, 0.125, 0.125, 0.5, 0.5, 0.5, rng=random.Random(1))
    assert n1 == 12 * 12 * 12          # (0.5-0.125)*16 cells * 2 per cell per axis
    n2 = fl.fillBlock(0.6, 0.125, 0.125, 0.75, 0.25, 0.25, rng=random.Random(2))
    assert n2 > n1
    p = fl.particle_pos[: n2 * 3].reshape(-1, 3)
    assert p.min() > 1.9 and p.max() < 12.1
    assert np.all(fl.particle_mass[:n2] == 1.0)


def test_line_box_intersect():
    assert host.line_box_intersect([0, 5, 5], [1, 0, 0], [2, 0, 0], [8, 10, 10]) == [2, 8]
    assert host.line_box_intersect([0, 50, 5], [1, 0, 0], [2, 0, 0], [8, 10, 10]) is None
    t = host.line_box_intersect([5, 5, 5], [0.6, 0.8, 0.0], [0, 0, 0], [10, 10, 10])
    assert t is not None and t[0] < 0 < t[1]


def test_params_pack_layout():
    fl = scenarios.HostFluid((24, 20, 22), 1234)
    p = host.pack_params(fl, 0.3)
    b = np.frombuffer(bytes(p), np.uint32)
    assert list(b[:4]) == [24, 20, 22, 1234]
    f = np.frombuffer(bytes(p), np.float32)
    assert f[4] == np.float32(0.3) and f[5] == np.float32(-0.98) and f[11] == 22.0 and f[16] == 2.0


def test_wall_pack_velocity_extension_and_dedup():
    wp = host.WallPacker()
    wp.set_wall(1, [1.0, 1.0, 5.0], [6.0, 8.0, 9.0])
    W, changed = wp.pack(0.3, (24, 20, 22), 2, (22, 18, 20))
    assert changed and W.count_pad[0] == 1.0
    w = W.walls[0]
    cx, cy, cz = 3.5, 4.5, 7.0
    assert tuple(w.center_cy[:3]) == (cx, cy, cz)
    # faces touching the boundary band extend outside the grid (fluid-gpu.js:381-391)
    assert w.lmin_sy[0] == np.float32(-4.0 - cx) and w.lmin_sy[1] == np.float32(-4.0 - cy)
    assert w.lmin_sy[2] == np.float32(5.0 - cz)
    assert tuple(w.vel_sp[:3]) == (0.0, 0.0, 0.0)     # appearing is not moving
    W2, changed2 = wp.pack(0.3, (24, 20, 22), 2, (22, 18, 20))
    assert not changed2
    wp.set_wall(1, [1.3, 1.0, 5.0], [6.3, 8.0, 9.0])
    wp.rotate_wall(1, 0.2)
    W3, changed3 = wp.pack(0.3, (24, 20, 22), 2, (22, 18, 20))
    assert changed3
    w3 = W3.walls[0]
    assert abs(w3.vel_sp[0] - (np.float32(1.3) - 1.0) / 0.3) < 1e-5
    assert abs(w3.omega_pad[1] - 0.2 / 0.3) < 1e-6
    assert abs(w3.center_cy[3] - math.cos(0.2)) < 1e-7
    W4, _ = wp.pack(0.3, (24, 20, 22), 2, (22, 18, 20))
    assert W4.walls[0].vel_sp[0] == 0.0               # no move since last frame -> vel 0
    wp.remove_wall(1)
    W5, _ = wp.pack(0.3, (24, 20, 22), 2, (22, 18, 20))
    assert W5.count_pad[0] == 0.0


def test_hand_box():
    fl = scenarios.HostFluid((24, 20, 22), 10)
    h, dims = host.pack_hand(fl, [10, 10, 10], [1, 0, 0], 3.0, 2.0, True, [10, 10, 40])
    # ray along -z through (10,10): box spans all z, x/y within radius
    assert (h.bbox_min_x, h.bbox_max_x) == (7, 13)
    assert (h.bbox_min_z, h.bbox_max_z) == (0, 21)
    assert dims == [7, 7, 22]
    h2, dims2 = host.pack_hand(fl, [10, 10, 10], [1, 0, 0], 3.0, 2.0, False, [10, 10, 40], buf=h)
    assert dims2 == [0, 0, 0] and h2.is_on == 0 and h2.bbox_min_x == 7   # stale box kept


def test_scene_generators_exact_and_seeded():
    a = scenes.dam_break_64(0)
    assert a.n == 65536 and a.grid == (64, 64, 64)
    p = a.pos[:, :3]
    assert p.min() >= 2.0 and p[:, 0].max() <= 18.0 and p[:, 1].max() <= 34.0
    b = scenes.dam_break_64(0)
    assert np.array_equal(a.pos, b.pos)
    c = scenes.dam_break_64(1)
    assert not np.array_equal(a.pos, c.pos)
    # 2x2x2 per cell
    cells = np.floor(p).astype(np.int64)
    key = (cells[:, 2] * 64 + cells[:, 1]) * 64 + cells[:, 0]
    counts = np.bincount(key)
    assert counts.max() <= 27 and np.isclose(counts[counts > 0].mean(), 8.0, rtol=0.1)


def test_splitmix64_known_values():
    # splitmix64 with state 0: first output 0xE220A8397B1DCDAF (published reference value)
    assert int(scenes.splitmix64(0, 1)[0]) == 0xE220A8397B1DCDAF
