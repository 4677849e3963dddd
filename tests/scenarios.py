"""Parity scenarios shared by the golden-fixture generator and the tests.

A scenario is a seeded scene plus a per-substep script of the host-side
uniforms (Params, WallParams, HandParams + dispatch box, GenParams with the
bumped seed, AdvectParams), produced by the same host logic FluidGPU runs
(mls_mpm_b200.host), so the oracle, the reference pin and the CUDA path all
see identical bytes.
"""
import numpy as np

from mls_mpm_b200 import host, scenes
from mls_mpm_b200.abi import AdvectParams, GenParams


class HostFluid:
    """The FluidGPU fields host.pack_params/pack_hand read (fluid-gpu.js:10-45)."""

    def __init__(self, grid, n):
        self.grid_X_num, self.grid_Y_num, self.grid_Z_num = grid
        self.active_particle_num = n
        self.DT, self.SUBSTEPS = 0.3, 1
        self.GRAVITY, self.REST_DENSITY, self.STIFFNESS, self.EOS_POWER = -0.98, 8.0, 100.0, 1
        self.VISCOSITY = 0.01
        self.HARD_MIN = 2
        self.HARD_MAX_X, self.HARD_MAX_Y, self.HARD_MAX_Z = grid[0] - 2, grid[1] - 2, grid[2] - 2
        self.WALL_MIN, self.WALL_STIFFNESS, self.LOOKAHEAD_K = 3.0, 1.0, 2.0


class Scenario:
    def __init__(self, name, scene, substeps, diffuse_max=0, walls=None, hand=None):
        self.name = name
        self.scene = scene
        self.substeps = substeps
        self.diffuse_max = diffuse_max
        self.walls_script = walls      # fn(step, WallPacker) or None
        self.hand_script = hand        # fn(step) -> (pos, vel, radius, strength, active, eye) or None

    def frames(self):
        """Yield per-substep (P, W, H, dims, gen, adv)."""
        fl = HostFluid(self.scene.grid, self.scene.n)
        packer = host.WallPacker()
        gen_seed = 1
        hand_buf = None
        H, dims = None, None
        for s in range(self.substeps):
            P = host.pack_params(fl, fl.DT / fl.SUBSTEPS)
            if self.walls_script:
                self.walls_script(s, packer)
            W, _ = packer.pack(fl.DT, self.scene.grid, fl.HARD_MIN, (fl.HARD_MAX_X, fl.HARD_MAX_Y, fl.HARD_MAX_Z))
            if self.hand_script:
                args = self.hand_script(s)
                hand_buf, d = host.pack_hand(fl, *args, buf=hand_buf)
                H, dims = hand_buf, (d if args[4] else [0, 0, 0])
            gen = adv = None
            if self.diffuse_max:
                gen_seed += 1            # diffuse-gpu.js:149 (first step uses 2)
                gen = GenParams(0.5, 3.0, 1.5, 6.0, 3.0, 1.0, 0.3, gen_seed)
                adv = AdvectParams(self.diffuse_max, 1.2, 4.0, 0.0)
            yield P, W, H, dims, gen, adv


def _walls_moving(s, packer):
    if s == 0:
        packer.set_wall(0, [12, 1, 6], [15, 12, 14])
        packer.set_wall(2, [3, 2, 15], [8, 6, 19])
    packer.set_wall(0, [12 - 0.05 * s, 1, 6], [15 - 0.05 * s, 12, 14])
    packer.rotate_wall(0, 0.01, 0.004)
    if s == 25:
        packer.remove_wall(2)


def _hand_sweep(s):
    active = (s % 12) < 9
    return ([8.0 + 0.2 * s, 9.0, 10.0], [1.0, -0.5, 0.2], 3.0, 2.0, active, [10.0, 30.0, 40.0])


def walls_hand_diffuse():
    sc = scenes.small_box(grid=(24, 20, 22), n=3000, seed=3, name="walls_hand_diffuse")
    return Scenario("walls_hand_diffuse", sc, 40, diffuse_max=500, walls=_walls_moving, hand=_hand_sweep)


def dam_break_64(substeps=200):
    """The 64^3 configuration (65,536 particles) over its full 200 substeps."""
    return Scenario("dam_break_64", scenes.dam_break_64(0), substeps)


def saturate():
    """Edge cases: encode clamp saturation and i32 wrap (huge velocities in one
    cell), particles on exact cell boundaries and at the hard bounds."""
    n = 64
    rng = np.random.default_rng(7)
    pos = np.zeros((n, 3), np.float64)
    pos[:16] = [8.0, 8.0, 8.0]                      # integer coordinates
    pos[16:32] = rng.uniform(2.0, 14.0, (16, 3))
    pos[32:40] = [[2.0, 2.0, 2.0]] * 8              # hard_min corner
    pos[40:48] = [[14.0, 14.0, 14.0]] * 8           # hard_max corner (16^3 grid)
    pos[48:] = rng.uniform(6.0, 10.0, (16, 3))
    vel = np.zeros((n, 3), np.float32)
    vel[:4] = [[1e6, -2e6, 3e6]] * 4                # saturates encode and wraps the i32 sum
    vel[16:20] = [[5e4, 0, -5e4]] * 4
    sc = scenes.Scene((16, 16, 16), pos.astype(np.float32), vel, name="saturate")
    return Scenario("saturate", sc, 6, diffuse_max=64)


def empty():
    sc = scenes.Scene((12, 12, 12), np.zeros((0, 3), np.float32), name="empty")
    return Scenario("empty", sc, 3, diffuse_max=32)


def crowded():
    """Hundreds of particles per cell (overpacked, very high pressure)."""
    sc = scenes.dam_break((20, 20, 20), (6.0, 6.0, 6.0), (16, 16, 16), 4096, seed=11, amplitude=0.01,
                          name="crowded")
    sc.pos[:, :3] = (6.0 + (sc.pos[:, :3] - 6.0) * 0.1).astype(np.float32)
    return Scenario("crowded", sc, 12, diffuse_max=1000)


SCENARIOS = {"walls_hand_diffuse": walls_hand_diffuse, "dam_break_64": dam_break_64, "saturate": saturate,
             "empty": empty, "crowded": crowded}
