"""Particle editing on the GPU against the oracle: deleteNear (COMPACT,
shaders.js:521-546), raycastFluid (RAYCAST, shaders.js:563-576) and the
buffer writes of spawnParticles (fluid-gpu.js:145-179), interleaved with
substeps, on both engines.  Bit-exact."""
import ctypes
import math

import numpy as np
import pytest

import oracle as O
from mls_mpm_b200 import abi, host, scenes
from mls_mpm_b200.abi import BUF, check
from mls_mpm_b200.fluid_gpu import Desc
from runner import ENGINES, diff_report
from scenarios import HostFluid

pytestmark = pytest.mark.gpu


def _unit(v):
    n = math.sqrt(sum(x * x for x in v))
    return [x / n for x in v]


def _ray(o, d, r):
    rp = abi.RayParams()
    rp.ox, rp.oy, rp.oz = (float(np.float32(x)) for x in o)
    rp.radius = float(np.float32(r))
    rp.dx, rp.dy, rp.dz = (float(np.float32(x)) for x in d)
    return rp


class Pair:
    """The same scene on the GPU (C ABI) and in the oracle, capacity > n."""

    def __init__(self, lib, scene, capacity, engine):
        self.lib, self.grid = lib, scene.grid
        X, Y, Z = scene.grid
        self.G = X * Y * Z
        self.cap = capacity
        self.fl = HostFluid(scene.grid, scene.n)
        self.h = ctypes.c_void_p()
        check(lib.mpm_create(ctypes.byref(Desc(X, Y, Z, capacity, 0, ENGINES[engine])), ctypes.byref(self.h)),
              "mpm_create")
        check(lib.mpm_upload_particles(self.h, abi.ptr(scene.pos), abi.ptr(scene.vel), abi.ptr(scene.affine),
                                       abi.ptr(scene.mass), scene.n), "upload")
        n = scene.n
        st = {"pos": np.zeros((capacity, 4), np.float32), "vel": np.zeros((capacity, 4), np.float32),
              "affine": np.zeros((capacity, 9), np.float32), "mass": np.zeros(capacity, np.float32),
              "density": np.zeros(capacity, np.float32),
              "cell_mv": np.zeros((self.G, 3), np.int32), "cell_mass": np.zeros(self.G, np.int32),
              "cell_mv_f32": np.zeros((self.G, 3), np.float32), "cell_mass_f32": np.zeros(self.G, np.float32)}
        st["pos"][:n], st["vel"][:n], st["affine"][:n], st["mass"][:n] = scene.pos, scene.vel, scene.affine, scene.mass
        self.st = st
        self.W = abi.WallParams()

    @property
    def n(self):
        return self.fl.active_particle_num

    def params(self):
        return host.pack_params(self.fl, self.fl.DT / self.fl.SUBSTEPS)

    def step(self, k):
        for _ in range(k):
            P = self.params()
            check(self.lib.mpm_set_params(self.h, ctypes.byref(P)), "set_params")
            check(self.lib.mpm_set_walls(self.h, ctypes.byref(self.W)), "set_walls")
            check(self.lib.mpm_step(self.h, 1), "step")
            O.substep(self.st, P, self.W)

    def read(self, name, rows):
        shapes = {"pos": ((rows, 4), np.float32), "vel": ((rows, 4), np.float32), "affine": ((rows, 9), np.float32),
                  "mass": ((rows,), np.float32), "density": ((rows,), np.float32),
                  "cell_mv": ((self.G, 3), np.int32), "cell_mass": ((self.G,), np.int32),
                  "cell_mv_f32": ((self.G, 3), np.float32), "cell_mass_f32": ((self.G,), np.float32)}
        shape, dt = shapes[name]
        a = np.zeros(shape, dt)
        check(self.lib.mpm_download(self.h, BUF[name], abi.ptr(a), a.nbytes), "download")
        return a

    def compare(self):
        n = self.n
        gpu, cpu = {}, {}
        for k in ("pos", "vel", "affine", "mass", "density"):
            gpu[k], cpu[k] = self.read(k, n), self.st[k][:n]
        for k in ("cell_mv", "cell_mass", "cell_mv_f32", "cell_mass_f32"):
            gpu[k], cpu[k] = self.read(k, n), self.st[k]
        return diff_report(cpu, gpu)

    def delete_near(self, origin, d, radius):
        o = (ctypes.c_double * 3)(*origin)
        dd = (ctypes.c_double * 3)(*d)
        m = ctypes.c_uint32()
        check(self.lib.mpm_delete_near(self.h, o, dd, float(radius), ctypes.byref(m)), "delete_near")
        P = self.params()
        cnt, po, vo, mo = O.compact(P, _ray(origin, d, radius), self.st["pos"], self.st["vel"], self.st["mass"])
        self.st["pos"][:cnt], self.st["vel"][:cnt], self.st["mass"][:cnt] = po[:cnt], vo[:cnt], mo[:cnt]
        self.fl.active_particle_num = cnt
        return m.value, cnt

    def raycast(self, origin, d, radius):
        o = (ctypes.c_double * 3)(*origin)
        dd = (ctypes.c_double * 3)(*d)
        hit, t, hp = ctypes.c_int(), ctypes.c_float(), (ctypes.c_double * 3)()
        check(self.lib.mpm_raycast_fluid(self.h, o, dd, float(radius), ctypes.byref(hit), ctypes.byref(t), hp),
              "raycast")
        bits = O.raycast(self.params(), _ray(origin, d, radius), self.st["pos"])
        gpu_bits = int(np.float32(t.value).view(np.uint32)) if hit.value else 0xFFFFFFFF
        return gpu_bits, bits, list(hp) if hit.value else None

    def append(self, pos4, vel4, mass):
        got = ctypes.c_uint32()
        check(self.lib.mpm_append_particles(self.h, abi.ptr(pos4), abi.ptr(vel4), abi.ptr(mass), len(mass),
                                            ctypes.byref(got)), "append")
        start = self.n
        k = min(len(mass), self.cap - start)
        self.st["pos"][start:start + k] = pos4[:k]
        self.st["vel"][start:start + k] = vel4[:k]
        self.st["mass"][start:start + k] = mass[:k]
        self.fl.active_particle_num = start + k
        return got.value, k

    def close(self):
        self.lib.mpm_destroy(self.h)


@pytest.mark.parametrize("engine", ["binned", "plain"])
def test_delete_raycast_append_match_oracle(gpu, engine):
    sc = scenes.small_box(grid=(24, 20, 22), n=3000, seed=11, name="edit")
    p = Pair(gpu, sc, 3600, engine)
    try:
        p.step(6)
        assert p.compare() == []
        # rays: one through the fluid, one that misses, one pointing away
        # (the block fills x 2..12, y 2..14, z 2..5.5)
        for o, d, r in (([7.0, 30.0, 4.0], _unit([0.05, -1.0, 0.02]), 2.0),
                        ([12.0, 19.5, 11.0], [1.0, 0.0, 0.0], 0.25),
                        ([7.0, 5.0, -4.0], [0.0, 0.0, -1.0], 3.0),
                        ([-3.0, 6.0, 4.0], [1.0, 0.0, 0.0], 0.5)):
            g, c, hp = p.raycast(o, d, r)
            assert g == c, (o, d, r, hex(g), hex(c))
        g, c, hp = p.raycast([7.0, 30.0, 4.0], _unit([0.05, -1.0, 0.02]), 2.0)
        assert hp is not None
        t = float(np.uint32(c).view(np.float32))
        d = _unit([0.05, -1.0, 0.02])
        assert hp == [[7.0, 30.0, 4.0][i] + t * d[i] for i in range(3)]
        g, c, hp = p.raycast([7.0, 5.0, -4.0], [0.0, 0.0, -1.0], 3.0)
        assert hp is None and c == 0xFFFFFFFF
        # delete a vertical cylinder through the block, then keep stepping
        m_gpu, m_cpu = p.delete_near([6.0, 10.0, 4.0], _unit([0.1, 1.0, -0.05]), 2.5)
        assert m_gpu == m_cpu and 0 < m_cpu < 3000
        p.step(3)
        assert p.compare() == []
        # append a seeded sphere of particles (more than fits: clamped to capacity)
        rng = np.random.default_rng(5)
        k = 3600 - m_cpu + 40
        pos4 = np.zeros((k, 4), np.float32)
        pos4[:, :3] = rng.uniform([6, 8, 6], [14, 14, 14], (k, 3)).astype(np.float32)
        vel4 = np.zeros((k, 4), np.float32)
        vel4[:, :3] = rng.uniform(-1, 1, (k, 3)).astype(np.float32)
        mass = np.ones(k, np.float32)
        got, want = p.append(pos4, vel4, mass)
        assert got == want == 3600 - m_cpu
        p.step(4)
        assert p.compare() == []
        # delete everything near the floor plane, then an empty delete
        m_gpu, m_cpu = p.delete_near([0.0, 3.0, 11.0], [1.0, 0.0, 0.0], 40.0)
        assert m_gpu == m_cpu == 0
        p.step(1)
        m_gpu, m_cpu = p.delete_near([0.0, 3.0, 11.0], [1.0, 0.0, 0.0], 1.0)
        assert m_gpu == m_cpu == 0
    finally:
        p.close()


def test_buffer_level_compact_and_raycast(gpu):
    """mpm_compact / mpm_raycast on caller-owned device buffers (torch memory)."""
    import torch
    rng = np.random.default_rng(7)
    for n in (0, 1, 2047, 2048, 2049, 100_003):
        pos = np.zeros((n, 4), np.float32)
        pos[:, :3] = rng.uniform(0, 32, (n, 3))
        pos[:, 3] = rng.uniform(-1, 1, n)
        vel = rng.standard_normal((n, 4)).astype(np.float32)
        mass = rng.uniform(0.5, 2, n).astype(np.float32)
        ray = _ray([16.0, 16.0, 16.0], _unit([1.0, 2.0, 0.5]), 6.0)
        P = abi.Params()
        P.particle_num = n
        cnt, po, vo, mo = O.compact(P, ray, pos, vel, mass)
        dev = torch.device("cuda:0")
        tp, tv, tm = (torch.from_numpy(a).to(dev) for a in (pos, vel, mass))
        op, ov, om = torch.zeros_like(tp), torch.zeros_like(tv), torch.zeros_like(tm)
        cdev = torch.full((1,), 12345, dtype=torch.int32, device=dev)
        s = torch.cuda.current_stream().cuda_stream
        check(gpu.mpm_compact(ctypes.byref(ray), n, tp.data_ptr(), tv.data_ptr(), tm.data_ptr(), op.data_ptr(),
                              ov.data_ptr(), om.data_ptr(), cdev.data_ptr(), s), "mpm_compact")
        hdev = torch.zeros((1,), dtype=torch.int32, device=dev)
        check(gpu.mpm_raycast(ctypes.byref(ray), n, tp.data_ptr(), hdev.data_ptr(), s), "mpm_raycast")
        torch.cuda.synchronize()
        assert int(cdev.item()) == cnt
        assert np.array_equal(op.cpu().numpy()[:cnt].view(np.uint32), po[:cnt].view(np.uint32))
        assert np.array_equal(ov.cpu().numpy()[:cnt].view(np.uint32), vo[:cnt].view(np.uint32))
        assert np.array_equal(om.cpu().numpy()[:cnt].view(np.uint32), mo[:cnt].view(np.uint32))
        assert (int(hdev.item()) & 0xFFFFFFFF) == O.raycast(P, ray, pos)
