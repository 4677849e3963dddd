"""FluidGPU / DiffuseGPU — the reference's JavaScript classes (fluid-gpu.js,
diffuse-gpu.js) restated over the native C ABI (include/mpm_b200.h).

Same constructor arguments, public fields and method names; the WebGPU
device/encoder/pass arguments become a CUDA device ordinal (initGPU) or
disappear (simFrame records nothing: it enqueues the substeps on the scene's
CUDA stream).  Buffers are device-resident after initGPU and are read with
read()/get_buffer().
"""
import ctypes
import math
import random

import numpy as np

from . import abi, host
from .abi import BUF, DIFFUSE_DTYPE, MAX_WALLS, AdvectParams, GenParams, HandParams, check, load_library


class Desc(ctypes.Structure):
    _fields_ = [("grid_X", ctypes.c_uint32), ("grid_Y", ctypes.c_uint32), ("grid_Z", ctypes.c_uint32),
                ("particle_capacity", ctypes.c_uint32), ("device", ctypes.c_int32), ("flags", ctypes.c_uint32)]


class FluidGPU:
    """fluid-gpu.js:9-685."""

    def __init__(self, aspectX, aspectY, aspectZ, particleRadius, particleNum, grid=None):
        if grid is None:
            grid = host.grid_dims(aspectX, aspectY, aspectZ, particleRadius)
        self.grid_X_num, self.grid_Y_num, self.grid_Z_num = (int(g) for g in grid)
        self.grid_num = self.grid_X_num * self.grid_Y_num * self.grid_Z_num
        self.particle_num = int(particleNum)
        self.active_particle_num = 0
        self.particle_pos = np.zeros(self.particle_num * 3, np.float32)
        self.particle_vel = np.zeros(self.particle_num * 3, np.float32)
        self.particle_affine = np.zeros(self.particle_num * 9, np.float32)
        self.particle_mass = np.zeros(self.particle_num, np.float32)
        # fluid-gpu.js:24-45
        self.DT = 0.3
        self.REST_DENSITY = 8.0
        self.STIFFNESS = 100.0
        self.EOS_POWER = 1
        self.VISCOSITY = 0.01
        self.GRAVITY = -0.98
        self.SUBSTEPS = 1
        self.WALL_MIN = 3.0
        self.WALL_STIFFNESS = 1.0
        self.LOOKAHEAD_K = 2.0
        HM = 2
        self.HARD_MIN = HM
        self.HARD_MAX_X = self.grid_X_num - HM
        self.HARD_MAX_Y = self.grid_Y_num - HM
        self.HARD_MAX_Z = self.grid_Z_num - HM
        self.diffuse = None
        self._walls = host.WallPacker()
        self.walls = self._walls.walls
        self.handActive = False
        self._hand = HandParams()
        self._hand_dims = [0, 0, 0]
        self._params_prev = None
        self.lastRayHit = None
        self._scene = None
        self._lib = None

    @classmethod
    def from_scene(cls, scene, device=0):
        """A FluidGPU holding a mls_mpm_b200.scenes.Scene, uploaded to `device`."""
        fl = cls(1, 1, 1, 1, scene.n, grid=scene.grid)
        fl.particle_pos[:] = scene.pos[:, :3].ravel()
        fl.particle_vel[:] = scene.vel[:, :3].ravel()
        fl.particle_affine[:] = scene.affine.ravel()
        fl.particle_mass[:] = scene.mass
        fl.active_particle_num = scene.n
        fl.initGPU(device)
        return fl

    # ---- walls (fluid-gpu.js:75-103) ----
    def setWall(self, i, mn, mx):
        self._walls.set_wall(i, mn, mx)

    def rotateWall(self, i, dTheta, dPhi=0.0):
        self._walls.rotate_wall(i, dTheta, dPhi)

    def removeWall(self, i):
        self._walls.remove_wall(i)

    # ---- seeding (fluid-gpu.js:107-128) ----
    def fillBlock(self, x0, y0, z0, x1, y1, z1, rng=None):
        """Lattice at 0.5-cell spacing with +-0.025-cell jitter; stacks from
        active_particle_num.  rng: a random.Random (the reference uses Math.random)."""
        rnd = (rng or random).random
        step, jitter = 0.5, 0.05
        gx0, gx1 = x0 * self.grid_X_num, x1 * self.grid_X_num
        gy0, gy1 = y0 * self.grid_Y_num, y1 * self.grid_Y_num
        gz0, gz1 = z0 * self.grid_Z_num, z1 * self.grid_Z_num
        p = self.active_particle_num
        gz = gz0 + step / 2
        while gz < gz1:
            gy = gy0 + step / 2
            while gy < gy1:
                gx = gx0 + step / 2
                while gx < gx1:
                    if p >= self.particle_num:
                        self.active_particle_num = p
                        return p
                    self.particle_pos[p * 3] = gx + (rnd() - 0.5) * jitter
                    self.particle_pos[p * 3 + 1] = gy + (rnd() - 0.5) * jitter
                    self.particle_pos[p * 3 + 2] = gz + (rnd() - 0.5) * jitter
                    self.particle_mass[p] = 1.0
                    p += 1
                    gx += step
                gy += step
            gz += step
        self.active_particle_num = p
        return p

    # ---- device ----
    def initGPU(self, device=0):
        """fluid-gpu.js:183-293: create device buffers, upload the particles."""
        lib = self._lib = load_library()
        d = Desc(self.grid_X_num, self.grid_Y_num, self.grid_Z_num, self.particle_num, int(device), 0)
        sc = ctypes.c_void_p()
        check(lib.mpm_create(ctypes.byref(d), ctypes.byref(sc)), "mpm_create")
        self._scene = sc
        n = self.particle_num
        pos4 = np.zeros((n, 4), np.float32)
        pos4[:, :3] = self.particle_pos.reshape(n, 3)
        vel4 = np.zeros((n, 4), np.float32)
        vel4[:, :3] = self.particle_vel.reshape(n, 3)
        aff = np.ascontiguousarray(self.particle_affine)
        mass = np.ascontiguousarray(self.particle_mass)
        check(lib.mpm_upload_particles(sc, abi.ptr(pos4), abi.ptr(vel4), abi.ptr(aff), abi.ptr(mass), n),
              "mpm_upload_particles")
        self._write_params_buffer(self.DT / self.SUBSTEPS)
        # the reference uploads the whole capacity; active count stays as filled
        return self

    def _write_params_buffer(self, dt):
        """fluid-gpu.js:295-328 (dedup: skip when the 80 bytes are unchanged)."""
        p = host.pack_params(self, dt)
        b = bytes(p)
        if b == self._params_prev:
            return
        self._params_prev = b
        check(self._lib.mpm_set_params(self._scene, ctypes.byref(p)), "mpm_set_params")

    def _write_wall_params(self):
        wp, changed = self._walls.pack(self.DT, (self.grid_X_num, self.grid_Y_num, self.grid_Z_num),
                                       self.HARD_MIN, (self.HARD_MAX_X, self.HARD_MAX_Y, self.HARD_MAX_Z))
        if changed:
            check(self._lib.mpm_set_walls(self._scene, ctypes.byref(wp)), "mpm_set_walls")

    def updateHand(self, pos, vel, radius, strength, active, eye):
        """fluid-gpu.js:479-527."""
        self.handActive = bool(active)
        self._hand, self._hand_dims = host.pack_hand(self, pos, vel, radius, strength, active, eye, self._hand)
        dims = (ctypes.c_int32 * 3)(*self._hand_dims)
        check(self._lib.mpm_set_hand(self._scene, ctypes.byref(self._hand), int(self.handActive), dims),
              "mpm_set_hand")

    # ---- particle editing (fluid-gpu.js:130-179, 529-628) ----
    def spawnParticles(self, cx, cy, cz, count, radius, vel=(0.0, 0.0, 0.0), sprayVel=3.0, rng=None):
        """fluid-gpu.js:145-179: up to `count` particles in a jittered sphere with
        an outward kick, clamped to the hard bounds; returns the number added.
        rng: a random.Random (the reference uses Math.random)."""
        rnd = (rng or random).random
        start = self.active_particle_num
        n = min(int(count), self.particle_num - start)
        if n <= 0:
            return 0
        pos4 = np.zeros((n, 4), np.float32)
        vel4 = np.zeros((n, 4), np.float32)
        hmin, hx, hy, hz = self.HARD_MIN, self.HARD_MAX_X, self.HARD_MAX_Y, self.HARD_MAX_Z
        for i in range(n):
            r = radius * math.pow(rnd(), 1.0 / 3.0)
            theta = rnd() * math.pi * 2
            cphi = rnd() * 2 - 1
            sphi = math.sqrt(1 - cphi * cphi)
            dx, dy, dz = r * sphi * math.cos(theta), r * sphi * math.sin(theta), r * cphi
            pos4[i, 0] = min(hx, max(hmin, cx + dx))
            pos4[i, 1] = min(hy, max(hmin, cy + dy))
            pos4[i, 2] = min(hz, max(hmin, cz + dz))
            rl = math.hypot(dx, dy, dz) or 1
            vel4[i, 0] = vel[0] + dx / rl * sprayVel
            vel4[i, 1] = vel[1] + dy / rl * sprayVel
            vel4[i, 2] = vel[2] + dz / rl * sprayVel
        mass = np.ones(n, np.float32)
        got = ctypes.c_uint32()
        check(self._lib.mpm_append_particles(self._scene, abi.ptr(pos4), abi.ptr(vel4), abi.ptr(mass), n,
                                             ctypes.byref(got)), "mpm_append_particles")
        self.active_particle_num = start + got.value
        return got.value

    def deleteNear(self, cmd, origin, dir, radius):
        """fluid-gpu.js:544-571 (+ pollDelete): the new active count is known
        when the call returns."""
        self._write_params_buffer(self.DT / self.SUBSTEPS)
        o = (ctypes.c_double * 3)(*origin)
        d = (ctypes.c_double * 3)(*dir)
        m = ctypes.c_uint32()
        check(self._lib.mpm_delete_near(self._scene, o, d, float(radius), ctypes.byref(m)), "mpm_delete_near")
        self.active_particle_num = m.value
        return True

    def pollDelete(self):
        """fluid-gpu.js:574-584: nothing is pending after deleteNear returns."""

    def raycastFluid(self, cmd, origin, dir, radius):
        """fluid-gpu.js:594-612 (+ pollRaycast): sets lastRayHit to the world
        position of the first particle along the ray, or None."""
        self._write_params_buffer(self.DT / self.SUBSTEPS)
        o = (ctypes.c_double * 3)(*origin)
        d = (ctypes.c_double * 3)(*dir)
        hit, t, hp = ctypes.c_int(), ctypes.c_float(), (ctypes.c_double * 3)()
        check(self._lib.mpm_raycast_fluid(self._scene, o, d, float(radius), ctypes.byref(hit), ctypes.byref(t), hp),
              "mpm_raycast_fluid")
        self.lastRayHit = [hp[0], hp[1], hp[2]] if hit.value else None
        return True

    def pollRaycast(self):
        """fluid-gpu.js:615-628: nothing is pending after raycastFluid returns."""

    def simFrame(self, cmd=None):
        """fluid-gpu.js:648-684: SUBSTEPS substeps (+ diffuse) on the scene stream."""
        self._write_params_buffer(self.DT / self.SUBSTEPS)
        self._write_wall_params()
        check(self._lib.mpm_step(self._scene, int(self.SUBSTEPS)), "mpm_step")
        if self.diffuse is not None:
            self.diffuse._seed = (self.diffuse._seed + int(self.SUBSTEPS)) & 0xFFFFFFFF

    def sync(self):
        check(self._lib.mpm_sync(self._scene), "mpm_sync")

    def wait(self, timeout_s):
        """True once the scene's work is done, False while it still runs after
        timeout_s seconds (mpm_wait); raises on a non-finite state."""
        st = self._lib.mpm_wait(self._scene, float(timeout_s))
        if st == 4:   # MPM_ERR_TIMEOUT
            return False
        check(st, "mpm_wait")
        return True

    def health(self, clear=False):
        """MPM_HEALTH_* bits of the scene (abi.HEALTH_NONFINITE, abi.HEALTH_SATURATED)."""
        f = ctypes.c_uint32()
        check(self._lib.mpm_get_health(self._scene, ctypes.byref(f), int(bool(clear))), "mpm_get_health")
        return f.value

    # ---- buffers ----
    def get_buffer(self, name):
        """(device pointer, bytes) of a reference-layout buffer."""
        p, sz = ctypes.c_void_p(), ctypes.c_size_t()
        check(self._lib.mpm_get_buffer(self._scene, BUF[name], ctypes.byref(p), ctypes.byref(sz)),
              "mpm_get_buffer")
        return p.value, sz.value

    def get_ipc_handle(self, name):
        """(handle bytes, offset, bytes) exporting a reference-layout buffer to
        another process (cudaIpcOpenMemHandle on the handle, then + offset)."""
        h = ctypes.create_string_buffer(64)
        off, sz = ctypes.c_size_t(), ctypes.c_size_t()
        check(self._lib.mpm_get_ipc_handle(self._scene, BUF[name], h, ctypes.byref(off), ctypes.byref(sz)),
              "mpm_get_ipc_handle")
        return h.raw, off.value, sz.value

    def read(self, name):
        """Download one buffer as a numpy array in the reference layout."""
        n, G = self.particle_num, self.grid_num
        M = self.diffuse.maxCount if self.diffuse is not None else 0
        shapes = {"pos": ((n, 4), np.float32), "vel": ((n, 4), np.float32), "affine": ((n, 9), np.float32),
                  "mass": ((n,), np.float32), "density": ((n,), np.float32),
                  "cell_mv": ((G, 3), np.int32), "cell_mass": ((G,), np.int32),
                  "cell_mv_f32": ((G, 3), np.float32), "cell_mass_f32": ((G,), np.float32),
                  "diffuse": ((M,), DIFFUSE_DTYPE), "free_list": ((M,), np.uint32), "free_top": ((1,), np.int32)}
        shape, dt = shapes[name]
        a = np.zeros(shape, dt)
        check(self._lib.mpm_download(self._scene, BUF[name], abi.ptr(a), a.nbytes), "mpm_download")
        return a

    def write(self, name, array):
        a = np.ascontiguousarray(array)
        check(self._lib.mpm_upload(self._scene, BUF[name], abi.ptr(a), a.nbytes), "mpm_upload")

    def destroy(self):
        if self._scene is not None:
            self._lib.mpm_destroy(self._scene)
            self._scene = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class DiffuseGPU:
    """diffuse-gpu.js:15-189."""

    def __init__(self, maxCount):
        self.maxCount = int(maxCount)
        self.KE_THRESHOLD = 0.5
        self.PRESSURE_THRESHOLD = 1.0
        self.CREST_DOT_THRESHOLD = 0.3
        self.SPAWN_RATE_K = 3.0
        self.LIFETIME_FOAM = 3.0
        self.BUOYANCY = 1.2
        self.DRAG = 4.0
        self.DENSITY_SPRAY_MAX = 1.5
        self.DENSITY_BUBBLE_MIN = 6.0
        self.aliveCount = 0
        self._seed = 1
        self.fluid = None

    def _gen(self):
        return GenParams(self.KE_THRESHOLD, self.SPAWN_RATE_K, self.DENSITY_SPRAY_MAX, self.DENSITY_BUBBLE_MIN,
                         self.LIFETIME_FOAM, self.PRESSURE_THRESHOLD, self.CREST_DOT_THRESHOLD, self._seed)

    def initGPU(self, device, fluid):
        """diffuse-gpu.js:39-94; also sets fluid.diffuse like main.js:651."""
        self.fluid = fluid
        adv = AdvectParams(self.maxCount, self.BUOYANCY, self.DRAG, 0.0)
        g = self._gen()
        check(fluid._lib.mpm_diffuse_enable(fluid._scene, self.maxCount, ctypes.byref(g), ctypes.byref(adv)),
              "mpm_diffuse_enable")
        fluid.diffuse = self
        return self

    def _writeGenParams(self):
        """diffuse-gpu.js:84-94: re-upload thresholds and the seed."""
        g = self._gen()
        check(self.fluid._lib.mpm_diffuse_set_gen_params(self.fluid._scene, ctypes.byref(g)),
              "mpm_diffuse_set_gen_params")

    def requestDebugReadback(self, cmd=None):
        """diffuse-gpu.js:172-176: queue a copy of the free-list top after the
        work submitted so far (asynchronous; a ring of 4 readbacks in flight)."""
        check(self.fluid._lib.mpm_diffuse_request_alive(self.fluid._scene), "mpm_diffuse_request_alive")

    def pollDebug(self):
        """diffuse-gpu.js:178-188: aliveCount = maxCount - top once a requested
        readback has landed; never waits.  Returns the current aliveCount."""
        a, ready = ctypes.c_int32(), ctypes.c_int32()
        check(self.fluid._lib.mpm_diffuse_poll_alive(self.fluid._scene, ctypes.byref(a), ctypes.byref(ready)),
              "mpm_diffuse_poll_alive")
        if ready.value:
            self.aliveCount = a.value
        return self.aliveCount

    def readAliveCount(self):
        """The alive count now (waits for the stream)."""
        a = ctypes.c_int32()
        check(self.fluid._lib.mpm_diffuse_alive_count(self.fluid._scene, ctypes.byref(a)),
              "mpm_diffuse_alive_count")
        self.aliveCount = a.value
        return self.aliveCount
