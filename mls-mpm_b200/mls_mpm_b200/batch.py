"""Batch of independent scenes over the C ABI (mpm_batch_*): one launch per
kernel per substep for all scenes, per-scene grids, uniforms and particles.

No counterpart in the reference (one FluidGPU per page); each scene behaves
exactly as the same scene in its own FluidGPU (bit-identical results).
"""
import ctypes

import numpy as np

from . import abi
from .abi import BUF, BatchDesc, BatchInfo, check, load_library


class Batch:
    def __init__(self, particle_capacity, cell_capacity, scene_capacity, device=0, flags=0, lib=None):
        self.lib = lib or load_library()
        d = BatchDesc(int(particle_capacity), int(scene_capacity), int(cell_capacity), int(device), int(flags))
        self.h = ctypes.c_void_p()
        check(self.lib.mpm_batch_create(ctypes.byref(d), ctypes.byref(self.h)), "mpm_batch_create")
        self.scenes = {}   # id -> (grid, n)

    @staticmethod
    def footprint(particle_capacity, cell_capacity, scene_capacity, lib=None):
        lib = lib or load_library()
        b = ctypes.c_uint64()
        check(lib.mpm_batch_footprint(int(particle_capacity), int(cell_capacity), int(scene_capacity),
                                      ctypes.byref(b)), "mpm_batch_footprint")
        return b.value

    def add(self, params, pos4, mass, vel4=None, affine9=None, walls=None):
        """params: abi.Params with the scene's grid dims; arrays in the reference layouts."""
        n = len(mass)
        sid = ctypes.c_int32()
        check(self.lib.mpm_batch_add(self.h, ctypes.byref(params), ctypes.byref(walls) if walls is not None else None,
                                     abi.ptr(pos4), abi.ptr(vel4), abi.ptr(affine9), abi.ptr(mass), n,
                                     ctypes.byref(sid)), "mpm_batch_add")
        self.scenes[sid.value] = ((params.grid_X, params.grid_Y, params.grid_Z), n)
        return sid.value

    def add_scene(self, scene, params=None, walls=None):
        """Add a mls_mpm_b200.scenes.Scene with default Params for its grid."""
        if params is None:
            params = default_params(scene.grid, scene.n, self.lib)
        return self.add(params, scene.pos, scene.mass, scene.vel, scene.affine, walls)

    def remove(self, sid):
        check(self.lib.mpm_batch_remove(self.h, int(sid)), "mpm_batch_remove")
        del self.scenes[sid]

    def set_params(self, sid, params):
        check(self.lib.mpm_batch_set_params(self.h, int(sid), ctypes.byref(params)), "mpm_batch_set_params")

    def set_walls(self, sid, walls):
        check(self.lib.mpm_batch_set_walls(self.h, int(sid), ctypes.byref(walls)), "mpm_batch_set_walls")

    def set_hand(self, sid, hand, active, dims):
        d = (ctypes.c_int32 * 3)(*dims)
        check(self.lib.mpm_batch_set_hand(self.h, int(sid), ctypes.byref(hand), int(active), d), "mpm_batch_set_hand")

    def step(self, substeps=1):
        check(self.lib.mpm_batch_step(self.h, int(substeps)), "mpm_batch_step")

    def sync(self):
        check(self.lib.mpm_batch_sync(self.h), "mpm_batch_sync")

    def health(self, sid, clear=False):
        """MPM_HEALTH_* bits of one scene (mpm_batch_get_health)."""
        f = ctypes.c_uint32()
        check(self.lib.mpm_batch_get_health(self.h, int(sid), ctypes.byref(f), int(bool(clear))),
              "mpm_batch_get_health")
        return f.value

    def stream(self):
        s = ctypes.c_void_p()
        check(self.lib.mpm_batch_get_stream(self.h, ctypes.byref(s)), "mpm_batch_get_stream")
        return s.value

    def info(self):
        i = BatchInfo()
        check(self.lib.mpm_batch_get_info(self.h, ctypes.byref(i)), "mpm_batch_get_info")
        return i

    def read(self, sid, name):
        (X, Y, Z), n = self.scenes[sid]
        G = X * Y * Z
        shapes = {"pos": ((n, 4), np.float32), "vel": ((n, 4), np.float32), "affine": ((n, 9), np.float32),
                  "mass": ((n,), np.float32), "density": ((n,), np.float32),
                  "cell_mv": ((G, 3), np.int32), "cell_mass": ((G,), np.int32),
                  "cell_mv_f32": ((G, 3), np.float32), "cell_mass_f32": ((G,), np.float32)}
        shape, dt = shapes[name]
        a = np.zeros(shape, dt)
        check(self.lib.mpm_batch_download(self.h, int(sid), BUF[name], abi.ptr(a), a.nbytes), "mpm_batch_download")
        return a

    def close(self):
        if self.h:
            self.lib.mpm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_params(grid, n, lib=None):
    """FluidGPU constructor defaults for this grid (fluid-gpu.js:24-45)."""
    from .fluid_gpu import Desc
    lib = lib or load_library()
    P = abi.Params()
    d = Desc(grid[0], grid[1], grid[2], n, 0, 0)
    check(lib.mpm_default_params(ctypes.byref(d), ctypes.byref(P)), "mpm_default_params")
    P.particle_num = n
    return P
