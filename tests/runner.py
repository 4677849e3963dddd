"""Runs a parity scenario on the oracle / reference pin (CPU) or on the CUDA
path through the C ABI, yielding the full state after every substep."""
import ctypes

import numpy as np

import oracle as O
from mls_mpm_b200 import abi
from mls_mpm_b200.abi import BUF, DIFFUSE_DTYPE, check
from mls_mpm_b200.fluid_gpu import Desc

FLUID_KEYS = ("pos", "vel", "affine", "density", "cell_mv", "cell_mass", "cell_mv_f32", "cell_mass_f32")
DIFFUSE_KEYS = ("diffuse", "free_list", "top")


def cpu_run(scenario, impl="oracle", threads=1):
    st = O.new_state(scenario.scene, scenario.diffuse_max)
    for P, W, H, dims, gen, adv in scenario.frames():
        O.substep(st, P, W, H, dims, gen, adv, threads=threads, impl=impl)
        yield st


class GpuScene:
    """A scene driven through the raw C ABI."""

    def __init__(self, lib, scene, diffuse_max=0, device=0, flags=0):
        self.lib = lib
        self.scene = scene
        self.n = scene.n
        X, Y, Z = scene.grid
        self.G = X * Y * Z
        self.M = diffuse_max
        d = Desc(X, Y, Z, scene.n, device, flags)
        self.h = ctypes.c_void_p()
        check(lib.mpm_create(ctypes.byref(d), ctypes.byref(self.h)), "mpm_create")
        check(lib.mpm_upload_particles(self.h, abi.ptr(scene.pos), abi.ptr(scene.vel), abi.ptr(scene.affine),
                                       abi.ptr(scene.mass), scene.n), "mpm_upload_particles")
        if diffuse_max:
            g, a = abi.GenParams(), abi.AdvectParams()
            check(lib.mpm_default_diffuse_params(diffuse_max, ctypes.byref(g), ctypes.byref(a)), "defaults")
            check(lib.mpm_diffuse_enable(self.h, diffuse_max, ctypes.byref(g), ctypes.byref(a)), "diffuse_enable")

    def frame(self, P, W, H, dims, substeps=1):
        lib = self.lib
        check(lib.mpm_set_params(self.h, ctypes.byref(P)), "mpm_set_params")
        check(lib.mpm_set_walls(self.h, ctypes.byref(W)), "mpm_set_walls")
        if H is not None:
            d = (ctypes.c_int32 * 3)(*dims)
            check(lib.mpm_set_hand(self.h, ctypes.byref(H), int(any(dims) and H.is_on != 0), d), "mpm_set_hand")
        check(lib.mpm_step(self.h, substeps), "mpm_step")

    def read(self, name):
        n, G, M = self.n, self.G, self.M
        shapes = {"pos": ((n, 4), np.float32), "vel": ((n, 4), np.float32), "affine": ((n, 9), np.float32),
                  "mass": ((n,), np.float32), "density": ((n,), np.float32),
                  "cell_mv": ((G, 3), np.int32), "cell_mass": ((G,), np.int32),
                  "cell_mv_f32": ((G, 3), np.float32), "cell_mass_f32": ((G,), np.float32),
                  "diffuse": ((M,), DIFFUSE_DTYPE), "free_list": ((M,), np.uint32), "top": ((1,), np.int32)}
        shape, dt = shapes[name]
        a = np.zeros(shape, dt)
        which = BUF["free_top" if name == "top" else name]
        check(self.lib.mpm_download(self.h, which, abi.ptr(a), a.nbytes), "mpm_download")
        return a

    def state(self):
        keys = FLUID_KEYS + (DIFFUSE_KEYS if self.M else ())
        return {k: self.read(k) for k in keys}

    def close(self):
        if self.h:
            self.lib.mpm_destroy(self.h)
            self.h = None


ENGINES = {"binned": 0, "plain": 1}


def gpu_run(lib, scenario, engine="binned"):
    g = GpuScene(lib, scenario.scene, scenario.diffuse_max, flags=ENGINES[engine])
    try:
        for P, W, H, dims, gen, adv in scenario.frames():
            g.frame(P, W, H, dims)
            yield g.state()
    finally:
        g.close()


def diff_report(a, b, keys=None):
    """Names of arrays that differ bitwise, with the first differing index."""
    out = []
    for k in keys or a.keys():
        if k not in b:
            continue
        x, y = np.ascontiguousarray(a[k]), np.ascontiguousarray(b[k])
        if x.shape != y.shape:
            out.append(f"{k}: shape {x.shape} vs {y.shape}")
            continue
        xb, yb = x.view(np.uint8).reshape(len(x), -1) if len(x) else x, y.view(np.uint8).reshape(len(y), -1) if len(y) else y
        if len(x) and not np.array_equal(xb, yb):
            idx = np.nonzero((xb != yb).any(axis=1))[0]
            out.append(f"{k}: {idx.size} rows differ, first {idx[0]}: {x[idx[0]]} vs {y[idx[0]]}")
    return out
