"""Python driver for the CPU oracle (mpm_oracle.cpp) and the reference pin
(oracle/_ref, the reference's WGSL compiled on the host).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product.

State is a dict of numpy arrays in the reference layouts:
  pos (N,4) f32, vel (N,4) f32, affine (N,9) f32, mass (N,) f32, density (N,) f32,
  cell_mv (G,3) i32, cell_mass (G,) i32, cell_mv_f32 (G,3) f32, cell_mass_f32 (G,) f32,
  and with diffuse: diffuse (M,) DIFFUSE_DTYPE, free_list (M,) u32, top (1,) i32.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "lib", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmpm_ref.so")

_libs = {}


def build_oracle():
    """Compile the oracle, and the reference pin when the reference checkout is
    present.  Where the checkout lies is the recipe's business: environment
    variable MPM_REFERENCE_DIR, else the Makefile's default; the recipe skips
    the pin when that directory holds no shaders.js."""
    subprocess.run(["make", "-s", "-C", HERE, "lib/liboracle.so"], check=True)
    subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)


def _load(path, build=True):
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path) and build:
        build_oracle()
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    _libs[path] = lib
    return lib


def oracle_lib():
    lib = _load(ORACLE_SO)
    if lib is None:
        raise RuntimeError("oracle library could not be built")
    return lib


def ref_lib():
    """The reference pin, or None when it was not built (no reference checkout)."""
    return _load(REF_SO)


def ref_available():
    return ref_lib() is not None


def new_state(scene, diffuse_max=0):
    """Oracle state for a mls_mpm_b200.scenes.Scene (copies its arrays)."""
    from mls_mpm_b200.abi import DIFFUSE_DTYPE
    X, Y, Z = scene.grid
    G = X * Y * Z
    st = {
        "pos": scene.pos.copy(), "vel": scene.vel.copy(), "affine": scene.affine.copy(),
        "mass": scene.mass.copy(), "density": np.zeros(scene.n, np.float32),
        "cell_mv": np.zeros((G, 3), np.int32), "cell_mass": np.zeros(G, np.int32),
        "cell_mv_f32": np.zeros((G, 3), np.float32), "cell_mass_f32": np.zeros(G, np.float32),
    }
    if diffuse_max:
        st["diffuse"] = np.zeros(diffuse_max, DIFFUSE_DTYPE)
        st["free_list"] = np.arange(diffuse_max, dtype=np.uint32)
        st["top"] = np.array([diffuse_max], np.int32)
    return st


def to_f64(st):
    out = {}
    for k, v in st.items():
        out[k] = v.astype(np.float64) if v.dtype == np.float32 else v.copy()
    if "diffuse" in st:
        out["diffuse"] = st["diffuse"].copy()   # f64 diffuse is not tracked
    return out


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _byref(s):
    return None if s is None else ctypes.byref(s)


def substep(st, params, walls=None, hand=None, hand_dims=None, gen=None, adv=None, threads=1,
            impl="oracle"):
    """One simFrame substep in place.  impl: 'oracle' (f32 restatement),
    'f64' (binary64 restatement, arrays must be float64), 'ref' (reference pin)."""
    dims = None if hand_dims is None else np.ascontiguousarray(hand_dims, np.int32)
    if impl == "ref":
        lib = ref_lib()
        if lib is None:
            raise RuntimeError("reference pin not built")
        fn = lib.ref_substep_f32
    elif impl == "f64":
        fn = oracle_lib().oracle_substep_f64
    else:
        fn = oracle_lib().oracle_substep_f32
    fn.restype = None
    dif = st.get("diffuse") if gen is not None else None
    fn(_byref(params), _byref(walls), _byref(hand), _p(dims),
       _p(st["pos"]), _p(st["vel"]), _p(st["affine"]), _p(st["mass"]), _p(st["density"]),
       _p(st["cell_mv"]), _p(st["cell_mass"]), _p(st["cell_mv_f32"]), _p(st["cell_mass_f32"]),
       _byref(gen), _byref(adv), _p(dif),
       _p(st.get("free_list") if dif is not None else None),
       _p(st.get("top") if dif is not None else None), ctypes.c_int(threads))


def compact(params, ray, pos, vel, mass, impl="oracle"):
    n = params.particle_num
    po, vo, mo = np.zeros_like(pos), np.zeros_like(vel), np.zeros_like(mass)
    lib = ref_lib() if impl == "ref" else oracle_lib()
    fn = lib.ref_compact_f32 if impl == "ref" else lib.oracle_compact_f32
    fn.restype = ctypes.c_uint32
    cnt = fn(ctypes.byref(params), ctypes.byref(ray), _p(pos), _p(vel), _p(mass), _p(po), _p(vo), _p(mo))
    return int(cnt), po, vo, mo


def raycast(params, ray, pos, impl="oracle"):
    lib = ref_lib() if impl == "ref" else oracle_lib()
    fn = lib.ref_raycast_f32 if impl == "ref" else lib.oracle_raycast_f32
    fn.restype = ctypes.c_uint32
    return int(fn(ctypes.byref(params), ctypes.byref(ray), _p(pos)))


STATE_KEYS = ("pos", "vel", "affine", "density", "cell_mv", "cell_mass", "cell_mv_f32", "cell_mass_f32")


def digest(st, keys=STATE_KEYS):
    """sha256 per array (hex), for golden fixtures."""
    import hashlib
    out = {}
    for k in keys:
        if k in st:
            out[k] = hashlib.sha256(np.ascontiguousarray(st[k]).tobytes()).hexdigest()
    if "diffuse" in st:
        for k in ("diffuse", "free_list", "top"):
            out[k] = hashlib.sha256(np.ascontiguousarray(st[k]).tobytes()).hexdigest()
    return out
