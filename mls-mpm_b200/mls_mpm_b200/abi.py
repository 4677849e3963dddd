"""ctypes mirrors of include/mpm_types.h and include/mpm_b200.h, plus the
library loader.

The structs are byte-for-byte the reference's uniform/storage layouts
(shaders.js:27-49, 123-133, 395-402, 725-743, 872-877), so the bytes a
JavaScript host would pass to queue.writeBuffer can be passed through
unchanged.  Loading the native library never falls back to anything else:
if libmpm_b200.so is missing, every entry point raises.
"""
import ctypes
import os

import numpy as np

MAX_WALLS = 4                 # config.js:11
DIFFUSE_MAX_COUNT = 30000     # config.js:7 (desktop)
WG_SIZE = 64                  # config.js:2 (desktop)

c_float_p = ctypes.POINTER(ctypes.c_float)


class Params(ctypes.Structure):
    """Params uniform (80 B), shaders.js:27-49 / fluid-gpu.js:295-313."""
    _fields_ = [("grid_X", ctypes.c_uint32), ("grid_Y", ctypes.c_uint32),
                ("grid_Z", ctypes.c_uint32), ("particle_num", ctypes.c_uint32),
                ("dt", ctypes.c_float), ("gravity", ctypes.c_float),
                ("rest_density", ctypes.c_float), ("stiffness", ctypes.c_float),
                ("eos_power", ctypes.c_float), ("viscosity", ctypes.c_float),
                ("hard_min", ctypes.c_float), ("hard_max_x", ctypes.c_float),
                ("hard_max_y", ctypes.c_float), ("hard_max_z", ctypes.c_float),
                ("wall_min", ctypes.c_float), ("wall_stiffness", ctypes.c_float),
                ("lookahead_k", ctypes.c_float), ("_pad0", ctypes.c_float),
                ("_pad1", ctypes.c_float), ("_pad2", ctypes.c_float)]


class Wall(ctypes.Structure):
    """One wall OBB (80 B), shaders.js:123-129."""
    _fields_ = [("center_cy", ctypes.c_float * 4), ("lmin_sy", ctypes.c_float * 4),
                ("lmax_cp", ctypes.c_float * 4), ("vel_sp", ctypes.c_float * 4),
                ("omega_pad", ctypes.c_float * 4)]


class WallParams(ctypes.Structure):
    """WallParams uniform (336 B), shaders.js:130-133."""
    _fields_ = [("count_pad", ctypes.c_float * 4), ("walls", Wall * MAX_WALLS)]


class HandParams(ctypes.Structure):
    """HandParams uniform (80 B), shaders.js:395-402."""
    _fields_ = [("px", ctypes.c_float), ("py", ctypes.c_float), ("pz", ctypes.c_float),
                ("radius", ctypes.c_float), ("vx", ctypes.c_float), ("vy", ctypes.c_float),
                ("vz", ctypes.c_float), ("is_on", ctypes.c_uint32), ("strength", ctypes.c_float),
                ("ex", ctypes.c_float), ("ey", ctypes.c_float), ("ez", ctypes.c_float),
                ("bbox_min_x", ctypes.c_int32), ("bbox_min_y", ctypes.c_int32),
                ("bbox_min_z", ctypes.c_int32), ("bbox_max_x", ctypes.c_int32),
                ("bbox_max_y", ctypes.c_int32), ("bbox_max_z", ctypes.c_int32),
                ("_pad0", ctypes.c_int32), ("_pad1", ctypes.c_int32)]


class GenParams(ctypes.Structure):
    """GenParams uniform (32 B), shaders.js:734-743 / diffuse-gpu.js:84-94."""
    _fields_ = [("ke_threshold", ctypes.c_float), ("spawn_rate_k", ctypes.c_float),
                ("density_spray_max", ctypes.c_float), ("density_bubble_min", ctypes.c_float),
                ("lifetime_foam", ctypes.c_float), ("pressure_threshold", ctypes.c_float),
                ("crest_dot_threshold", ctypes.c_float), ("seed", ctypes.c_uint32)]


class AdvectParams(ctypes.Structure):
    """AdvectParams uniform (16 B), shaders.js:872-877 / diffuse-gpu.js:70-76."""
    _fields_ = [("diffuse_max", ctypes.c_uint32), ("buoyancy", ctypes.c_float),
                ("drag", ctypes.c_float), ("_pad", ctypes.c_float)]


class RayParams(ctypes.Structure):
    """RayParams uniform (32 B), shaders.js:78."""
    _fields_ = [("ox", ctypes.c_float), ("oy", ctypes.c_float), ("oz", ctypes.c_float),
                ("radius", ctypes.c_float), ("dx", ctypes.c_float), ("dy", ctypes.c_float),
                ("dz", ctypes.c_float), ("_pad", ctypes.c_float)]


# DiffuseParticle (48 B), shaders.js:725-732.
DIFFUSE_DTYPE = np.dtype([("pos", "<f4", (4,)), ("vel", "<f4", (4,)), ("ptype", "<u4"),
                          ("alive", "<u4"), ("lifetime", "<f4"), ("_pad", "<f4")])

for _s, _n in ((Params, 80), (Wall, 80), (WallParams, 336), (HandParams, 80), (GenParams, 32),
               (AdvectParams, 16), (RayParams, 32)):
    assert ctypes.sizeof(_s) == _n, (_s, ctypes.sizeof(_s))
assert DIFFUSE_DTYPE.itemsize == 48


def ptr(a):
    """Raw data pointer of a C-contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return ctypes.c_void_p(a.ctypes.data)


# ---------------------------------------------------------------------------
# Native library (include/mpm_b200.h).  Built in-tree by
# mls_mpm_b200.build.build(); there is no fallback path.
# ---------------------------------------------------------------------------
PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libmpm_b200.so")

_lib = None


class MpmError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__(f"{what} failed: {status_name(status)} ({status}): {last_error()}")


STATUS = {0: "MPM_OK", 1: "MPM_ERR_INVALID_ARG", 2: "MPM_ERR_OOM", 3: "MPM_ERR_DEVICE",
          4: "MPM_ERR_TIMEOUT", 5: "MPM_ERR_NAN", 6: "MPM_ERR_NO_DEVICE", 7: "MPM_ERR_BUSY",
          8: "MPM_ERR_UNSUPPORTED", 9: "MPM_ERR_CAPACITY"}


def status_name(s):
    return STATUS.get(s, "MPM_ERR_UNKNOWN")


def load_library(path=None):
    """Load libmpm_b200.so (raises if it is absent — the product has no CPU path)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"native library missing: {p} (run __graft_entry__.build())")
    lib = ctypes.CDLL(p)
    _declare(lib)
    if path is None:
        _lib = lib
    return lib


def last_error():
    if _lib is None:
        return ""
    return _lib.mpm_last_error().decode(errors="replace")


def check(status, what):
    if status != 0:
        raise MpmError(status, what)


# name -> (restype, argtypes)
_V = ctypes.c_void_p
_I = ctypes.c_int
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_SZ = ctypes.c_size_t
SIGNATURES = {
    "mpm_abi_version": (_I, []),
    "mpm_last_error": (ctypes.c_char_p, []),
    "mpm_device_count": (_I, [ctypes.POINTER(_I)]),
    "mpm_create": (_I, [_V, ctypes.POINTER(_V)]),
    "mpm_destroy": (_I, [_V]),
    "mpm_upload_particles": (_I, [_V, _V, _V, _V, _V, _U32]),
    "mpm_set_params": (_I, [_V, _V]),
    "mpm_set_walls": (_I, [_V, _V]),
    "mpm_set_hand": (_I, [_V, _V, _I, _V]),
    "mpm_diffuse_enable": (_I, [_V, _U32, _V, _V]),
    "mpm_diffuse_set_gen_params": (_I, [_V, _V]),
    "mpm_step": (_I, [_V, _I]),
    "mpm_sync": (_I, [_V]),
    "mpm_get_buffer": (_I, [_V, _I, ctypes.POINTER(_V), ctypes.POINTER(_SZ)]),
    "mpm_download": (_I, [_V, _I, _V, _SZ]),
    "mpm_upload": (_I, [_V, _I, _V, _SZ]),
    "mpm_diffuse_alive_count": (_I, [_V, ctypes.POINTER(ctypes.c_int32)]),
    "mpm_diffuse_request_alive": (_I, [_V]),
    "mpm_get_ipc_handle": (_I, [_V, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                ctypes.POINTER(ctypes.c_size_t)]),
    "mpm_diffuse_poll_alive": (_I, [_V, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
    "mpm_get_stream": (_I, [_V, ctypes.POINTER(_V)]),
    "mpm_phase_name": (ctypes.c_char_p, [_I]),
    "mpm_profile_enable": (_I, [_V, _I]),
    "mpm_profile_read": (_I, [_V, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_U64), _I]),
    "mpm_launch_count": (_I, [_V, ctypes.POINTER(_U64)]),
    "mpm_default_params": (_I, [_V, _V]),
    "mpm_default_diffuse_params": (_I, [_U32, _V, _V]),
    "mpm_desc_from_aspect": (_I, [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, _U32, _V]),
    "mpm_delete_near": (_I, [_V, _V, _V, ctypes.c_double, ctypes.POINTER(_U32)]),
    "mpm_raycast_fluid": (_I, [_V, _V, _V, ctypes.c_double, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_float), _V]),
    "mpm_append_particles": (_I, [_V, _V, _V, _V, _U32, ctypes.POINTER(_U32)]),
    "mpm_compact": (_I, [_V, _U32, _V, _V, _V, _V, _V, _V, _V, _V]),
    "mpm_raycast": (_I, [_V, _U32, _V, _V, _V]),
    "mpm_compact_noalloc": (_I, [_V, _U32, _V, _V, _V, _V, _V, _V, _V, _V]),
    "mpm_batch_footprint": (_I, [_U32, _U64, _U32, ctypes.POINTER(_U64)]),
    "mpm_batch_create": (_I, [_V, ctypes.POINTER(_V)]),
    "mpm_batch_destroy": (_I, [_V]),
    "mpm_batch_add": (_I, [_V, _V, _V, _V, _V, _V, _V, _U32, ctypes.POINTER(ctypes.c_int32)]),
    "mpm_batch_remove": (_I, [_V, ctypes.c_int32]),
    "mpm_batch_set_params": (_I, [_V, ctypes.c_int32, _V]),
    "mpm_batch_set_walls": (_I, [_V, ctypes.c_int32, _V]),
    "mpm_batch_set_hand": (_I, [_V, ctypes.c_int32, _V, _I, _V]),
    "mpm_batch_step": (_I, [_V, _I]),
    "mpm_batch_sync": (_I, [_V]),
    "mpm_batch_download": (_I, [_V, ctypes.c_int32, _I, _V, _SZ]),
    "mpm_batch_get_stream": (_I, [_V, ctypes.POINTER(_V)]),
    "mpm_batch_get_info": (_I, [_V, _V]),
    "mpm_server_create": (_I, [_V, ctypes.POINTER(_V)]),
    "mpm_server_destroy": (_I, [_V]),
    "mpm_server_submit": (_I, [_V, _V, _V, _V, _V, _U32, _U32, ctypes.c_double, ctypes.POINTER(ctypes.c_int64)]),
    "mpm_server_run": (_I, [_V, _V]),
    "mpm_server_job": (_I, [_V, ctypes.c_int64, _V]),
    "mpm_server_download": (_I, [_V, ctypes.c_int64, _I, _V, _SZ]),
    "mpm_wait": (_I, [_V, ctypes.c_double]),
    "mpm_set_device_memory_limit": (_I, [_U64]),
    "mpm_device_memory_in_use": (_I, [ctypes.POINTER(_U64)]),
    "mpm_get_health": (_I, [_V, ctypes.POINTER(_U32), _I]),
    "mpm_batch_get_health": (_I, [_V, ctypes.c_int32, ctypes.POINTER(_U32), _I]),
}

# MPM_HEALTH_* bits (mpm_get_health, mpm_batch_get_health, JobResult.health)
HEALTH_NONFINITE = 1
HEALTH_SATURATED = 2

SERVER_KEEP_STATE = 0x100


class ServerDesc(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("cells_per_particle", ctypes.c_double),
                ("scene_capacity", ctypes.c_uint32), ("device", ctypes.c_int32), ("flags", ctypes.c_uint32),
                ("max_inflight", ctypes.c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("jobs", ctypes.c_uint64), ("substeps", ctypes.c_uint64), ("particle_updates", ctypes.c_uint64),
                ("wall_s", ctypes.c_double), ("p50_latency_s", ctypes.c_double), ("p99_latency_s", ctypes.c_double),
                ("mean_latency_s", ctypes.c_double), ("max_latency_s", ctypes.c_double),
                ("mean_active", ctypes.c_double), ("max_active", ctypes.c_double),
                ("particle_capacity", ctypes.c_uint64), ("cell_capacity", ctypes.c_uint64),
                ("launches", ctypes.c_uint64)]


class JobResult(ctypes.Structure):
    _fields_ = [("arrival_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("finish_s", ctypes.c_double),
                ("n", ctypes.c_uint32), ("substeps", ctypes.c_uint32), ("done", ctypes.c_int32),
                ("health", ctypes.c_int32)]

BATCH_NO_GRAPH = 1
BATCH_AUTOTUNE = 2


class BatchDesc(ctypes.Structure):
    _fields_ = [("particle_capacity", ctypes.c_uint32), ("scene_capacity", ctypes.c_uint32),
                ("cell_capacity", ctypes.c_uint64), ("device", ctypes.c_int32), ("flags", ctypes.c_uint32)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("scenes", ctypes.c_uint32), ("particles", ctypes.c_uint32), ("cells", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("substeps", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64),
                ("item_blocks", ctypes.c_uint32), ("grid_blocks", ctypes.c_uint32)]

COMPACT_NOALLOC_MAX_N = 1 << 24

PHASE_COUNT = 10

BUF = {"pos": 0, "vel": 1, "affine": 2, "mass": 3, "density": 4, "cell_mv": 5, "cell_mass": 6,
       "cell_mv_f32": 7, "cell_mass_f32": 8, "diffuse": 9, "free_list": 10, "free_top": 11}


def _declare(lib):
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
