"""The C ABI library loads, exports every declared entry point, and its
argument checking and defaults work without a GPU."""
import ctypes
import glob
import os
import re

import pytest

from mls_mpm_b200 import abi
from mls_mpm_b200.fluid_gpu import Desc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*[\w\s\*]+?\b(mpm_\w+)\s*\(", src, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "mpm_create" in names and "mpm_step" in names and len(names) >= 20


def test_library_exports_every_declared_symbol(native):
    missing = [n for n in declared_functions() if not hasattr(native, n)]
    assert not missing, missing


def test_struct_sizes():
    assert ctypes.sizeof(abi.Params) == 80
    assert ctypes.sizeof(abi.WallParams) == 336
    assert ctypes.sizeof(abi.HandParams) == 80
    assert ctypes.sizeof(abi.GenParams) == 32
    assert ctypes.sizeof(abi.AdvectParams) == 16
    assert abi.DIFFUSE_DTYPE.itemsize == 48
    assert ctypes.sizeof(Desc) == 24


def test_version_and_defaults(native):
    assert native.mpm_abi_version() == 1
    d = Desc()
    assert native.mpm_desc_from_aspect(ctypes.c_double(2), ctypes.c_double(2), ctypes.c_double(3),
                                       ctypes.c_double(0.0125), 400000, ctypes.byref(d)) == 0
    assert (d.grid_X, d.grid_Y, d.grid_Z, d.particle_capacity) == (40, 40, 60, 400000)
    p = abi.Params()
    assert native.mpm_default_params(ctypes.byref(d), ctypes.byref(p)) == 0
    assert (p.dt, p.rest_density, p.stiffness, p.eos_power, p.viscosity) == (
        pytest.approx(0.3), 8.0, 100.0, 1.0, pytest.approx(0.01))
    assert (p.hard_min, p.hard_max_x, p.hard_max_z) == (2.0, 38.0, 58.0)
    g, a = abi.GenParams(), abi.AdvectParams()
    assert native.mpm_default_diffuse_params(30000, ctypes.byref(g), ctypes.byref(a)) == 0
    assert g.seed == 1 and a.diffuse_max == 30000 and g.ke_threshold == 0.5


def test_invalid_arguments_report_status(native):
    assert native.mpm_create(None, None) == 1
    assert b"NULL" in native.mpm_last_error()
    assert native.mpm_step(None, 1) == 1
    assert native.mpm_desc_from_aspect(ctypes.c_double(-1), ctypes.c_double(1), ctypes.c_double(1),
                                       ctypes.c_double(0.1), 1, ctypes.byref(Desc())) == 1


def test_create_without_device_is_an_error_not_a_fallback(native):
    n = ctypes.c_int()
    assert native.mpm_device_count(ctypes.byref(n)) == 0
    if n.value:
        pytest.skip("a GPU is visible; covered by the gpu tests")
    d = Desc(16, 16, 16, 100, 0, 0)
    h = ctypes.c_void_p()
    assert native.mpm_create(ctypes.byref(d), ctypes.byref(h)) == 6   # MPM_ERR_NO_DEVICE
    assert not h.value


def test_batch_footprint_without_device(native):
    """mpm_batch_footprint is host arithmetic: usable for admission before any device work."""
    import ctypes
    out = []
    for p, c, s in ((1 << 20, 1 << 21, 1), (1 << 22, 1 << 21, 64), (1 << 22, 1 << 23, 64)):
        b = ctypes.c_uint64()
        assert native.mpm_batch_footprint(p, c, s, ctypes.byref(b)) == 0
        out.append(b.value)
    # ~150 B per particle (two state copies + layout) + ~56 B per cell (two i32 grids + decoded grid)
    assert 140 * (1 << 20) + 50 * (1 << 21) < out[0] < 200 * (1 << 20) + 80 * (1 << 21)
    assert out[0] < out[1] < out[2]


def test_noalloc_source_calls_no_allocator():
    """mpm_compact_noalloc's source names no device allocator or pool call
    (comments aside), so the entry point cannot allocate on any path."""
    src = open(os.path.join(ROOT, "mls-mpm_b200", "csrc", "mpm_noalloc.cu")).read()
    code = re.sub(r"//[^\n]*", "", re.sub(r"/\*.*?\*/", "", src, flags=re.S))
    banned = re.findall(r"\b(cudaMalloc\w*|cudaFree\w*|cudaMemPool\w*|cuMem\w*|malloc|free|new\s|"
                        r"cudaHostAlloc|cudaMallocHost|c10|torch)\b", code)
    assert not banned, banned
