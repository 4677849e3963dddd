"""Zero-copy export through CUDA IPC: a second process opens the handle that
mpm_get_ipc_handle returns and reads the same bytes mpm_download returns."""
import os
import subprocess
import sys

import numpy as np
import pytest

import scenarios

# The consumer: opens the IPC handle with the CUDA runtime through ctypes and
# copies the buffer to a file.
CONSUMER = r"""
import ctypes, glob, os, sys
handle_hex, offset, nbytes, out = sys.argv[1], int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
cands = ["libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so.12"]
cands += glob.glob(os.path.join(sys.prefix, "lib", "python*", "site-packages", "nvidia", "cuda_runtime", "lib",
                                "libcudart.so.12"))
rt = None
for c in cands:
    try:
        rt = ctypes.CDLL(c)
        break
    except OSError:
        pass
assert rt is not None, "no CUDA runtime library"
class Handle(ctypes.Structure):
    _fields_ = [("reserved", ctypes.c_char * 64)]
h = Handle()
ctypes.memmove(ctypes.addressof(h), bytes.fromhex(handle_hex), 64)
assert rt.cudaSetDevice(0) == 0
ptr = ctypes.c_void_p()
rt.cudaIpcOpenMemHandle.argtypes = [ctypes.POINTER(ctypes.c_void_p), Handle, ctypes.c_uint]
err = rt.cudaIpcOpenMemHandle(ctypes.byref(ptr), h, 1)
assert err == 0, f"cudaIpcOpenMemHandle: {err}"
buf = ctypes.create_string_buffer(nbytes)
rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
err = rt.cudaMemcpy(buf, ctypes.c_void_p(ptr.value + offset), nbytes, 2)
assert err == 0, f"cudaMemcpy: {err}"
rt.cudaIpcCloseMemHandle(ptr)
open(out, "wb").write(buf.raw)
"""


@pytest.mark.gpu
def test_ipc_export_matches_download(gpu, tmp_path):
    from mls_mpm_b200 import DiffuseGPU, FluidGPU
    sc = scenarios.walls_hand_diffuse()
    fl = FluidGPU.from_scene(sc.scene)
    DiffuseGPU(sc.diffuse_max).initGPU(0, fl)
    for _ in range(4):
        fl.simFrame()
    fl.sync()
    try:
        for name in ("pos", "density", "cell_mass_f32", "cell_mv", "diffuse"):
            handle, offset, nbytes = fl.get_ipc_handle(name)
            fl.sync()
            want = np.ascontiguousarray(fl.read(name)).tobytes()
            out = tmp_path / f"{name}.bin"
            r = subprocess.run([sys.executable, "-c", CONSUMER, handle.hex(), str(offset), str(len(want)), str(out)],
                               capture_output=True, text=True, timeout=300, env=dict(os.environ))
            assert r.returncode == 0, r.stderr[-2000:]
            assert nbytes >= len(want)
            assert out.read_bytes() == want, name
    finally:
        fl.destroy()
