"""Reference-layout render buffers (particle_pos, particle_vel,
particle_density) kept current by every substep once a consumer has taken
their device pointers: the bytes at the pointers equal the oracle's state
after each later step, with no export call in between, and the pointers never
move (fluid-renderer.js:315-328 binds them once as vertex inputs)."""
import ctypes

import numpy as np
import pytest

import oracle as O
import scenarios as S
from mls_mpm_b200.abi import BUF, check
from runner import GpuScene, diff_report

pytestmark = pytest.mark.gpu


def _read_device(ptr, nbytes, dtype, shape):
    from cuda.bindings import driver
    out = np.empty(shape, dtype)
    assert out.nbytes == nbytes
    err, = driver.cuMemcpyDtoH(out.ctypes.data, ptr, nbytes)
    assert err == driver.CUresult.CUDA_SUCCESS, err
    return out


def _pointer(lib, h, name):
    p, sz = ctypes.c_void_p(), ctypes.c_size_t()
    check(lib.mpm_get_buffer(h, BUF[name], ctypes.byref(p), ctypes.byref(sz)), "mpm_get_buffer")
    return p.value, sz.value


@pytest.mark.parametrize("name", ["walls_hand_diffuse", "crowded"])
def test_render_buffers_follow_every_step(gpu, name):
    scn = S.SCENARIOS[name]()
    scn.substeps = min(scn.substeps, 12)
    g = GpuScene(gpu, scn.scene, scn.diffuse_max)
    st = O.new_state(scn.scene, scn.diffuse_max)
    n = scn.scene.n
    ptrs = None
    try:
        for s, (P, W, H, dims, gen, adv) in enumerate(scn.frames()):
            g.frame(P, W, H, dims)
            O.substep(st, P, W, H, dims, gen, adv)
            if s == 1:   # the consumer binds its vertex buffers after the first frames
                ptrs = {k: _pointer(gpu, g.h, k) for k in ("pos", "vel", "density")}
            if ptrs is None:
                continue
            check(gpu.mpm_sync(g.h), "mpm_sync")
            assert {k: _pointer(gpu, g.h, k) for k in ptrs} == ptrs          # the pointers stay put
            got = {"pos": _read_device(ptrs["pos"][0], n * 16, np.float32, (n, 4)),
                   "vel": _read_device(ptrs["vel"][0], n * 16, np.float32, (n, 4)),
                   "density": _read_device(ptrs["density"][0], n * 4, np.float32, (n,))}
            bad = diff_report(got, st)
            assert not bad, f"{name} substep {s}: {bad}"
        # the rest of the state is unaffected by the mirror writes
        assert not diff_report(g.state(), st)
    finally:
        g.close()
