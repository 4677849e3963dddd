"""Alive-count readbacks (DiffuseGPU.requestDebugReadback / pollDebug,
diffuse-gpu.js:172-188) through the C ABI, both engines.

A request returns maxCount - top as of the work enqueued before it: after
steps (the value the last kill pass recorded on the device), after many more
steps than that device history holds, and after the caller uploaded the
free-list top (then top itself is copied).  Integer values, compared exactly.
"""
import ctypes

import numpy as np
import pytest

import scenarios
from runner import ENGINES, GpuScene
from mls_mpm_b200 import abi
from mls_mpm_b200.abi import BUF, check

pytestmark = pytest.mark.gpu

HISTORY = 256   # kill passes the device keeps (DiffuseState::kTopHist)


def _alive_sync(lib, g):
    a = ctypes.c_int32()
    check(lib.mpm_diffuse_alive_count(g.h, ctypes.byref(a)), "mpm_diffuse_alive_count")
    return a.value


def _request(lib, g):
    check(lib.mpm_diffuse_request_alive(g.h), "mpm_diffuse_request_alive")


def _poll(lib, g):
    a, ready = ctypes.c_int32(), ctypes.c_int32()
    check(lib.mpm_diffuse_poll_alive(g.h, ctypes.byref(a), ctypes.byref(ready)), "mpm_diffuse_poll_alive")
    return a.value, ready.value


@pytest.mark.parametrize("engine", ["binned", "plain"])
def test_readback_value_as_of_request(gpu, engine):
    sc = scenarios.walls_hand_diffuse()
    frames = list(sc.frames())
    lib = gpu
    g = GpuScene(lib, sc.scene, sc.diffuse_max, flags=ENGINES[engine])
    try:
        def step(i):
            P, W, H, dims, _, _ = frames[min(i, len(frames) - 1)]
            g.frame(P, W, H, dims)

        for i in range(6):
            step(i)
        want = _alive_sync(lib, g)
        _request(lib, g)
        # more kill passes than the device history holds, no poll in between
        for i in range(6, 6 + HISTORY + 40):
            step(i)
        check(lib.mpm_sync(g.h), "mpm_sync")
        assert _poll(lib, g) == (want, 1)
        assert _poll(lib, g) == (want, 0)   # nothing new landed

        # one readback per step, polled without waiting: every value landed by
        # the final sync equals the count right after its step
        seen = []
        for i in range(3):
            step(HISTORY + 46 + i)
            seen.append(_alive_sync(lib, g))
            _request(lib, g)
        check(lib.mpm_sync(g.h), "mpm_sync")
        assert _poll(lib, g) == (seen[-1], 1)

        # the caller moves the free-list top: the next readback copies top itself
        top = g.read("top")
        moved = np.array([top[0] - 3], np.int32)
        check(lib.mpm_upload(g.h, BUF["free_top"], abi.ptr(moved), 4), "mpm_upload")
        _request(lib, g)
        check(lib.mpm_sync(g.h), "mpm_sync")
        assert _poll(lib, g) == (sc.diffuse_max - int(moved[0]), 1)
        # and after the next step the kill pass's record again
        step(HISTORY + 50)
        after = _alive_sync(lib, g)
        _request(lib, g)
        check(lib.mpm_sync(g.h), "mpm_sync")
        assert _poll(lib, g) == (after, 1)
    finally:
        g.close()


def test_readback_requested_right_after_steps(gpu):
    """Binned engine: a step leaves its DiffuseGPU.step (spawn, ADVECT, kill)
    to run beside the next step's first passes; a readback requested right
    after the step still reports the count that step leaves.  The same frames
    on a second scene, read synchronously after every step, give the values."""
    sc = scenarios.walls_hand_diffuse()
    frames = list(sc.frames())
    lib = gpu
    ref = GpuScene(lib, sc.scene, sc.diffuse_max)
    g = GpuScene(lib, sc.scene, sc.diffuse_max)
    try:
        want = []
        for i in range(len(frames)):
            ref.frame(*frames[i][:4])
            want.append(_alive_sync(lib, ref))
        assert len(set(want)) > 3          # the count moves
        last = -1
        for i in range(len(frames)):
            g.frame(*frames[i][:4])
            _request(lib, g)
            a, ready = _poll(lib, g)        # never waits; what landed is some earlier step's count
            if ready:
                k = want.index(a, last + 1 if last + 1 < len(want) else 0)
                assert k <= i
                last = k
        check(lib.mpm_sync(g.h), "mpm_sync")
        assert _poll(lib, g) == (want[-1], 1)
        # the whole state equals the reference scene's
        from runner import diff_report
        assert not diff_report(g.state(), ref.state())
    finally:
        g.close()
        ref.close()
