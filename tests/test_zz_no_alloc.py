"""mpm_compact_noalloc against mpm_compact: same survivors, counts and order
on two calls in a row with different inputs (the second call must not see
the first call's scratch); no allocation from the device's default memory
pool during a call, where mpm_compact's stream-ordered scratch shows up (so
the check can see an allocation); n = 0, NULL arguments and the size limit
rejected or handled on the host.  mpm_compact_noalloc is for callers that
must not allocate device memory while they run: a frame loop with a fixed
memory plan, or a host whose allocator belongs to someone else.  Collected
last so it also runs after every other GPU test in the same process."""
import ctypes

import numpy as np
import pytest

from mls_mpm_b200 import abi
from mls_mpm_b200.abi import COMPACT_NOALLOC_MAX_N, check

pytestmark = pytest.mark.gpu


def _inputs(rng, n):
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0, 48, (n, 3))
    vel = rng.standard_normal((n, 4)).astype(np.float32)
    mass = rng.uniform(0.5, 2.0, n).astype(np.float32)
    return pos, vel, mass


def _ray(o, d, r):
    d = np.asarray(d, np.float64)
    d = d / np.linalg.norm(d)
    rp = abi.RayParams()
    rp.ox, rp.oy, rp.oz = o
    rp.radius = r
    rp.dx, rp.dy, rp.dz = (float(x) for x in d)
    return rp


def _outputs(tensors):
    import torch
    tp, tv, tm = tensors
    cnt = torch.full((1,), 99, dtype=torch.int32, device=tp.device)
    return cnt, torch.full_like(tp, -7.0), torch.full_like(tv, -7.0), torch.full_like(tm, -7.0)


class _PoolHighWater:
    """High-water mark of the device's default memory pool (where
    cudaMallocAsync takes stream-ordered memory), through the driver API."""

    def __init__(self, ordinal=0):
        from cuda.bindings import driver
        self.d = driver
        err, = driver.cuInit(0)
        assert err == driver.CUresult.CUDA_SUCCESS, err
        err, dev = driver.cuDeviceGet(ordinal)
        assert err == driver.CUresult.CUDA_SUCCESS, err
        err, self.pool = driver.cuDeviceGetDefaultMemPool(dev)
        assert err == driver.CUresult.CUDA_SUCCESS, err

    def _attr(self, name):
        err, v = self.d.cuMemPoolGetAttribute(self.pool, getattr(self.d.CUmemPool_attribute, name))
        assert err == self.d.CUresult.CUDA_SUCCESS, err
        return int(v)

    def reset(self):
        """Restart the high-water mark at the bytes in use now; returns them."""
        zero = self.d.cuuint64_t(0)
        err, = self.d.cuMemPoolSetAttribute(self.pool, self.d.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                           zero)
        assert err == self.d.CUresult.CUDA_SUCCESS, err
        return self._attr("CU_MEMPOOL_ATTR_USED_MEM_CURRENT")

    def high(self):
        return self._attr("CU_MEMPOOL_ATTR_USED_MEM_HIGH")


def _run(lib, fn, ray, tensors, n, stream, outs=None):
    tp, tv, tm = tensors
    cnt, op, ov, om = outs if outs is not None else _outputs(tensors)
    check(getattr(lib, fn)(ctypes.byref(ray), n, tp.data_ptr(), tv.data_ptr(), tm.data_ptr(), op.data_ptr(),
                           ov.data_ptr(), om.data_ptr(), cnt.data_ptr(), stream), fn)
    return cnt, op, ov, om


def test_noalloc_compact_matches_mpm_compact_two_calls_in_a_row(gpu):
    import torch
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(2024)
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(300_001, _ray((24.0, 24.0, 24.0), (1.0, 0.5, 0.2), 9.0)),   # drops a thick cylinder
             (70_000, _ray((5.0, 40.0, 10.0), (0.0, 0.0, 1.0), 2.0))]     # fewer particles, thin cylinder
    pool = _PoolHighWater(0)
    for n, ray in cases:
        tensors = tuple(torch.from_numpy(a).to(dev) for a in _inputs(rng, n))
        outs = _outputs(tensors)
        torch.cuda.synchronize()
        in_use = pool.reset()
        got = _run(gpu, "mpm_compact_noalloc", ray, tensors, n, stream, outs)
        torch.cuda.synchronize()
        # nothing was taken from the pool during the call
        assert pool.high() == in_use
        in_use = pool.reset()
        want = _run(gpu, "mpm_compact", ray, tensors, n, stream)
        torch.cuda.synchronize()
        # the allocating entry point does show up: the check can see an allocation
        assert pool.high() > in_use
        m = int(want[0].item())
        assert int(got[0].item()) == m
        assert 0 < m < n
        for g, w in zip(got[1:], want[1:]):
            assert torch.equal(g[:m].view(torch.int32), w[:m].view(torch.int32))
            # nothing past the survivors is written
            assert bool((g[m:] == -7.0).all())


def test_noalloc_compact_empty_input_sets_count_only(gpu):
    """n = 0: *count_dev becomes 0 and no output is touched."""
    import torch
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(11)
    tensors = tuple(torch.from_numpy(a).to(dev) for a in _inputs(rng, 8))
    outs = _outputs(tensors)
    ray = _ray((1.0, 1.0, 1.0), (0.0, 1.0, 0.0), 3.0)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        cnt, op, ov, om = _run(gpu, "mpm_compact_noalloc", ray, tensors, 0, stream, outs)
        torch.cuda.synchronize()
        assert int(cnt.item()) == 0
        for o in (op, ov, om):
            assert bool((o == -7.0).all())
        cnt.fill_(99)


def test_noalloc_compact_null_arguments_rejected(gpu):
    import torch
    dev = torch.device("cuda:0")
    t = torch.zeros((4, 4), dtype=torch.float32, device=dev)
    cnt = torch.zeros((1,), dtype=torch.int32, device=dev)
    ray = _ray((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 1.0)
    p = t.data_ptr()
    stream = torch.cuda.current_stream().cuda_stream
    # NULL ray, NULL count, NULL input with n > 0: MPM_ERR_INVALID_ARG, nothing enqueued
    assert gpu.mpm_compact_noalloc(None, 4, p, p, p, p, p, p, cnt.data_ptr(), stream) == 1
    assert gpu.mpm_compact_noalloc(ctypes.byref(ray), 4, p, p, p, p, p, p, None, stream) == 1
    assert gpu.mpm_compact_noalloc(ctypes.byref(ray), 4, None, p, p, p, p, p, cnt.data_ptr(), stream) == 1
    assert b"NULL" in gpu.mpm_last_error()


def test_noalloc_compact_rejects_oversize_on_the_host(gpu):
    import torch
    dev = torch.device("cuda:0")
    small = torch.zeros((4, 4), dtype=torch.float32, device=dev)
    cnt = torch.zeros((1,), dtype=torch.int32, device=dev)
    ray = _ray((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 1.0)
    st = gpu.mpm_compact_noalloc(ctypes.byref(ray), COMPACT_NOALLOC_MAX_N + 1, small.data_ptr(), small.data_ptr(),
                                 small.data_ptr(), small.data_ptr(), small.data_ptr(), small.data_ptr(),
                                 cnt.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == 9   # MPM_ERR_CAPACITY
    assert b"MPM_COMPACT_NOALLOC_MAX_N" in gpu.mpm_last_error()


def test_noalloc_compact_at_the_limit(gpu):
    """n == MPM_COMPACT_NOALLOC_MAX_N uses every scratch word."""
    import torch
    dev = torch.device("cuda:0")
    n = COMPACT_NOALLOC_MAX_N
    g = torch.Generator(device=dev).manual_seed(5)
    tp = torch.rand((n, 4), generator=g, device=dev) * 48.0
    tv = torch.arange(n, device=dev, dtype=torch.float32).repeat_interleave(4).view(n, 4)
    tm = torch.arange(n, device=dev, dtype=torch.float32)
    ray = _ray((24.0, 24.0, 24.0), (0.3, 1.0, 0.1), 12.0)
    stream = torch.cuda.current_stream().cuda_stream
    got = _run(gpu, "mpm_compact_noalloc", ray, (tp, tv, tm), n, stream)
    want = _run(gpu, "mpm_compact", ray, (tp, tv, tm), n, stream)
    torch.cuda.synchronize()
    m = int(want[0].item())
    assert int(got[0].item()) == m and 0 < m < n
    for a, b in zip(got[1:], want[1:]):
        assert torch.equal(a[:m].view(torch.int32), b[:m].view(torch.int32))
    # survivors keep index order (mass holds the source index)
    assert bool((got[3][1:m] > got[3][:m - 1]).all())
