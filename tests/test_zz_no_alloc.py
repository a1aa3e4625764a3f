"""cryo_probe_pressure_noalloc against cryo_probe_pressure through the C ABI.

The no-allocation probe is for callers that must not allocate device memory
once running (a control loop probing tank pressure every cycle under a fixed
memory budget).  It stages points and results through one fixed device array
per device instead of a pool allocation per call; it must give the same
pressures as the allocating entry point (same kernel, same inputs: the
comparison allows 1e-6 relative), on two calls in a row, refuse more points
than its fixed array holds and a context that is not yet initialised, and
allocate nothing: the device's memory pool keeps its high-water mark and
reservation and the free device memory does not change across the call
(the allocating probe, measured the same way, does raise the mark).
Collected last so it also runs after every other GPU test in the same
process; it needs nothing from them."""
import ctypes as C

import numpy as np
import pytest

import cryo_cabi as cabi
import scenarios as S

pytestmark = pytest.mark.gpu

MAX_POINTS = 16384  # CRYO_PROBE_STATIC_MAX in include/cryosph_b200.h


def _probe(ctx, fn, pts):
    pts = np.ascontiguousarray(pts, np.float32)
    out = np.full(len(pts), -1.0, np.float32)
    rc = getattr(ctx.L, fn)(ctx.h, pts.ctypes.data_as(C.POINTER(C.c_float)), len(pts),
                            out.ctypes.data_as(C.POINTER(C.c_float)))
    return rc, out


def _points(lo, hi, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
    return (lo + (hi - lo) * rng.random((n, 3), dtype=np.float32)).astype(np.float32)


def _same(a, b):
    assert np.array_equal(np.isnan(a), np.isnan(b))
    ok = ~np.isnan(a)
    assert ok.any()
    scale = max(float(np.abs(b[ok]).max()), 1.0)
    assert float(np.abs(a[ok] - b[ok]).max()) <= 1e-6 * scale


def test_noalloc_probe_matches_the_allocating_probe(cuda_device):
    cfg, fl, parts, lo, hi = S.c1()
    ctx = cabi.Context(cfg, fl)
    ctx.set_particles(parts, lo, hi)
    ctx.step(3)
    for call, seed in enumerate((11, 12)):  # two calls in a row, different points
        pts = _points(lo, hi, 5000 + 97 * call, seed)
        rc_a, ref = _probe(ctx, "cryo_probe_pressure", pts)
        rc_b, got = _probe(ctx, "cryo_probe_pressure_noalloc", pts)
        assert rc_a == cabi.CRYO_OK and rc_b == cabi.CRYO_OK, ctx.L.cryo_last_error(ctx.h)
        assert (~np.isnan(ref)).sum() > len(pts) // 10  # inside the liquid for a fair share
        _same(got, ref)
    ctx.step(2)
    pts = _points(lo, hi, MAX_POINTS, 13)  # the largest size the fixed array takes
    _, ref = _probe(ctx, "cryo_probe_pressure", pts)
    rc, got = _probe(ctx, "cryo_probe_pressure_noalloc", pts)
    assert rc == cabi.CRYO_OK
    _same(got, ref)


def test_noalloc_probe_rejects_more_points_than_it_holds(cuda_device):
    cfg, fl, parts, lo, hi = S.c1()
    ctx = cabi.Context(cfg, fl)
    ctx.set_particles(parts, lo, hi)
    pts = _points(lo, hi, MAX_POINTS + 1, 14)
    rc, out = _probe(ctx, "cryo_probe_pressure_noalloc", pts)
    assert rc == cabi.CRYO_ERANGE
    assert b"fixed scratch" in ctx.L.cryo_last_error(ctx.h)
    assert (out == -1.0).all()
    # not initialised yet: initialising may allocate, so the call refuses
    rc, out = _probe(ctx, "cryo_probe_pressure_noalloc", pts[:100])
    assert rc == cabi.CRYO_EINVAL
    assert b"not initialised" in ctx.L.cryo_last_error(ctx.h)
    assert (out == -1.0).all()
    ctx.step(1)
    rc, _ = _probe(ctx, "cryo_probe_pressure_noalloc", pts[:100])
    assert rc == cabi.CRYO_OK


def _pool_marks():
    """(used high-water mark, reserved bytes) of device 0's current memory pool
    (the pool cudaMallocAsync draws on), through the driver API."""
    from cuda.bindings import driver as drv
    err, = drv.cuInit(0)
    assert err == drv.CUresult.CUDA_SUCCESS
    err, dev = drv.cuDeviceGet(0)
    assert err == drv.CUresult.CUDA_SUCCESS
    err, pool = drv.cuDeviceGetMemPool(dev)
    assert err == drv.CUresult.CUDA_SUCCESS
    out = []
    for attr in (drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                 drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT):
        err, v = drv.cuMemPoolGetAttribute(pool, attr)
        assert err == drv.CUresult.CUDA_SUCCESS
        out.append(int(v))
    return pool, out[0], out[1]


def _reset_high_mark(pool):
    from cuda.bindings import driver as drv
    err, = drv.cuMemPoolSetAttribute(pool, drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                     drv.cuuint64_t(0))
    assert err == drv.CUresult.CUDA_SUCCESS


def test_noalloc_probe_allocates_nothing(cuda_device):
    import torch
    cfg, fl, parts, lo, hi = S.c1()
    ctx = cabi.Context(cfg, fl)
    ctx.set_particles(parts, lo, hi)
    ctx.step(2)
    pts = _points(lo, hi, MAX_POINTS, 15)
    ctx.L.cryo_synchronize(ctx.h)
    # the measurement sees a pool allocation: the allocating probe raises the
    # pool's high-water mark by at least its point/result buffer
    pool, _, _ = _pool_marks()
    _reset_high_mark(pool)
    _, used_before, _ = _pool_marks()
    rc, _ = _probe(ctx, "cryo_probe_pressure", pts)
    assert rc == cabi.CRYO_OK
    _, used_high, _ = _pool_marks()
    assert used_high >= used_before + MAX_POINTS * 16
    # the first call may make the driver load the code module that holds the
    # fixed array (CUDA's lazy module loading): a one-time placement, made
    # here before the measured calls
    rc, _ = _probe(ctx, "cryo_probe_pressure_noalloc", pts[:10])
    assert rc == cabi.CRYO_OK
    for call in range(2):
        torch.cuda.synchronize(0)
        _reset_high_mark(pool)
        _, high0, reserved0 = _pool_marks()
        free0 = torch.cuda.mem_get_info(0)[0]
        rc, _ = _probe(ctx, "cryo_probe_pressure_noalloc", pts)
        assert rc == cabi.CRYO_OK
        _, high1, reserved1 = _pool_marks()
        free1 = torch.cuda.mem_get_info(0)[0]
        assert (high1, reserved1, free1) == (high0, reserved0, free0), call
