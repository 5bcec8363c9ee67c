"""The forward-intensity entry point that allocates no device memory, for callers that cannot
call cudaMalloc once their handle exists (a fixed device-memory budget, a capped service): on a
fresh handle it runs before anything else has made the handle's scratch, its calls leave the
device's memory pool and the device's free memory unchanged, and its model intensities match
the allocating `ptyb_forward_intensity` through the C ABI on two calls in a row (the second on
other frames, so the shared scratch's leftover contents must not leak into it). It runs last in
the suite and also alone in a fresh process."""
import numpy as np
import pytest

from ptyrs_b200 import GpuPtycho, Scan, sim
from scenarios import far_field

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the suite's one-update bound; the two paths run the same kernel


def _driver():
    from cuda.bindings import driver as cu
    (err,) = cu.cuInit(0)
    assert err == cu.CUresult.CUDA_SUCCESS
    return cu


def _pool_used(cu, device=0):
    """Bytes in use from the device's default stream-ordered pool (the library's allocator)."""
    err, dev = cu.cuDeviceGet(device)
    assert err == cu.CUresult.CUDA_SUCCESS
    err, pool = cu.cuDeviceGetDefaultMemPool(dev)
    assert err == cu.CUresult.CUDA_SUCCESS
    err, used = cu.cuMemPoolGetAttribute(
        pool, cu.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
    assert err == cu.CUresult.CUDA_SUCCESS
    return int(used)


def _device_free(cu):
    err, free, _ = cu.cuMemGetInfo()
    assert err == cu.CUresult.CUDA_SUCCESS
    return int(free)


@pytest.mark.parametrize("n,k,nframe,side", [(64, 2, 30, 192), (256, 2, 40, 512)])
def test_noalloc_matches_the_allocating_entry_point(n, k, nframe, side):
    cu = _driver()
    s = far_field(n, k, nframe, side, seed=3)
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    first = np.arange(nframe, dtype=np.int32)
    second = np.arange(nframe - 1, -1, -3, dtype=np.int32)
    with GpuPtycho(scan, s["object"], s["probe"]) as g:
        # a fresh handle: the no-alloc calls come first, before any call has made its scratch
        used0 = _pool_used(cu)
        got = [g.forward_intensity_noalloc(first), g.forward_intensity_noalloc(second)]
        free0 = _device_free(cu)
        again = g.forward_intensity_noalloc(first)
        assert _device_free(cu) == free0
        assert _pool_used(cu) == used0
        for frames, out in ((first, got[0]), (second, got[1]), (first, again)):
            want = g.forward_intensity(frames)
            assert out.shape == want.shape
            assert np.abs(out - want).max() <= TOL * np.abs(want).max()
