"""The forward-intensity entry point that allocates no device memory, for callers that cannot
call cudaMalloc once their handle exists (a fixed device-memory budget, a capped service): its
model intensities against the allocating `ptyb_forward_intensity`, through the C ABI, on two
calls in a row (the second on other frames, so the shared scratch's leftover contents must not
leak into it). It runs last in the suite and also alone in a fresh process."""
import numpy as np
import pytest

from ptyrs_b200 import GpuPtycho, Scan, sim
from scenarios import far_field

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the suite's one-update bound; the two paths run the same kernel


@pytest.mark.parametrize("n,k,nframe,side", [(64, 2, 30, 192), (256, 2, 40, 512)])
def test_noalloc_matches_the_allocating_entry_point(n, k, nframe, side):
    s = far_field(n, k, nframe, side, seed=3)
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    with GpuPtycho(scan, s["object"], s["probe"]) as g:
        first = np.arange(nframe, dtype=np.int32)
        second = np.arange(nframe - 1, -1, -3, dtype=np.int32)
        for frames in (first, second):
            want = g.forward_intensity(frames)
            got = g.forward_intensity_noalloc(frames)
            assert got.shape == want.shape
            assert np.abs(got - want).max() <= TOL * np.abs(want).max()
