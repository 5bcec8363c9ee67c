"""The launch-shape autotuner: every candidate of the cluster size and the stack runs and is
timed on the device; the winner is one of them, and a run under it gives the same arrays as
the engine's default shapes to FP32 rounding."""
import numpy as np
import pytest

from ptyrs_b200 import GpuPtycho, Scan, sim
from ptyrs_b200.tune import autotune
from scenarios import far_field, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,k,nframe,side", [(128, 2, 24, 320), (256, 2, 10, 448)])
def test_autotune_picks_a_candidate_that_runs(n, k, nframe, side):
    s = far_field(n, k, nframe, side, masked=True, seed=n + k)
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    run = lambda h: h.ml(2, update_probe=True, zero_phase_ramp=False)
    best, table = autotune(scan, s["object"], s["probe"], run, stacks=(4, 16))
    assert best in [o for _, o in table]
    assert all(ms is not None and ms > 0 for ms, _ in table)
    with GpuPtycho(scan, s["object"], s["probe"], **best) as a, \
            GpuPtycho(scan, s["object"], s["probe"]) as b:
        run(a)
        run(b)
        assert rel_l2(a.object(), b.object()) < 1e-5
        assert rel_l2(a.probe(), b.probe()) < 1e-5


def test_batch_tuning_per_side():
    """One tuning per frame side, applied to every scan of that side."""
    from ptyrs_b200 import batch_run
    from ptyrs_b200.tune import autotune_batch, clusters_for
    scans = [dict(far_field(n, 1, 12, 3 * n, seed=n), n=n) for n in (64, 128, 64)]
    make = lambda s: (Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE,
                           sim.DETECTOR_PIXEL), s["object"], s["probe"])
    opts, chosen = autotune_batch(
        scans, run=lambda h: batch_run([h], 1, 1, rpie=dict(batch_size=4, obj_alpha=0.1,
                                                             probe_alpha=0.1, seed=7),
                                       lsqml=dict(batch_size=4, cost="poisson", seed=7)),
        stacks=(4, 8), make=make)
    assert sorted(chosen) == [64, 128]
    assert opts[0] == opts[2] == chosen[64][0]
    assert opts[1]["cluster"] in clusters_for(128) and opts[1]["stack_size"] in (4, 8)
