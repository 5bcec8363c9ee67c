"""Independent scans at once (`ptyb_batch_run`): three scans of different frame sides and probe
modes, each handle on its own stream from its own host thread, give bit for bit the arrays and
LLK records that the same rPIE-then-LSQML sequence gives each scan alone, with the batch's
device time; a failing handle is named and leaves the others' results; a repeated handle is
refused."""
import numpy as np
import pytest

from ptyrs_b200 import GpuPtycho, PtybError, Scan, batch_run, sim
from scenarios import far_field

pytestmark = pytest.mark.gpu

SHAPES = [(64, 1, 40, 192), (128, 2, 24, 320), (256, 2, 10, 448)]
RPIE = dict(batch_size=8, obj_alpha=0.1, probe_alpha=0.1, seed=5)
LSQML = dict(batch_size=8, cost="poisson", seed=9)


def gpu_of(s, **kw):
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    return GpuPtycho(scan, s["object"], s["probe"], **kw)


@pytest.fixture(scope="module")
def cases():
    return [far_field(n, k, nf, side, masked=True, seed=n + k) for n, k, nf, side in SHAPES]


def alone(s):
    with gpu_of(s) as g:
        g.rpie(2, calc_llk=1, **RPIE)
        g.lsqml(2, calc_llk=1, **LSQML)
        return g.object(), g.probe(), g.history()["poisson"]


def test_batch_matches_each_scan_alone(cases):
    want = [alone(s) for s in cases]
    handles = [gpu_of(s) for s in cases]
    try:
        ms = batch_run(handles, rpie_epochs=2, lsqml_epochs=2, calc_llk=1, rpie=RPIE, lsqml=LSQML)
        assert ms > 0.0
        for g, (o, p, h) in zip(handles, want):
            assert np.array_equal(g.object(), o)
            assert np.array_equal(g.probe(), p)
            assert np.array_equal(g.history()["poisson"], h)
            assert g.cycle() == 4
    finally:
        for g in handles:
            g.close()


def test_a_failing_handle_is_named_and_the_others_run(cases):
    s = cases[1]
    ms_scan = dict(s, object=np.concatenate([s["object"], s["object"]]))
    want = alone(cases[0])
    good = gpu_of(cases[0])
    bad = gpu_of(ms_scan, gaps=[1e-6])   # rPIE refuses a multislice handle
    try:
        with pytest.raises(PtybError, match="handle 1"):
            batch_run([good, bad], rpie_epochs=2, lsqml_epochs=2, calc_llk=1, rpie=RPIE,
                      lsqml=LSQML)
        assert np.array_equal(good.object(), want[0])
        with pytest.raises(PtybError):
            batch_run([good, good], rpie_epochs=1, lsqml_epochs=0)
    finally:
        good.close()
        bad.close()
