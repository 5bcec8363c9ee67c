"""Frame sides 96 and 192 (the line FFT's 24-point first stage: 8-point DFTs and radix-3
butterflies) against the f64 oracle, through every kernel family: the start LLK, rPIE and LSQML
epochs, ML cycles, DM, the position model under rPIE and ML, and LSQML through slices; to the
same bounds as the power-of-two sides (the reference's GPU-vs-CPU 1e-4, one step 1e-5)."""
import numpy as np
import pytest

from oracle import ops
from oracle.lsqml import Lsqml
from oracle.ptycho import Ptycho
from ptyrs_b200 import GpuPtycho, Scan, sim
from scenarios import far_field, oracle_state, rel_l2

pytestmark = pytest.mark.gpu

ONE_STEP_TOL = 1e-5
RUN_TOL = 1e-4
ML_LLK_TOL = 3e-4

SHAPES = [(96, 2, 24, 288), (192, 2, 10, 448)]


def gpu_of(s, **kw):
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    return GpuPtycho(scan, s["object"], s["probe"], **kw)


@pytest.fixture(scope="module", params=SHAPES, ids=lambda p: f"n{p[0]}k{p[1]}")
def case(request):
    n, k, nframe, side = request.param
    return far_field(n, k, nframe, side, masked=True, seed=n + k)


def test_start_llk(case):
    cpu = oracle_state(case)
    with gpu_of(case) as g:
        got, ref = g.llk(), cpu.llk()
        for key in ("poisson", "gaussian", "euclidian", "nb_photons_calc"):
            assert abs(got[key] - getattr(ref, key)) <= ONE_STEP_TOL * abs(getattr(ref, key))


def test_forward_intensity_matches_the_oracle(case):
    cpu = oracle_state(case)
    far = cpu.optics.exit_forward(cpu.calc_psi())
    want = ops.icalc_of(far, cpu.addr.nmode)   # zero frequency at [0, 0], as the counts
    with gpu_of(case) as g:
        got = g.forward_intensity()
    assert rel_l2(got, want) < ONE_STEP_TOL


def test_rpie_and_lsqml_epochs(case):
    cpu = oracle_state(case)
    cpu.rpie(2, batch_size=7, calc_llk=1, seed=7)
    run = Lsqml(8, "poisson", 7)
    for _ in range(2):
        cpu.object, cpu.probe, _ = run.epoch(cpu.addr, cpu.obs, cpu.optics, cpu.object,
                                             cpu.probe)
    with gpu_of(case) as g:
        g.rpie(2, batch_size=7, calc_llk=1, seed=7)
        g.lsqml(2, batch_size=8, cost="poisson", seed=7)
        assert rel_l2(g.object(), cpu.object) < RUN_TOL
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL


def test_ml_and_dm_cycles(case):
    cpu = oracle_state(case)
    cpu.ml(3, update_probe=True, calc_llk=1, zero_phase_ramp=True)
    cpu.dm(3, calc_llk=1)
    with gpu_of(case) as g:
        g.ml(3, update_probe=True, calc_llk=1, zero_phase_ramp=True)
        g.dm(3, calc_llk=1)
        assert rel_l2(g.object(), cpu.object) < RUN_TOL
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL
        want = np.array([r["poisson"] for r in cpu.history])
        assert np.abs(g.history()["poisson"] - want).max() <= ML_LLK_TOL * np.abs(want).max()


@pytest.mark.parametrize("algorithm", ["rpie", "ml"])
def test_refined_positions(case, algorithm):
    nframe = len(case["counts"])
    d0 = np.random.default_rng(6).uniform(-0.6, 0.6, (nframe, 2))
    start = dict(case, object=case["truth"] * 0.9 * np.exp(0.1j))
    cpu = oracle_state(start)
    cpu.set_positions(d0, refine=True)
    with gpu_of(start) as g:
        g.set_positions(d0, refine=True)
        if algorithm == "rpie":
            cpu.rpie(2, batch_size=5, seed=3)
            g.rpie(2, batch_size=5, seed=3)
        else:
            cpu.ml(2, update_probe=True, zero_phase_ramp=False)
            g.ml(2, update_probe=True, zero_phase_ramp=False)
        assert rel_l2(g.object(), cpu.object) < RUN_TOL
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL
        assert rel_l2(g.positions() - d0, cpu.offsets - d0) < RUN_TOL


def test_lsqml_through_slices(case):
    n = case["n"]
    gaps = (1e-6,)
    optics = ops.Optics.far_field(sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL, [n, n])
    optics = optics.with_slices([ops.Wavefield([n, n], sim.WAVELENGTH, optics.pixel, gaps[0])])
    objs = [case["object"], case["object"] * np.exp(0.05j)]
    cpu = Ptycho(case["counts"], case["y"], case["x"], optics, objs[0], case["probe"])
    run = Lsqml(8, "poisson", 7)
    o, p, _ = run.epoch(cpu.addr, cpu.obs, optics, list(objs), cpu.probe)
    with gpu_of(dict(case, object=np.concatenate(objs)), gaps=gaps) as g:
        g.lsqml(1, batch_size=8, cost="poisson", seed=7)
        got = g.objects()
        for k in range(2):
            assert rel_l2(got[k] - objs[k][0], o[k][0] - objs[k][0]) < RUN_TOL
        assert rel_l2(g.probe(), p) < RUN_TOL
