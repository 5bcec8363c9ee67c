"""pty-chi's OPR probe variation inside LSQML on the CUDA path (`ptyb_set_probe_variation`:
every frame's own probe c_f·P_0 + Σ_i w_fi·U_i, and each batch's step of the eigenmodes and the
refined weights) through the C ABI against the f64 oracle (`Lsqml(var=...)`, pinned to the
reference's golden OPR sets): two epochs, the object, the probe, the eigenmodes, the weights,
the main mode's weights and the LLK of every frame's own probe, to the reference's GPU-vs-CPU
1e-4; with the position model (held and refined offsets) and through a multislice object."""
import numpy as np
import pytest

from oracle.lsqml import Lsqml
from oracle.opr import ProbeVariation
from ptyrs_b200 import GpuPtycho, Scan, sim
from scenarios import far_field, oracle_state, rel_l2

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-4
SHAPES = [(64, 2, 40, 192), (128, 3, 24, 320)]


def gpu_of(s):
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    return GpuPtycho(scan, s["object"], s["probe"])


@pytest.fixture(scope="module", params=SHAPES, ids=lambda p: f"n{p[0]}k{p[1]}")
def case(request):
    n, k, nframe, side = request.param
    return far_field(n, k, nframe, side, masked=True, seed=n + k)


def start_variation(s, k, seed=3):
    """k smooth eigenmodes at the main mode's scale and small weights."""
    rng = np.random.default_rng(seed)
    p0 = s["probe"][0]
    scale = np.sqrt((np.abs(p0) ** 2).mean())
    u = []
    for i in range(k):
        g = sim.smooth_object(p0.shape[-1], seed + i)[0] - 1.0
        u.append(p0 * g * scale / np.sqrt((np.abs(p0 * g) ** 2).mean()))
    w = rng.uniform(-0.1, 0.1, (len(s["counts"]), k))
    return np.array(u), w


@pytest.mark.parametrize("cost,intensity,refine_w", [("poisson", True, True),
                                                      ("amplitude", False, True),
                                                      ("poisson", False, False)],
                         ids=["poisson_c", "amplitude", "held_w"])
def test_lsqml_with_opr(case, cost, intensity, refine_w):
    nframe = len(case["counts"])
    u, w = start_variation(case, 2)
    c = np.linspace(0.9, 1.1, nframe) if intensity else None
    var = ProbeVariation(u, w.ravel(), refine_weights=refine_w, intensity=c)
    cpu = oracle_state(case)
    run = Lsqml(8, cost, 7, var=var)
    obj, probe = cpu.object, cpu.probe
    for _ in range(2):
        obj, probe, _ = run.epoch(cpu.addr, cpu.obs, cpu.optics, obj, probe)
    ref = run.llk(cpu.addr, cpu.obs, cpu.optics, obj, probe)
    with gpu_of(case) as g:
        g.set_probe_variation(u, w, refine_weights=refine_w, intensity=c)
        g.lsqml(2, batch_size=8, cost=cost, seed=7, calc_llk=1)
        assert rel_l2(g.object(), obj) < RUN_TOL
        assert rel_l2(g.probe(), probe) < RUN_TOL
        gu, gw, gc = g.probe_variation()
        assert rel_l2(gu, var.eigenmodes) < RUN_TOL
        want_w = var.weights.reshape(nframe, 2)
        if refine_w:
            assert np.abs(gw - want_w).max() <= RUN_TOL * np.abs(want_w - w).max() + 1e-12
        else:
            assert np.array_equal(gw, w)
        if intensity:
            assert np.abs(gc - var.intensity).max() <= RUN_TOL * np.abs(var.intensity - c).max() + 1e-12
        got = g.history()["poisson"][-1]
        assert abs(got - ref.poisson) <= RUN_TOL * abs(ref.poisson)


@pytest.mark.parametrize("refine", [False, True], ids=["held", "refined"])
def test_lsqml_with_opr_and_positions(case, refine):
    """The probe variation under the position model (reference GPU engine/gpu/lsqml.rs:63-121,
    oracle pinned to the reference's `lsqml_pos_opr` set): every frame's own planes moved by
    its offset, the OPR step from the raw and the moved-back frame directions; two epochs, the
    object, probe, eigenmodes, weights, main-mode weights, offsets and the LLK."""
    nframe = len(case["counts"])
    u, w = start_variation(case, 2)
    c = np.linspace(0.9, 1.1, nframe)
    d0 = np.random.default_rng(7).uniform(-0.5, 0.5, (nframe, 2))
    var = ProbeVariation(u, w.ravel(), intensity=c)
    cpu = oracle_state(case)
    run = Lsqml(8, "poisson", 7, offsets=d0.copy(), refine=refine, var=var)
    obj, probe = cpu.object, cpu.probe
    for _ in range(2):
        obj, probe, _ = run.epoch(cpu.addr, cpu.obs, cpu.optics, obj, probe)
    ref = run.llk(cpu.addr, cpu.obs, cpu.optics, obj, probe)
    with gpu_of(case) as g:
        g.set_probe_variation(u, w, intensity=c)
        g.set_positions(d0, refine=refine)
        g.lsqml(2, batch_size=8, cost="poisson", seed=7, calc_llk=1)
        assert rel_l2(g.object(), obj) < RUN_TOL
        assert rel_l2(g.probe(), probe) < RUN_TOL
        gu, gw, gc = g.probe_variation()
        assert rel_l2(gu, var.eigenmodes) < RUN_TOL
        want_w = var.weights.reshape(nframe, 2)
        assert np.abs(gw - want_w).max() <= RUN_TOL * np.abs(want_w - w).max() + 1e-12
        assert np.abs(gc - var.intensity).max() <= RUN_TOL * np.abs(var.intensity - c).max() + 1e-12
        d = g.positions()
        if refine:
            assert rel_l2(d - d0, run.offsets - d0) < RUN_TOL
        else:
            assert np.array_equal(d, d0)
        got = g.history()["poisson"][-1]
        assert abs(got - ref.poisson) <= RUN_TOL * abs(ref.poisson)


def test_lsqml_with_opr_through_slices():
    """The probe variation on a multislice object: every frame's own planes enter slice 0, the
    OPR step on slice 0 (engine/lsqml.rs:571-643), against the oracle over two epochs."""
    from test_gpu_multislice import gpu_of as ms_gpu_of, multislice_scan, oracle_of
    s = multislice_scan(64, 2, 30, 192, (2e-6, 3e-6), seed=9)
    nframe = len(s["counts"])
    u, w = start_variation(dict(probe=s["probe"], counts=s["counts"]), 2)
    var = ProbeVariation(u, w.ravel())
    cpu = oracle_of(s)
    run = Lsqml(8, "poisson", 7, var=var)
    objs, probe = list(s["objects"]), cpu.probe
    for _ in range(2):
        objs, probe, _ = run.epoch(cpu.addr, cpu.obs, cpu.optics, objs, probe)
    with ms_gpu_of(s) as g:
        g.set_probe_variation(u, w)
        g.lsqml(2, batch_size=8, cost="poisson", seed=7)
        got = g.objects()
        for k in range(3):
            assert rel_l2(got[k] - 1.0, objs[k][0] - 1.0) < RUN_TOL, k
        assert rel_l2(g.probe(), probe) < RUN_TOL
        gu, gw, _ = g.probe_variation()
        assert rel_l2(gu, var.eigenmodes) < RUN_TOL
        want_w = var.weights.reshape(nframe, 2)
        assert np.abs(gw - want_w).max() <= RUN_TOL * np.abs(want_w - w).max() + 1e-12
