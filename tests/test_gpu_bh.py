"""pty-chi's BH on the CUDA path (`ptyb_bh`: the amplitude cost's gradient pass, the gathers,
the bilinear Hessian per frame and the conjugate or steepest direction) through the C ABI
against the float64 oracle (oracle/bh.py, pinned to the reference's golden BH runs): every
step's β, α, ⟨-g, D⟩ and H(D, D), the object, the probe and the LLK, over epochs with one batch
of every frame (conjugate directions) and with smaller batches (steepest descent)."""
import numpy as np
import pytest

from oracle.bh import Bh
from ptyrs_b200 import GpuPtycho, PtybError, Scan, sim
from scenarios import far_field, oracle_state, rel_l2

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-4
SHAPES = [(64, 2, 40, 192), (128, 3, 24, 320), (256, 2, 10, 448)]


def gpu_of(s):
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    return GpuPtycho(scan, s["object"], s["probe"])


@pytest.fixture(scope="module", params=SHAPES, ids=lambda p: f"n{p[0]}k{p[1]}")
def case(request):
    n, k, nframe, side = request.param
    s = far_field(n, k, nframe, side, masked=True, seed=n + k)
    s["object"] = s["truth"] * 0.9 * np.exp(0.1j)
    return s


@pytest.mark.parametrize("full", [True, False], ids=["cg", "mini"])
def test_bh_epochs(case, full):
    nframe = len(case["counts"])
    batch = nframe if full else max(2, nframe // 3)
    nepoch = 3
    cpu = oracle_state(case)
    run = Bh(batch, probe_rho=0.01, seed=7)
    obj, probe = cpu.object, cpu.probe
    for _ in range(nepoch):
        obj, probe, steps = run.epoch(cpu.addr, cpu.obs, cpu.optics, obj, probe)
    with gpu_of(case) as g:
        g.bh(nepoch, batch_size=batch, probe_rho=0.01, seed=7, calc_llk=1)
        got = g.bh_steps()
        assert [s["count"] for s in got] == [len(s["frames"]) for s in steps]
        for gs, cs in zip(got, steps):
            for key in ("alpha", "top", "bottom"):
                assert abs(gs[key] - cs[key]) <= RUN_TOL * abs(cs[key]), key
            if cs["beta"] == 0.0:
                assert gs["beta"] == 0.0
            else:
                assert abs(gs["beta"] - cs["beta"]) <= 10 * RUN_TOL * abs(cs["beta"])
        assert rel_l2(g.object(), obj) < RUN_TOL
        assert rel_l2(g.probe(), probe) < RUN_TOL
        hist = g.history()
        assert list(hist["algorithm"]) == ["bh"] * nepoch
        cpu.object, cpu.probe = obj, probe
        assert abs(hist["poisson"][-1] - cpu.llk().poisson) <= RUN_TOL * cpu.llk().poisson


def test_bh_is_deterministic(case):
    outs = []
    for _ in range(2):
        with gpu_of(case) as g:
            g.bh(2, batch_size=len(case["counts"]), seed=3)
            outs.append((g.object(), g.probe(), g.bh_steps()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]


@pytest.mark.parametrize("refine", [True, False], ids=["refined", "held"])
@pytest.mark.parametrize("full", [True, False], ids=["cg", "mini"])
def test_bh_epochs_with_offsets(case, full, refine):
    """Under the position model (Patch): every frame's probe moved by its offset, held or
    refined as BH variables (position_rho 2, the reference test's), against the oracle (pinned
    to the reference's bh_pos runs): steps, object, probe, offsets and the LLK."""
    nframe = len(case["counts"])
    batch = nframe if full else max(2, nframe // 3)
    nepoch = 2
    d0 = np.random.default_rng(5).uniform(-0.8, 0.8, (nframe, 2))
    cpu = oracle_state(case)
    run = Bh(batch, probe_rho=0.01, seed=7, position_rho=2.0, offsets=d0, refine=refine)
    obj, probe = cpu.object, cpu.probe
    for _ in range(nepoch):
        obj, probe, steps = run.epoch(cpu.addr, cpu.obs, cpu.optics, obj, probe)
    with gpu_of(case) as g:
        g.set_positions(d0, refine=refine)
        g.bh(nepoch, batch_size=batch, probe_rho=0.01, position_rho=2.0, seed=7, calc_llk=1)
        got = g.bh_steps()
        assert [s["count"] for s in got] == [len(s["frames"]) for s in steps]
        for gs, cs in zip(got, steps):
            for key in ("alpha", "top", "bottom"):
                assert abs(gs[key] - cs[key]) <= RUN_TOL * abs(cs[key]), key
            if cs["beta"] == 0.0:
                assert gs["beta"] == 0.0
            else:
                assert abs(gs["beta"] - cs["beta"]) <= 10 * RUN_TOL * abs(cs["beta"])
        assert rel_l2(g.object(), obj) < RUN_TOL
        assert rel_l2(g.probe(), probe) < RUN_TOL
        d = g.positions()
        if refine:
            moved = run.offsets - d0
            assert np.abs(moved).max() > 1e-6
            assert np.abs((d - d0) - moved).max() <= RUN_TOL * np.abs(moved).max()
        else:
            assert np.array_equal(d, d0)
        cpu.object, cpu.probe = obj, probe
        cpu.set_positions(run.offsets if refine else d0)
        want = cpu.llk().poisson
        assert abs(g.history()["poisson"][-1] - want) <= RUN_TOL * want


def test_bh_refusals(case):
    with gpu_of(case) as g:
        with pytest.raises(PtybError):
            g.bh(1, batch_size=0)
        g.set_positions(np.zeros((len(case["counts"]), 2)))
        g.bh(1, batch_size=4)
        g.set_positions(None)
        g.bh(1, batch_size=4)
        assert np.isfinite(g.object()).all()
