"""The CUDA path through the C ABI against the f64 oracle on the same seeded far-field scans,
as the reference holds its GPU engine to its CPU oracle (ptyrs/tests/engine_gpu.rs:160-165,
298-322: relative error < 1e-4 on the LLK records and the final object and probe). One epoch
of one batch is held to 1e-5 (FP32 against FP64 for one update); several epochs to 1e-4.
Frame sides 64, 128 and 256 run the cluster sizes 1, 2 and 8."""
import numpy as np
import pytest

from oracle.lsqml import Lsqml
from ptyrs_b200 import GpuPtycho, PtybError, Scan, sim
from scenarios import far_field, oracle_state, rel_l2

pytestmark = pytest.mark.gpu

ONE_STEP_TOL = 1e-5
RUN_TOL = 1e-4
# One LSQML batch under the Poisson cost on the 64² hard-edged apertures: the residual
# 1 − I/(Ĩ + 1e-6) and the far-field step's xi = 1 − I/(Ĩ + 1e-5) weigh the pixels at the
# aperture's far-field zeros, where Ĩ is the FP32 FFT's absolute rounding (~1e-7 of the field's
# largest value): measured there 3.6e-5 (a_far), 3.7e-5 (a_obj) and 1.8e-5 (probe) of the
# float64 step, against 1e-6 or less for the amplitude cost and the 128² and 256² probes.
POISSON_64_ONE_STEP_TOL = 1e-4
# ML's LLK records after its first Newton step: on the two-mode 64² scan a 1e-7 relative change
# of the start probe moves the float64 record after the first step by 3.3e-5 (an amplification
# of ~300), so the FP32 path's records hold to 3e-4 of the largest there.
ML_LLK_TOL = 3e-4

# (frame side, probe modes, frames, object side)
SHAPES = [(64, 1, 40, 192), (64, 2, 40, 192), (128, 3, 24, 320), (256, 2, 10, 448)]


def gpu_of(s, **kw):
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    return GpuPtycho(scan, s["object"], s["probe"], **kw)


@pytest.fixture(scope="module", params=SHAPES, ids=lambda p: f"n{p[0]}k{p[1]}")
def case(request):
    n, k, nframe, side = request.param
    return far_field(n, k, nframe, side, masked=True, seed=n + k)


def test_corners_and_start_llk(case):
    cpu = oracle_state(case)
    with gpu_of(case) as g:
        want = np.stack([cpu.addr.views["oy"], cpu.addr.views["ox"]], 1)[::cpu.addr.nmode]
        assert (g.corners() == want).all()
        got, ref = g.llk(), cpu.llk()
        for key in ("poisson", "gaussian", "euclidian", "nb_photons_calc"):
            assert abs(got[key] - getattr(ref, key)) <= ONE_STEP_TOL * abs(getattr(ref, key)), key


def test_rpie_one_batch(case):
    cpu = oracle_state(case)
    nframe = len(case["counts"])
    cpu.rpie(1, obj_alpha=0.1, probe_alpha=0.1, batch_size=nframe, seed=7)
    with gpu_of(case) as g:
        g.rpie(1, obj_alpha=0.1, probe_alpha=0.1, batch_size=nframe, seed=7)
        assert g.launches() > 0
        assert rel_l2(g.object() - case["object"], cpu.object - case["object"]) < ONE_STEP_TOL
        assert rel_l2(g.probe() - case["probe"], cpu.probe - case["probe"]) < ONE_STEP_TOL


@pytest.mark.parametrize("batch", [7, 13])
def test_rpie_epochs(case, batch):
    cpu = oracle_state(case)
    cpu.rpie(3, obj_alpha=0.1, probe_alpha=0.1, batch_size=batch, calc_llk=1, seed=7)
    with gpu_of(case) as g:
        g.rpie(3, obj_alpha=0.1, probe_alpha=0.1, batch_size=batch, calc_llk=1, seed=7)
        assert rel_l2(g.object(), cpu.object) < RUN_TOL
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL
        h = g.history()
        want = np.array([r["poisson"] for r in cpu.history])
        assert list(h["cycle"]) == [r["cycle"] for r in cpu.history]
        assert np.abs(h["poisson"] - want).max() <= RUN_TOL * np.abs(want).max()
        assert g.cycle() == 3


def test_rpie_single_frame_batches():
    """Batches of one frame (pty-chi's per-frame rPIE) on a scan whose f64 run moves by < 1e-5
    under a 1e-7 change of the start: the single-mode aperture scans amplify such a change to
    1e-2 in three epochs in f64 alone, so no FP32 run can be held to them."""
    s = far_field(64, 2, 40, 192, masked=True, seed=66)
    cpu = oracle_state(s)
    cpu.rpie(2, batch_size=1, seed=7)
    with gpu_of(s) as g:
        g.rpie(2, batch_size=1, seed=7)
        assert rel_l2(g.object(), cpu.object) < RUN_TOL
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL


def test_rpie_holds_an_array_without_its_step(case):
    cpu = oracle_state(case)
    cpu.rpie(1, obj_step=None, batch_size=7, seed=3)
    with gpu_of(case) as g:
        g.rpie(1, obj_step=None, batch_size=7, seed=3)
        assert np.array_equal(g.object(), case["object"].astype(np.complex64).astype(complex))
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL


def lsqml_cpu(case, nepoch, batch, cost):
    cpu = oracle_state(case)
    run = Lsqml(batch, cost, 7)
    obj, probe, steps = cpu.object, cpu.probe, None
    for _ in range(nepoch):
        obj, probe, steps = run.epoch(cpu.addr, cpu.obs, cpu.optics, obj, probe)
    return obj, probe, steps


@pytest.mark.parametrize("cost", ["poisson", "amplitude"])
def test_lsqml_one_batch(case, cost):
    nframe = len(case["counts"])
    obj, probe, steps = lsqml_cpu(case, 1, nframe, cost)
    with gpu_of(case) as g:
        g.lsqml(1, batch_size=nframe, cost=cost, seed=7)
        got = g.lsqml_steps()
        assert len(got) == 1 and got[0]["frames"] == steps[0]["frames"]
        tol = POISSON_64_ONE_STEP_TOL if cost == "poisson" and case["n"] == 64 else ONE_STEP_TOL
        for key in ("a_far", "a_obj", "a_probe"):
            a, b = np.array(got[0][key]), np.array(steps[0][key])
            assert np.abs(a - b).max() <= tol * np.abs(b).max(), key
        assert rel_l2(g.object() - case["object"], obj - case["object"]) < tol
        assert rel_l2(g.probe() - case["probe"], probe - case["probe"]) < tol


@pytest.mark.parametrize("cost", ["poisson", "amplitude"])
def test_lsqml_epochs(case, cost):
    """Three epochs of batches of 8: every step's a_far, a_obj and a_probe, the object and the
    probe to 1e-4 (the worst measured, a_far on the single 64² aperture under the Poisson cost,
    6e-5)."""
    nepoch = 3
    obj, probe, steps = lsqml_cpu(case, nepoch, 8, cost)
    with gpu_of(case) as g:
        g.lsqml(nepoch, batch_size=8, cost=cost, seed=7)
        got = g.lsqml_steps()
        assert [s["frames"] for s in got] == [s["frames"] for s in steps]
        for gs, cs in zip(got, steps):
            for key in ("a_far", "a_obj", "a_probe"):
                a, b = np.array(gs[key]), np.array(cs[key])
                assert np.abs(a - b).max() <= RUN_TOL * np.abs(b).max() + 1e-30, key
        assert rel_l2(g.object(), obj) < RUN_TOL
        assert rel_l2(g.probe(), probe) < RUN_TOL


def test_runs_are_deterministic(case):
    outs = []
    for _ in range(2):
        with gpu_of(case) as g:
            g.rpie(2, batch_size=6, seed=11)
            g.lsqml(2, batch_size=6, seed=5)
            outs.append((g.object(), g.probe()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_invalid_calls_leave_the_state():
    s = far_field(64, 1, 12, 160, seed=1)
    with gpu_of(s) as g:
        before = g.object()
        with pytest.raises(PtybError) as e:
            g.rpie(1, batch_size=0)
        assert e.value.status == "invalid"
        assert np.array_equal(g.object(), before)
        g.rpie(1, batch_size=4)  # still usable
    bad = dict(s, y=s["y"] * 100.0)
    with pytest.raises(PtybError) as e:
        gpu_of(bad)
    assert e.value.status == "invalid"
    with pytest.raises(PtybError):
        gpu_of(dict(s, object=np.ones((2, 160, 160), complex)))


@pytest.mark.parametrize("update_probe", [False, True])
@pytest.mark.parametrize("ramp", [False, True])
def test_ml_cycles(case, update_probe, ramp):
    """Poisson ML conjugate gradient (scale, gradients, Polak–Ribière, Newton step) over four
    cycles against the oracle's `Ptycho::ml`, with and without the probe and the final phase
    ramp removal."""
    cpu = oracle_state(case)
    cpu.ml(4, update_probe=update_probe, calc_llk=1, zero_phase_ramp=ramp)
    with gpu_of(case) as g:
        g.ml(4, update_probe=update_probe, calc_llk=1, zero_phase_ramp=ramp)
        assert rel_l2(g.object(), cpu.object) < RUN_TOL
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL
        h = g.history()
        want = np.array([r["poisson"] for r in cpu.history])
        assert list(h["algorithm"]) == ["ml"] * 4
        assert np.abs(h["poisson"] - want).max() <= ML_LLK_TOL * np.abs(want).max()


@pytest.mark.parametrize("refine", [False, True])
def test_lsqml_with_positions(case, refine):
    """LSQML with per-frame sub-pixel offsets under Patch sampling (each frame's probe moved by
    its offset, the probe directions moved back, and with `refine` pty-chi's position step)
    against the oracle, which is pinned to pty-chi's golden step: the step sizes, the arrays,
    the offset changes and the LLK of the moved-probe model. The single hard-edged aperture
    runs the amplitude cost: under the Poisson cost its step sizes are FP32-limited at the
    aperture's far-field zeros (see test_lsqml_epochs)."""
    nframe = len(case["counts"])
    d0 = np.random.default_rng(5).uniform(-0.6, 0.6, (nframe, 2))
    single = case["probe"].shape[0] == 1
    nepoch = 1 if single else 2
    cost = "amplitude" if single else "poisson"
    cpu = oracle_state(case)
    run = Lsqml(8, cost, 7, offsets=d0, refine=refine)
    obj, probe, steps = cpu.object, cpu.probe, None
    for _ in range(nepoch):
        obj, probe, steps = run.epoch(cpu.addr, cpu.obs, cpu.optics, obj, probe)
    with gpu_of(case) as g:
        g.set_positions(d0, refine=refine)
        g.lsqml(nepoch, batch_size=8, cost=cost, seed=7)
        got = g.lsqml_steps()
        assert [s["frames"] for s in got] == [s["frames"] for s in steps]
        for gs, cs in zip(got, steps):
            for key in ("a_far", "a_obj", "a_probe"):
                a, b = np.array(gs[key]), np.array(cs[key])
                assert np.abs(a - b).max() <= RUN_TOL * np.abs(b).max(), key
        assert rel_l2(g.object(), obj) < RUN_TOL
        assert rel_l2(g.probe(), probe) < RUN_TOL
        d = g.positions()
        if refine:
            moved = run.offsets - d0
            assert np.abs(moved).max() > 0
            assert np.abs((d - d0) - moved).max() <= RUN_TOL * 10 * np.abs(moved).max()
        else:
            assert np.array_equal(d, d0)
        cpu.object, cpu.probe = obj, probe
        want = run.llk(cpu.addr, cpu.obs, cpu.optics, obj, probe).poisson
        assert abs(g.llk()["poisson"] - want) <= RUN_TOL * abs(want)


@pytest.mark.parametrize("refine", [False, True])
def test_ml_with_positions(case, refine):
    """Poisson ML under per-frame sub-pixel offsets (Patch sampling: every view's probe moved by
    its frame's offset in the LLK, the gradients and the line search, the probe gradient moved
    back), with `refine` AP's position step from the magnitude projection of the estimate each
    cycle starts from, against the oracle's `Ptycho::ml`: the arrays, the LLK records and the
    offsets' changes. The start object is the perturbed truth: under a flat object the
    intensities do not depend on the offsets, so their step would be rounding. The single
    hard-edged aperture runs one cycle: its moved copies ring over the whole frame, and at
    the far-field zeros, where the Poisson gradient 2(1 − I/Ĩ) is led by Ĩ, FP32 rounding of
    the moves grows over the CG cycles."""
    nframe = len(case["counts"])
    ncycle = 1 if case["probe"].shape[0] == 1 else 4
    d0 = np.random.default_rng(6).uniform(-0.6, 0.6, (nframe, 2))
    start = dict(case, object=case["truth"] * 0.9 * np.exp(0.1j))
    cpu = oracle_state(start)
    cpu.set_positions(d0, refine=refine)
    cpu.ml(ncycle, update_probe=True, calc_llk=1, zero_phase_ramp=False)
    with gpu_of(start) as g:
        g.set_positions(d0, refine=refine)
        g.ml(ncycle, update_probe=True, calc_llk=1, zero_phase_ramp=False)
        assert rel_l2(g.object(), cpu.object) < RUN_TOL
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL
        h = g.history()
        want = np.array([r["poisson"] for r in cpu.history])
        assert np.abs(h["poisson"] - want).max() <= ML_LLK_TOL * np.abs(want).max()
        d = g.positions()
        if refine:
            moved = cpu.offsets - d0
            assert np.abs(moved).max() > 0
            assert np.abs((d - d0) - moved).max() <= RUN_TOL * 10 * np.abs(moved).max()
        else:
            assert np.array_equal(d, d0)


@pytest.mark.parametrize("refine", [False, True])
def test_rpie_with_positions(case, refine):
    """rPIE under per-frame sub-pixel offsets (every frame's probe moved by its offset, each
    frame's probe direction moved back, with `refine` pty-chi's position step from mode 0)
    against the oracle, which is pinned to pty-chi's golden run: the arrays and the offset
    changes after two epochs of batches of 13."""
    nframe = len(case["counts"])
    d0 = np.random.default_rng(7).uniform(-0.6, 0.6, (nframe, 2))
    start = dict(case, object=case["truth"] * 0.9 * np.exp(0.1j))
    cpu = oracle_state(start)
    cpu.set_positions(d0, refine=refine)
    cpu.rpie(2, obj_alpha=0.1, probe_alpha=0.1, batch_size=13, seed=7)
    with gpu_of(start) as g:
        g.set_positions(d0, refine=refine)
        g.rpie(2, obj_alpha=0.1, probe_alpha=0.1, batch_size=13, seed=7)
        assert rel_l2(g.object() - start["object"], cpu.object - start["object"]) < RUN_TOL
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL
        d = g.positions()
        if refine:
            moved = cpu.offsets - d0
            assert np.abs(moved).max() > 0
            assert np.abs((d - d0) - moved).max() <= RUN_TOL * 10 * np.abs(moved).max()
        else:
            assert np.array_equal(d, d0)


@pytest.mark.parametrize("offsets", [False, True], ids=["shared", "moved"])
def test_ml_opening_rescale_without_masked_pixels(offsets):
    """With no pixel masked, ML's opening rescale takes the model's photons in the exit plane
    (Parseval: Σ|P·O|² over each window, no transform) instead of from an LLK pass: against the
    oracle, whose rescale sums |Ψ|² in the detector plane, the arrays, the LLK records and (with
    moved probes) the offsets after four cycles."""
    s = far_field(128, 2, 24, 320, seed=9)
    assert (s["counts"] >= 0).all()
    nframe = len(s["counts"])
    d0 = np.random.default_rng(8).uniform(-0.6, 0.6, (nframe, 2))
    start = dict(s, object=s["truth"] * 0.9 * np.exp(0.1j))
    cpu = oracle_state(start)
    if offsets:
        cpu.set_positions(d0, refine=True)
    cpu.ml(4, update_probe=True, calc_llk=1, zero_phase_ramp=False)
    with gpu_of(start) as g:
        if offsets:
            g.set_positions(d0, refine=True)
        g.ml(4, update_probe=True, calc_llk=1, zero_phase_ramp=False)
        assert rel_l2(g.object(), cpu.object) < RUN_TOL
        assert rel_l2(g.probe(), cpu.probe) < RUN_TOL
        h = g.history()
        want = np.array([r["poisson"] for r in cpu.history])
        assert np.abs(h["poisson"] - want).max() <= ML_LLK_TOL * np.abs(want).max()
        if offsets:
            moved = cpu.offsets - d0
            assert np.abs(moved).max() > 0
            assert np.abs((g.positions() - d0) - moved).max() <= RUN_TOL * 10 * np.abs(moved).max()
