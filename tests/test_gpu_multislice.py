"""pty-chi's multislice object on the CUDA path against the f64 oracle (oracle.lsqml with a list
of slices, itself pinned to the reference's golden multislice runs): the LLK through the slices,
LSQML epochs with every slice's step sizes, every slice and the probe, with and without the
position model, on the far field of three slices with two unequal angular-spectrum gaps. Frame sides 64, 128 and 256 run the
cluster sizes 1, 2 and 16."""
import numpy as np
import pytest

from oracle import ops
from oracle.base import fftshift2
from oracle.lsqml import Lsqml, SliceWaves
from oracle.ptycho import Ptycho
from ptyrs_b200 import GpuPtycho, PtybError, Scan, sim
from scenarios import rel_l2

pytestmark = pytest.mark.gpu

ONE_STEP_TOL = 1e-5
RUN_TOL = 1e-4

# (frame side, probe modes, frames, object side, gaps in metres)
SHAPES = [(64, 2, 30, 192, (2e-6, 3e-6)), (128, 2, 16, 320, (1e-6, 1.5e-6)),
          (256, 2, 8, 448, (0.4e-6, 0.6e-6))]


def slice_optics(n, gaps):
    optics = ops.Optics.far_field(sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL, [n, n])
    return optics.with_slices([ops.Wavefield([n, n], sim.WAVELENGTH, optics.pixel, d)
                               for d in gaps])


def multislice_scan(n, nmode, nframe, side, gaps, photons=1e5, seed=0):
    """Poisson counts of three smooth slices (the first with the strongest phase) under a
    Hermite probe of `nmode` modes, some pixels masked; the start is slices of ones and the
    probe scaled to the photons, perturbed in modulus and phase."""
    rng = np.random.default_rng(seed)
    truth = [sim.smooth_object(side, seed + 1),
             sim.smooth_object(side, seed + 2, np.pi / 5),
             sim.smooth_object(side, seed + 3, np.pi / 7)]
    probe = sim.hermite_probe(n, n / 4.0, [0.8, 0.15, 0.05][:nmode])
    probe = probe * np.sqrt(photons / (np.abs(probe) ** 2).sum())
    pos = sim.fermat_positions(nframe, n / 8.0) + rng.uniform(-0.5, 0.5, (nframe, 2))
    px = sim.object_pixel(n)
    y, x = pos[:, 0] * px, pos[:, 1] * px
    optics = slice_optics(n, gaps)
    cpu = Ptycho(np.zeros((nframe, n, n), np.float32), y, x, optics, truth[0], probe)
    run = Lsqml(nframe, "poisson", 0)
    uviews = run.unique_views(cpu.addr.views, nframe, nmode, cpu.addr.nmode)
    uprobe = run.frame_probes(range(nframe), probe, optics.slice_quad(0))
    waves = SliceWaves(optics, uviews, truth, uprobe[uviews["probe"].astype(np.int64)])
    far = optics.exit_forward(waves.psi)
    inten = (np.abs(far) ** 2).reshape(nframe, -1, n, n).sum(axis=1)
    counts = rng.poisson(fftshift2(inten)).astype(np.float32)
    counts[:, n // 2 - 1:n // 2 + 1, :3] = -1.0
    counts[rng.uniform(size=counts.shape) < 0.002] = -1.0
    start = [np.ones((1, side, side), np.complex128) for _ in truth]
    return dict(counts=counts, y=y, x=x, objects=start, probe=probe * 0.9 * np.exp(0.2j),
                gaps=gaps, n=n)


def oracle_of(s):
    optics = slice_optics(s["n"], s["gaps"])
    return Ptycho(s["counts"], s["y"], s["x"], optics, s["objects"][0], s["probe"])


def gpu_of(s, **kw):
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    return GpuPtycho(scan, np.concatenate(s["objects"]), s["probe"], gaps=s["gaps"], **kw)


@pytest.fixture(scope="module", params=SHAPES, ids=lambda p: f"n{p[0]}k{p[1]}")
def case(request):
    n, k, nframe, side, gaps = request.param
    return multislice_scan(n, k, nframe, side, gaps, seed=n + k)


def lsqml_cpu(case, nepoch, batch, cost):
    cpu = oracle_of(case)
    run = Lsqml(batch, cost, 7)
    objs, probe, steps = list(case["objects"]), cpu.probe, None
    for _ in range(nepoch):
        objs, probe, steps = run.epoch(cpu.addr, cpu.obs, cpu.optics, objs, probe)
    return cpu, run, objs, probe, steps


def test_start_llk_through_slices(case):
    cpu = oracle_of(case)
    ref = Lsqml(8, "poisson", 7).llk(cpu.addr, cpu.obs, cpu.optics, case["objects"], cpu.probe)
    with gpu_of(case) as g:
        assert g.nslice() == 3
        got = g.llk()
        for key in ("poisson", "gaussian", "euclidian", "nb_photons_calc"):
            assert abs(got[key] - getattr(ref, key)) <= ONE_STEP_TOL * abs(getattr(ref, key)), key


@pytest.mark.parametrize("cost", ["poisson", "amplitude"])
def test_lsqml_epochs_through_slices(case, cost):
    """Two epochs of batches of 8: every step's a_far, each slice's a_obj and a_probe, every
    slice, the probe and the LLK after them."""
    cpu, run, objs, probe, steps = lsqml_cpu(case, 2, 8, cost)
    with gpu_of(case) as g:
        g.lsqml(2, batch_size=8, cost=cost, seed=7)
        got = g.lsqml_steps()
        assert [s["frames"] for s in got] == [s["frames"] for s in steps]
        for gs, cs in zip(got, steps):
            for key in ("a_far", "a_probe"):
                a, b = np.array(gs[key]), np.array(cs[key])
                assert np.abs(a - b).max() <= RUN_TOL * np.abs(b).max() + 1e-30, key
            for k in range(3):
                a, b = np.array(gs["a_obj"][k]), np.array(cs["a_obj"][k])
                assert np.abs(a - b).max() <= RUN_TOL * np.abs(b).max() + 1e-30, ("a_obj", k)
        got_objs = g.objects()
        for k in range(3):
            assert rel_l2(got_objs[k] - 1.0, objs[k][0] - 1.0) < RUN_TOL, k
        assert np.array_equal(g.object(), got_objs[:1])
        assert rel_l2(g.probe(), probe) < RUN_TOL
        ref = run.llk(cpu.addr, cpu.obs, cpu.optics, objs, probe)
        assert abs(g.llk()["poisson"] - ref.poisson) <= RUN_TOL * abs(ref.poisson)


def test_multislice_runs_are_deterministic(case):
    outs = []
    for _ in range(2):
        with gpu_of(case) as g:
            g.lsqml(1, batch_size=8, seed=3)
            outs.append((g.objects(), g.probe()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_multislice_refuses_other_algorithms(case):
    with gpu_of(case) as g:
        with pytest.raises(PtybError):
            g.rpie(1, batch_size=8)
        with pytest.raises(PtybError):
            g.forward_intensity([0])
        g.set_positions(np.zeros((len(case["counts"]), 2)))
        with pytest.raises(PtybError):
            g.gradients(positions=False)  # not built through slices under the position model
        # the handle still runs LSQML after the refusals
        g.lsqml(1, batch_size=8)
        assert np.isfinite(g.objects()).all()


def test_set_object_replaces_slice_zero(case):
    with gpu_of(case) as g:
        side = case["objects"][0].shape[-1]
        new = np.full((1, side, side), 0.5 + 0.25j)
        g.set_object(new)
        objs = g.objects()
        assert np.array_equal(objs[0:1], new)
        assert np.array_equal(objs[1:], np.ones((2, side, side)))


def test_gradients_through_slices_match_oracle(case):
    """The adjoint through the slices (`ptyb_gradients` on a multislice handle): the Poisson
    sum, every slice's gradient and the probe's against the oracle's `multislice_grads`, whose
    gradients match central differences (test_oracle_multislice_grad.py); and the torch
    function on it."""
    import torch

    from oracle.lsqml import multislice_grads
    from ptyrs_b200.autograd import poisson_loss
    cpu = oracle_of(case)
    rng = np.random.default_rng(2)
    objs = [o * (1 + 0.05 * rng.normal(size=o.shape)) * np.exp(0.05j) for o in case["objects"]]
    loss, d_objs, d_probe = multislice_grads(cpu.addr, cpu.obs, cpu.optics, objs, cpu.probe)
    with gpu_of(case) as g:
        g.set_objects(np.concatenate(objs))
        got = g.gradients(positions=False)
        assert abs(got["loss"] - loss) <= ONE_STEP_TOL * abs(loss)
        for k in range(3):
            assert rel_l2(got["object"][k], d_objs[k][0]) < RUN_TOL, k
        assert rel_l2(got["probe"], d_probe) < RUN_TOL
        o = torch.tensor(np.concatenate(objs), requires_grad=True)
        p = torch.tensor(case["probe"], requires_grad=True)
        t = poisson_loss(o, p, None, g)
        t.backward()
        assert np.array_equal(o.grad.numpy(), got["object"])
        assert np.array_equal(p.grad.numpy(), got["probe"])


@pytest.mark.parametrize("refine", [False, True], ids=["held", "refined"])
def test_lsqml_epochs_through_slices_with_positions(case, refine):
    """Two epochs of batches of 8 under the position model (Patch): every frame's probe moved
    by its sub-pixel offset before slice 0, the probe directions moved back, and with
    refinement pty-chi's position step on the middle slice (oracle pinned to the reference's
    `lsqml_multislice_pos` set): steps, slices, probe, offsets and the LLK."""
    nframe = len(case["counts"])
    d0 = np.random.default_rng(5).uniform(-0.5, 0.5, (nframe, 2))
    cpu = oracle_of(case)
    run = Lsqml(8, "poisson", 7, offsets=d0.copy(), refine=refine)
    objs, probe, steps = list(case["objects"]), cpu.probe, None
    for _ in range(2):
        objs, probe, steps = run.epoch(cpu.addr, cpu.obs, cpu.optics, objs, probe)
    with gpu_of(case) as g:
        g.set_positions(d0, refine=refine)
        g.lsqml(2, batch_size=8, cost="poisson", seed=7)
        got = g.lsqml_steps()
        assert [s["frames"] for s in got] == [s["frames"] for s in steps]
        for gs, cs in zip(got, steps):
            a, b = np.array(gs["a_probe"]), np.array(cs["a_probe"])
            assert np.abs(a - b).max() <= RUN_TOL * np.abs(b).max() + 1e-30
            for k in range(3):
                a, b = np.array(gs["a_obj"][k]), np.array(cs["a_obj"][k])
                assert np.abs(a - b).max() <= RUN_TOL * np.abs(b).max() + 1e-30, ("a_obj", k)
        got_objs = g.objects()
        for k in range(3):
            assert rel_l2(got_objs[k] - 1.0, objs[k][0] - 1.0) < RUN_TOL, k
        assert rel_l2(g.probe(), probe) < RUN_TOL
        d = g.positions()
        if refine:
            assert rel_l2(d - d0, run.offsets - d0) < RUN_TOL
            assert np.abs(d - d0).max() > 0
        else:
            assert np.array_equal(d, d0)
        ref = run.llk(cpu.addr, cpu.obs, cpu.optics, objs, probe)
        assert abs(g.llk()["poisson"] - ref.poisson) <= RUN_TOL * abs(ref.poisson)


@pytest.mark.parametrize("probe_too", [True, False], ids=["object_probe", "object"])
def test_ml_through_slices(case, probe_too):
    """ML conjugate gradient through the slices (`ptyb_ml` on a multislice handle): the
    gradients through the slices, the Polak–Ribière direction over every slice and the probe
    and the Poisson line search on the second-order expansion through the slices, against the
    oracle's `multislice_ml` (its line-search terms checked by central differences) over three
    cycles: every slice, the probe and the LLK records."""
    from oracle.lsqml import multislice_ml
    cpu = oracle_of(case)
    objs, probe, recs = multislice_ml(cpu.addr, cpu.obs, cpu.optics, case["objects"], cpu.probe,
                                      3, update_probe=probe_too, calc_llk=1)
    with gpu_of(case) as g:
        g.ml(3, update_object=True, update_probe=probe_too, calc_llk=1, zero_phase_ramp=False)
        got = g.objects()
        for k in range(3):
            assert rel_l2(got[k] - 1.0, objs[k][0] - 1.0) < RUN_TOL, k
        assert rel_l2(g.probe(), probe) < RUN_TOL
        hist = g.history()
        want = [r.poisson for r in recs]
        assert np.abs(hist["poisson"] - want).max() <= RUN_TOL * max(want)
        with pytest.raises(PtybError):
            g.ml(1, zero_phase_ramp=True)


@pytest.mark.parametrize("full", [True, False], ids=["cg", "mini"])
def test_bh_through_slices(case, full):
    """pty-chi's BH through the slices (`ptyb_bh` on a multislice handle): the amplitude cost's
    gradients through the slices, β from H(u, v) by polarization of the quadratic form on the
    second-order expansion through the slices, α·D on every slice and the probe, against the
    oracle (pinned to the reference's bh_multislice runs) over two epochs with one batch of every
    frame (conjugate directions) and with smaller batches: every step, every slice, the probe."""
    from oracle.bh import Bh
    cpu = oracle_of(case)
    nframe = len(case["counts"])
    batch = nframe if full else max(2, nframe // 3)
    run = Bh(batch, probe_rho=0.01, seed=7)
    objs, probe = list(case["objects"]), cpu.probe
    for _ in range(2):
        objs, probe, steps = run.epoch(cpu.addr, cpu.obs, cpu.optics, objs, probe)
    with gpu_of(case) as g:
        g.bh(2, batch_size=batch, probe_rho=0.01, seed=7, calc_llk=1)
        got = g.bh_steps()
        assert [s["count"] for s in got] == [len(s["frames"]) for s in steps]
        for gs, cs in zip(got, steps):
            for key in ("alpha", "top", "bottom"):
                assert abs(gs[key] - cs[key]) <= RUN_TOL * abs(cs[key]), key
            if cs["beta"] == 0.0:
                assert gs["beta"] == 0.0
            else:
                assert abs(gs["beta"] - cs["beta"]) <= 10 * RUN_TOL * abs(cs["beta"])
        got_objs = g.objects()
        for k in range(3):
            assert rel_l2(got_objs[k] - 1.0, objs[k][0] - 1.0) < RUN_TOL, k
        assert rel_l2(g.probe(), probe) < RUN_TOL
        assert list(g.history()["algorithm"]) == ["bh"] * 2
        g.set_positions(np.zeros((nframe, 2)))
        with pytest.raises(PtybError):
            g.bh(1, batch_size=batch)
