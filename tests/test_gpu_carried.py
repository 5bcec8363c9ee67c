"""PyNX's AP, DM and RAAR on the CUDA path (the frame kernel's carry mode: the mix of the
estimate's exit waves with the carried waves, the magnitude projection and the carried update in
one pass; the blends of the object and probe from every frame's carried waves) through the C ABI
against the f64 oracle's `Ptycho.ap / dm / raar`, itself pinned to the reference's PyNX runs
(engine_reconstruct.rs:186-220, engine_pynx_near.rs:98-205): the LLK records, the object and the
probe to 1e-4 of their norms (the reference's GPU-against-CPU bound, engine_gpu.rs:160-165)."""
import numpy as np
import pytest

from ptyrs_b200 import GpuPtycho, PtybError, Scan, sim
from scenarios import far_field, oracle_state, rel_l2

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-4

# (frame side, probe modes, frames, object side)
SHAPES = [(64, 1, 40, 192), (64, 2, 40, 192), (128, 3, 24, 320), (256, 2, 10, 448)]


def gpu_of(s, **kw):
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    return GpuPtycho(scan, s["object"], s["probe"], **kw)


@pytest.fixture(scope="module", params=SHAPES, ids=lambda p: f"n{p[0]}k{p[1]}")
def case(request):
    n, k, nframe, side = request.param
    return far_field(n, k, nframe, side, masked=True, seed=n + k)


def assert_matches(g, cpu, algorithm):
    assert rel_l2(g.object(), cpu.object) < RUN_TOL
    assert rel_l2(g.probe(), cpu.probe) < RUN_TOL
    h = g.history()
    assert list(h["cycle"]) == [r["cycle"] for r in cpu.history]
    assert h["algorithm"] == [algorithm] * len(cpu.history)
    for key in ("poisson", "gaussian", "euclidian", "nb_photons_calc"):
        want = np.array([r[key] for r in cpu.history])
        assert np.abs(h[key] - want).max() <= RUN_TOL * np.abs(want).max(), key


@pytest.mark.parametrize("probe_inertia", [None, 0.001], ids=["object", "object_probe"])
def test_ap_cycles(case, probe_inertia):
    """Four AP cycles recording each: the LLK of the field each projection reads, both blends
    from the old arrays."""
    cpu = oracle_state(case)
    cpu.ap(4, probe_inertia=probe_inertia, calc_llk=1, zero_phase_ramp=False)
    with gpu_of(case) as g:
        g.ap(4, probe_inertia=probe_inertia, calc_llk=1, zero_phase_ramp=False)
        assert_matches(g, cpu, "ap")
        assert g.cycle() == 4


@pytest.mark.parametrize("algorithm", ["dm", "raar"])
def test_dm_raar_cycles(case, algorithm):
    """Five cycles at PyNX's defaults, recording every second one (each record followed by the
    balance of Σ|O| and Σ|P|), then the phase ramp's removal."""
    cpu = oracle_state(case)
    getattr(cpu, algorithm)(5, calc_llk=2)
    with gpu_of(case) as g:
        getattr(g, algorithm)(5, calc_llk=2)
        assert_matches(g, cpu, algorithm)


@pytest.mark.parametrize("algorithm", ["dm", "raar"])
def test_dm_raar_options(case, algorithm):
    """A non-default mix, two object-then-probe updates per cycle, the object held fixed in a
    second call whose cycle 0 restarts from the estimate's exit waves."""
    mix = dict(alpha=0.1) if algorithm == "dm" else dict(beta=0.75)
    cpu = oracle_state(case)
    getattr(cpu, algorithm)(3, loop_obj_probe=2, calc_llk=1, zero_phase_ramp=False, **mix)
    getattr(cpu, algorithm)(2, obj_inertia=None, probe_inertia=0.01, calc_llk=1,
                            zero_phase_ramp=False, **mix)
    with gpu_of(case) as g:
        getattr(g, algorithm)(3, loop_obj_probe=2, calc_llk=1, zero_phase_ramp=False, **mix)
        getattr(g, algorithm)(2, obj_inertia=None, probe_inertia=0.01, calc_llk=1,
                              zero_phase_ramp=False, **mix)
        assert_matches(g, cpu, algorithm)


def test_carried_runs_are_deterministic(case):
    outs = []
    for _ in range(2):
        with gpu_of(case) as g:
            g.dm(2, calc_llk=1)
            g.ap(1, probe_inertia=0.001)
            g.raar(2)
            outs.append((g.object(), g.probe(), g.history()["poisson"]))
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)


def test_carried_refusals(case):
    """Negative counts are refused with the state unchanged."""
    with gpu_of(case) as g:
        before = g.object()
        with pytest.raises(PtybError):
            g.dm(-1)
        with pytest.raises(PtybError):
            g.raar(1, loop_obj_probe=-1)
        with pytest.raises(PtybError):
            g.ap(-2)
        assert np.array_equal(g.object(), before)


@pytest.mark.parametrize("algorithm", ["ap", "dm", "raar"])
@pytest.mark.parametrize("refine", [False, True], ids=["held", "refined"])
def test_carried_with_positions(case, algorithm, refine):
    """Under per-frame sub-pixel offsets (Patch sampling: every frame's probe moved by its
    offset), held or refined: the carried waves of the moved model, the object blend under the
    moved probes, the probe's line-searched step through the move's adjoint and, refining, the
    position step from the carried waves' sums, against the oracle: the arrays, the LLK records
    and the offsets' changes. The start object is the perturbed truth (under a flat object the
    intensities do not depend on the offsets); DM also runs two updates per cycle. The single
    hard-edged aperture runs one cycle (its moved copies ring over the whole frame)."""
    nframe = len(case["counts"])
    ncycle = 1 if case["probe"].shape[0] == 1 else 3
    d0 = np.random.default_rng(6).uniform(-0.6, 0.6, (nframe, 2))
    start = dict(case, object=case["truth"] * 0.9 * np.exp(0.1j))
    kw = dict(calc_llk=1, zero_phase_ramp=False)
    kw.update(dict(probe_inertia=0.001) if algorithm == "ap" else
              dict(loop_obj_probe=2) if algorithm == "dm" else {})
    cpu = oracle_state(start)
    cpu.set_positions(d0, refine=refine)
    getattr(cpu, algorithm)(ncycle, **kw)
    with gpu_of(start) as g:
        g.set_positions(d0, refine=refine)
        getattr(g, algorithm)(ncycle, **kw)
        assert_matches(g, cpu, algorithm)
        d = g.positions()
        if refine:
            assert rel_l2(d - d0, cpu.offsets - d0) < RUN_TOL
        else:
            assert np.array_equal(d, d0)
