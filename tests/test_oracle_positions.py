"""The oracle's ML position model (Patch sampling, engine/features.rs `Shifted`) checked for
internal consistency: with zero offsets it is the unshifted model; its back-projections are
the adjoints of its forward map; its gradients and position derivatives match central finite
differences of the Poisson LLK and of the exit waves; the ML loop with refined offsets moves
them toward the offsets the data were made with (slowly: AP's step from the magnitude
projection moves a frame by a few thousandths of a pixel per cycle here). The probe update of
AP, DM and RAAR under the move holds the reference's own checks (engine/ptycho.rs:1495-1596):
with zero offsets it is the blend, the overlap error never rises, the solution is a fixed
point; and AP, DM and RAAR refining positions move them toward the drawn ones."""
import numpy as np
import pytest

from oracle import ops
from oracle.ptycho import Ptycho, Shifted
from ptyrs_b200 import sim


def small_scan(offsets=None, seed=3, n=32, side=96, nframe=14, nmode=2, photons=1e5):
    """Counts from `offsets` (the true sub-pixel positions on top of the corners) and the
    oracle state at the nominal positions."""
    rng = np.random.default_rng(seed)
    truth = sim.smooth_object(side, seed + 1)
    probe = sim.hermite_probe(n, n / 4.0, [0.8, 0.2][:nmode])
    probe = probe * np.sqrt(photons / (np.abs(probe) ** 2).sum())
    pos = sim.fermat_positions(nframe, n / 8.0) + rng.uniform(-0.5, 0.5, (nframe, 2))
    px = sim.object_pixel(n)
    optics = ops.Optics.far_field(sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL, [n, n])
    y, x = pos[:, 0] * px, pos[:, 1] * px
    zeros = np.zeros((nframe, n, n), np.float32)
    gen = Ptycho(zeros, y, x, optics, truth, probe)
    if offsets is not None:
        gen.set_positions(offsets)
    far = optics.exit_forward(gen.calc_psi())
    inten = (np.abs(far) ** 2).reshape(nframe, nmode, n, n).sum(axis=1)
    counts = rng.poisson(np.fft.fftshift(inten, axes=(-2, -1))).astype(np.float32)
    return Ptycho(counts, y, x, optics, truth * 0.95, probe * 0.9 * np.exp(0.2j)), truth


def test_zero_offsets_are_the_unshifted_model():
    p, _ = small_scan()
    views, q = p.addr.views, p.optics.quad
    s = Shifted(views, p.probe, q, np.zeros((p.addr.nframe, 2)))
    psi = ops.obj_probe_to_psi(views, p.object, p.probe, q)
    assert np.abs(s.to_psi(p.object) - psi).max() < 1e-12 * np.abs(psi).max()
    g = p.grad_psi()
    a = ops.accumulate_obj(views, p.object.shape, p.probe, q, g)[0]
    b = s.accumulate_obj(p.object.shape, g)[0]
    assert np.abs(a - b).max() < 1e-12 * np.abs(a).max()
    a = ops.accumulate_probe(views, p.object, p.probe.shape, q, g)[0]
    b = s.accumulate_probe(p.object, p.probe.shape, g)[0]
    assert np.abs(a - b).max() < 1e-12 * np.abs(a).max()


def test_back_projections_are_adjoints():
    p, _ = small_scan()
    rng = np.random.default_rng(0)
    d = rng.normal(0, 0.4, (p.addr.nframe, 2))
    s = Shifted(p.addr.views, p.probe, p.optics.quad, d)
    psi = rng.normal(size=(len(p.addr.views),) + p.probe.shape[-2:]) * (1 + 1j)
    # <psi, A dO> = <A^H psi, dO> for the object, and the same for the probe
    d_obj = rng.normal(size=p.object.shape) + 1j * rng.normal(size=p.object.shape)
    lhs = np.vdot(psi, s.to_psi(d_obj))
    rhs = np.vdot(s.accumulate_obj(p.object.shape, psi)[0], d_obj)
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)
    d_probe = rng.normal(size=p.probe.shape) + 1j * rng.normal(size=p.probe.shape)
    sd = Shifted(p.addr.views, d_probe, p.optics.quad, d)
    lhs = np.vdot(psi, sd.to_psi(p.object))
    rhs = np.vdot(s.accumulate_probe(p.object, p.probe.shape, psi)[0], d_probe)
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)


def poisson_sum(p):
    """The Poisson LLK sum (not normalised) of the oracle's current estimate."""
    psi = p.optics.exit_forward(p.calc_psi())
    return ops.llk(p.obs, slice(0, p.addr.nframe), p.addr.nmode, psi).poisson


def test_gradients_under_offsets_match_central_differences():
    """`grads` is `2·∂L/∂X*` = ∂L/∂Re X + i·∂L/∂Im X (engine/ptycho.rs:492-515)."""
    p, _ = small_scan()
    rng = np.random.default_rng(1)
    p.set_positions(rng.normal(0, 0.4, (p.addr.nframe, 2)))
    go, gp = p.grads()
    h = 1e-6
    for arr, g, picks in ((p.object, go, [(0, 40, 40), (0, 50, 61)]),
                          (p.probe, gp, [(0, 16, 16), (1, 12, 19)])):
        for idx in picks:
            for unit in (1.0, 1j):
                base = arr[idx]
                arr[idx] = base + h * unit
                up = poisson_sum(p)
                arr[idx] = base - h * unit
                down = poisson_sum(p)
                arr[idx] = base
                fd = (up - down) / (2 * h)
                an = g[idx].real if unit == 1.0 else g[idx].imag
                assert abs(fd - an) < 1e-5 * max(abs(an), 1e-3 * np.abs(g).max()), (idx, unit)


def test_position_derivatives_match_central_differences():
    p, _ = small_scan()
    rng = np.random.default_rng(2)
    d = rng.normal(0, 0.4, (p.addr.nframe, 2))
    s = Shifted(p.addr.views, p.probe, p.optics.quad, d)
    h = 1e-5
    for axis in range(2):
        dpsi = s.derivatives(p.object, axis)
        dp, dm = d.copy(), d.copy()
        dp[:, axis] += h
        dm[:, axis] -= h
        fd = (Shifted(p.addr.views, p.probe, p.optics.quad, dp).to_psi(p.object)
              - Shifted(p.addr.views, p.probe, p.optics.quad, dm).to_psi(p.object)) / (2 * h)
        assert np.abs(fd - dpsi).max() < 1e-6 * np.abs(dpsi).max()


def test_position_step_centres_and_clips():
    d = np.zeros((3, 2))
    # axis 0: dens 1, 1, 3 (max 3); axis 1: dens 1, 0, 1 (max 1)
    sums = np.array([[[1.0, -2.0], [1.0, 1.0]],
                     [[0.0, 0.5], [1.0, 0.0]],
                     [[100.0, 0.0], [3.0, 1.0]]])
    ops.position_step(d, sums)
    step = np.array([[0.3 * 1.0 / 4.0, -0.1], [0.0, 0.1], [0.1, 0.0]])
    want = step - step.mean(axis=0)
    assert np.allclose(d, want, rtol=0, atol=1e-15)


@pytest.mark.parametrize("update_probe", [False, True])
def test_ml_with_refined_positions_lowers_llk_and_recovers_offsets(update_probe):
    rng = np.random.default_rng(5)
    true = rng.normal(0, 0.35, (14, 2))
    true -= true.mean(axis=0)
    p, truth = small_scan(true)
    p.object = truth.copy()
    p.set_positions(np.zeros((p.addr.nframe, 2)), refine=True)
    before = np.abs(p.offsets - true).mean()
    l0 = p.llk().poisson
    p.ml(12, update_probe=update_probe, zero_phase_ramp=False, calc_llk=1)
    assert p.llk().poisson < l0
    assert np.abs(p.offsets - true).mean() < before
    moved = p.offsets.ravel()
    assert np.dot(moved, true.ravel()) > 0.8 * np.linalg.norm(moved) * np.linalg.norm(true)


# The probe update of AP, DM and RAAR under the move (engine/features.rs:653-725), checked as the
# reference checks it (engine/ptycho.rs:1495-1596): five frames of a 3-pixel Fermat spiral, 16²
# frames, two probe modes, an object of random phase whose modulus is `modulus(u)` of a uniform
# u, the exit waves those of a truth probe, the probe started 30 % away from it.

def overlap_state(modulus=None, offsets=None, seed=11):
    n, nframe = 16, 5
    rng = np.random.default_rng(seed)
    pos = sim.fermat_positions(nframe, 3.0)
    side = 40
    obj = sim.smooth_object(side, seed)
    if modulus is not None:
        u = rng.uniform(size=(1, side, side))
        obj = modulus(u) * np.exp(2j * np.pi * rng.uniform(size=(1, side, side)))
    truth = sim.hermite_probe(n, n / 4.0, [0.7, 0.3])
    px = sim.object_pixel(n)
    optics = ops.Optics.far_field(sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL, [n, n])
    p = Ptycho(np.zeros((nframe, n, n), np.float32), pos[:, 0] * px, pos[:, 1] * px, optics,
               obj, truth)
    if offsets is not None:
        p.set_positions(np.array([offsets(f) for f in range(nframe)], np.float64))
    psi = p.calc_psi()
    p.probe = truth * (1.0 + 0.3 * rng.normal(size=truth.shape)) * np.exp(0.3j)
    return p, psi, truth


def fractional(f):
    return [np.sin(1.3 * f + 0.2), -np.cos(0.7 * f)]


def whole(f):
    return [(f % 5) - 2.0, ((2 * f + 1) % 3) - 1.0]


def probe_update(p, psi, inertia):
    s = p.shifted()
    if s is None:
        views, q = p.addr.views, p.optics.quad
        num, norm = ops.accumulate_probe(views, p.object, p.probe.shape, q, psi)
        from oracle.ptycho import _blend
        return _blend(p.probe, num, norm, inertia)
    return s.psi_to_obj_probe(p.object, p.probe, psi, None, inertia)[1]


def overlap_error(p, psi):
    return float((np.abs(p.calc_psi() - psi) ** 2).sum())


@pytest.mark.parametrize("inertia", [0.0, 0.001])
def test_probe_update_under_zero_offsets_is_the_blend(inertia):
    plain, psi, _ = overlap_state()
    still, psi2, _ = overlap_state(offsets=lambda f: [0.0, 0.0])
    a, b = probe_update(still, psi2, inertia), probe_update(plain, psi, inertia)
    assert np.abs(a - b).max() < 1e-14 * np.abs(b).max()


@pytest.mark.parametrize("modulus", [lambda u: 10.0 ** (-3.0 * u),
                                     lambda u: np.where(u < 0.5, 0.0, 1.0)],
                         ids=["decades", "binary"])
@pytest.mark.parametrize("offsets", [whole, fractional], ids=["whole", "fractional"])
@pytest.mark.parametrize("inertia", [0.0, 0.05])
def test_overlap_error_never_rises_under_a_moved_probe(modulus, offsets, inertia):
    p, psi, _ = overlap_state(modulus, offsets)
    first = before = overlap_error(p, psi)
    rise = 0.0
    for _ in range(30):
        p.probe = probe_update(p, psi, inertia)
        now = overlap_error(p, psi)
        if before > 1e-24 * first:
            rise = max(rise, now / before)
        before = now
    assert rise <= 1.0 + 1e-12
    assert before / first < (1.0 if inertia == 0.0 else 0.2)


@pytest.mark.parametrize("inertia", [0.0, 0.001])
def test_probe_update_under_a_moved_probe_holds_the_solution(inertia):
    p, psi, truth = overlap_state(lambda u: 0.2 + 0.8 * u, fractional)
    p.probe = truth.copy()
    for _ in range(3):
        p.probe = probe_update(p, psi, inertia)
    assert np.abs(p.probe - truth).max() < 1e-13 * np.abs(truth).max()
    p.probe = np.zeros_like(truth)
    assert not probe_update(p, np.zeros_like(psi), inertia).any()


@pytest.mark.parametrize("algorithm", ["ap", "dm", "raar"])
def test_carried_algorithms_with_refined_positions_recover_offsets(algorithm):
    """AP, DM and RAAR under the move with the positions refined, from the nominal positions of
    counts made at sub-pixel offsets: the LLK falls and the offsets move toward the drawn ones."""
    d0 = np.random.default_rng(8).uniform(-0.8, 0.8, (14, 2))
    p, truth = small_scan(offsets=d0)
    p.object = truth * 0.97 * np.exp(0.05j)
    p.set_positions(np.zeros((p.addr.nframe, 2)), refine=True)
    start = p.llk().poisson
    kw = dict(probe_inertia=0.001) if algorithm == "ap" else {}
    getattr(p, algorithm)(15, calc_llk=0, zero_phase_ramp=False, **kw)
    err0 = np.abs(d0 - d0.mean(0)).mean()
    err = np.abs((d0 - d0.mean(0)) - (p.offsets - p.offsets.mean(0))).mean()
    assert p.llk().poisson < start
    assert err < err0
