"""The BH oracle (oracle/bh.py) on the reference's seeded far-field scenario
(`dm_scenario(32, 40, 2, 2e5, 4.0)` after `scale_obj_probe`, redrawn by oracle/scenario.py):
its gradient and Hessian against central differences, and two epochs with one batch of every
frame and with batches of 16 against the reference's float64 BH runs
(ptyrs/tests/engine_bh.rs:85-243, `bh_{full,mini}_*_f64.txt`); with the offsets refined under
Patch the same against central differences over object, probe and offsets and two epochs
against the reference's float64 model (ptyrs/tests/engine_bh_pos.rs:62-170,
`bh_pos_{full,mini}_*_f64.txt`, position_rho 2)."""
import numpy as np
import pytest

from oracle.bh import Bh, BhBatch, amplitude_cost
from test_oracle_farfield import golden, max_rel, state

FRAMES = range(0, 16)


def rel(a, b):
    return abs(a - b) / abs(b)


def direction(like, rng):
    scale = np.abs(like).max()
    return scale * (rng.uniform(-0.5, 0.5, like.shape) + 1j * rng.uniform(-0.5, 0.5, like.shape))


def batch_views(p):
    return np.concatenate([p.addr.frame_views(f) for f in FRAMES])


def test_grads_match_central_differences():
    """engine_bh.rs:95-125: ⟨g, d⟩ against (F(x + h·d) − F(x − h·d))/2h along random object
    and probe directions (the gradient carries the 1e-8 amplitude offset, the differences do
    not)."""
    p = state()
    views = batch_views(p)
    b = BhBatch(views, p.obs, p.optics, p.object, p.probe)
    g_obj, g_probe, _ = b.grads()
    rng = np.random.default_rng(1)
    d_obj, d_probe = direction(p.object, rng), direction(p.probe, rng)
    h = 1e-5
    f = lambda o, pr: amplitude_cost(views, p.obs, p.optics, o, pr)
    fo = (f(p.object + h * d_obj, p.probe) - f(p.object - h * d_obj, p.probe)) / (2 * h)
    fp = (f(p.object, p.probe + h * d_probe) - f(p.object, p.probe - h * d_probe)) / (2 * h)
    an_o = float(np.sum((np.conj(g_obj) * d_obj).real))
    an_p = float(np.sum((np.conj(g_probe) * d_probe).real))
    assert rel(an_o, fo) < 1e-6 and rel(an_p, fp) < 1e-6


def test_hessian_matches_central_differences():
    """engine_bh.rs:127-152: H(u, v) = H(v, u), and against the central difference of
    ⟨g(x + h·v), u⟩."""
    p = state()
    views = batch_views(p)
    rng = np.random.default_rng(2)
    u = (direction(p.object, rng), direction(p.probe, rng))
    v = (direction(p.object, rng), direction(p.probe, rng))
    b = BhBatch(views, p.obs, p.optics, p.object, p.probe)
    h_uv, h_vu = b.hessian(u, v), b.hessian(v, u)
    assert rel(h_vu, h_uv) < 1e-13

    def du(t):
        g = BhBatch(views, p.obs, p.optics, p.object + t * v[0], p.probe + t * v[1]).grads()[:2]
        return float(np.sum((np.conj(g[0]) * u[0]).real) + np.sum((np.conj(g[1]) * u[1]).real))

    h = 1e-6
    assert rel(h_uv, (du(h) - du(-h)) / (2 * h)) < 1e-6


@pytest.mark.parametrize("name,batch", [("bh_full", 40), ("bh_mini", 16)])
def test_epochs_match_reference(name, batch):
    """engine_bh.rs:154-243: two epochs (seed 7, probe_rho 0.01): every step's frames, β, α,
    ⟨-g, D⟩ and H(D, D), and the object and probe changes of each epoch."""
    p = state()
    g = golden(name)
    run = Bh(batch, probe_rho=0.01, seed=7)
    obj, probe = p.object, p.probe
    got, changes = [], []
    for e in range(2):
        o0, p0 = obj, probe
        obj, probe, steps = run.epoch(p.addr, p.obs, p.optics, obj, probe)
        got += [(e, s) for s in steps]
        changes.append((obj - o0, probe - p0))
    rows = g["steps"]
    assert len(got) == len(rows)
    for k, ((e, s), r) in enumerate(zip(got, rows)):
        count = int(r[2])
        assert [k, e, count] == [int(r[0]), int(r[1]), len(s["frames"])]
        assert s["frames"] == [int(f) for f in r[7:7 + count]]
        if r[3] == 0.0:
            assert s["beta"] == 0.0
        else:
            assert rel(s["beta"], r[3]) < 1e-12
        for key, want in (("alpha", r[4]), ("top", r[5]), ("bottom", r[6])):
            assert rel(s[key], want) < 1e-12, (k, key)
    for e, (d_obj, d_probe) in enumerate(changes):
        o = g["obj"][:, 2 + 2 * e] + 1j * g["obj"][:, 3 + 2 * e]
        pr = g["probe"][:, 3 + 2 * e] + 1j * g["probe"][:, 4 + 2 * e]
        assert max_rel(np.stack([d_obj.ravel().real, d_obj.ravel().imag], 1),
                       np.stack([o.real, o.imag], 1)) < 1e-12
        assert max_rel(np.stack([d_probe.ravel().real, d_probe.ravel().imag], 1),
                       np.stack([pr.real, pr.imag], 1)) < 5e-12


def start_offsets(name="bh_pos_full"):
    """The reference run's start offsets, `[dy, dx]` per frame (columns 1-2 of its table)."""
    return golden(name)["offsets"][:, 1:3].copy()


def test_grads_with_offsets_match_central_differences():
    """⟨g, d⟩ over object, probe and the refined offsets against central differences of F
    (bh_pos.py's check)."""
    p = state()
    views = batch_views(p)
    d0 = start_offsets()[list(FRAMES)]
    b = BhBatch(views, p.obs, p.optics, p.object, p.probe, d0, refine=True)
    g_obj, g_probe, g_d = b.grads()
    rng = np.random.default_rng(3)
    u_obj, u_probe = direction(p.object, rng), direction(p.probe, rng)
    u_d = rng.uniform(-1, 1, d0.shape)
    f = lambda o, pr, d: amplitude_cost(views, p.obs, p.optics, o, pr, d)
    h = 1e-5
    for an, plus, minus in (
            (float(np.sum((np.conj(g_obj) * u_obj).real)),
             (p.object + h * u_obj, p.probe, d0), (p.object - h * u_obj, p.probe, d0)),
            (float(np.sum((np.conj(g_probe) * u_probe).real)),
             (p.object, p.probe + h * u_probe, d0), (p.object, p.probe - h * u_probe, d0)),
            (float((g_d * u_d).sum()),
             (p.object, p.probe, d0 + h * u_d), (p.object, p.probe, d0 - h * u_d))):
        assert rel(an, (f(*plus) - f(*minus)) / (2 * h)) < 1e-6


@pytest.mark.parametrize("refine", [True, False])
def test_hessian_with_offsets_matches_central_differences(refine):
    """H(u, v) = H(v, u) and against the central difference of ⟨g(x + h·v), u⟩ over object,
    probe and (refined) offsets; held offsets move the probe only."""
    p = state()
    views = batch_views(p)
    d0 = start_offsets()[list(FRAMES)]
    rng = np.random.default_rng(4)
    nd = lambda: rng.uniform(-1, 1, d0.shape) if refine else None
    u = (direction(p.object, rng), direction(p.probe, rng), nd())
    v = (direction(p.object, rng), direction(p.probe, rng), nd())
    b = BhBatch(views, p.obs, p.optics, p.object, p.probe, d0, refine=refine)
    h_uv, h_vu = b.hessian(u, v), b.hessian(v, u)
    assert rel(h_vu, h_uv) < 1e-12

    def du(t):
        d = d0 + t * v[2] if refine else d0
        g = BhBatch(views, p.obs, p.optics, p.object + t * v[0], p.probe + t * v[1], d,
                    refine=refine).grads()
        s = float(np.sum((np.conj(g[0]) * u[0]).real) + np.sum((np.conj(g[1]) * u[1]).real))
        return s + (float((g[2] * u[2]).sum()) if refine else 0.0)

    h = 1e-6
    assert rel(h_uv, (du(h) - du(-h)) / (2 * h)) < 1e-6


@pytest.mark.parametrize("name,batch", [("bh_pos_full", 40), ("bh_pos_mini", 16)])
def test_epochs_with_refined_offsets_match_reference(name, batch):
    """engine_bh_pos.rs:62-170: two epochs (seed 7, probe_rho 0.01, position_rho 2) from the
    reference run's offsets: every step's frames, β, α, −⟨g, D⟩ and H(D, D) to 3e-12, the
    object and probe changes relative to the largest start value and the offsets' changes
    relative to the largest of them, to 3e-12."""
    p = state()
    g = golden(name)
    start = g["offsets"][:, 1:3]
    run = Bh(batch, probe_rho=0.01, seed=7, position_rho=2.0, offsets=start, refine=True)
    obj, probe = p.object, p.probe
    got = []
    for e in range(2):
        obj, probe, steps = run.epoch(p.addr, p.obs, p.optics, obj, probe)
        got += [(e, s) for s in steps]
    rows = g["steps"]
    assert len(got) == len(rows)
    for k, ((e, s), r) in enumerate(zip(got, rows)):
        count = int(r[2])
        assert [k, e, count] == [int(r[0]), int(r[1]), len(s["frames"])]
        assert s["frames"] == [int(f) for f in r[7:7 + count]]
        if r[3] == 0.0:
            assert s["beta"] == 0.0
        for key, want in (("beta", r[3]), ("alpha", r[4]), ("top", r[5]), ("bottom", r[6])):
            if want != 0.0:
                assert rel(s[key], want) < 3e-12, (k, key)
    d_obj, d_probe = obj - p.object, probe - p.probe
    want_o = g["obj"][:, 2] + 1j * g["obj"][:, 3]
    want_p = g["probe"][:, 3] + 1j * g["probe"][:, 4]
    ri = lambda z: np.stack([np.ravel(z).real, np.ravel(z).imag], 1)
    assert max_rel(ri(d_obj), ri(want_o), np.abs(ri(p.object)).max()) < 3e-12
    assert max_rel(ri(d_probe), ri(want_p), np.abs(ri(p.probe)).max()) < 3e-12
    want_d = g["offsets"][:, 3:5] - start
    assert max_rel(run.offsets - start, want_d) < 3e-12


def test_epochs_through_slices_match_reference():
    """engine_bh_multislice.rs:116-190: BH through three slices (the multislice LSQML state and
    counts; angular-spectrum, Fresnel and far-field exits), CG over one batch of all 16 frames
    and steepest descent over batches of 6, three epochs (seed 7, probe_rho 1): every step's
    frames, β, α, top and bottom to 2e-13 and the slices' and the probe's changes to 2e-12, the
    reference's own bounds (measured here 2e-14 and 2.4e-13 with the Hessian's bilinear form by
    polarization)."""
    from test_oracle_golden import multislice_state
    g = golden("bh_multislice")
    _, addr, objs0, probe0, cases = multislice_state()
    ri = lambda z: np.stack([np.ravel(z).real, np.ravel(z).imag], 1).ravel()
    for case, (optics, obs, _) in enumerate(cases):
        for method, batch in enumerate((16, 6)):
            run = Bh(batch, probe_rho=1.0, seed=7)
            objs, probe = list(objs0), probe0.copy()
            got = []
            for e in range(3):
                objs, probe, steps = run.epoch(addr, obs, optics, objs, probe)
                got += [(e, s) for s in steps]
            sel = lambda t: t[(t[:, 0] == case) & (t[:, 1] == method)]
            rows = sel(g["steps"])
            assert len(got) == len(rows)
            for k, ((e, s), r) in enumerate(zip(got, rows)):
                count = int(r[4])
                assert [k, e, count] == [int(r[2]), int(r[3]), len(s["frames"])]
                assert s["frames"] == [int(f) for f in r[10:10 + count]]
                if r[5] == 0.0:
                    assert s["beta"] == 0.0
                for key, want in (("beta", r[5]), ("alpha", r[6]), ("top", r[7]),
                                  ("bottom", r[8])):
                    if want != 0.0:
                        assert rel(s[key], want) < 2e-13, (case, method, k, key)
            d_objs = np.concatenate([ri(o - o0) for o, o0 in zip(objs, objs0)])
            assert max_rel(d_objs, sel(g["obj"])[:, 5:7].ravel()) < 2e-12
            assert max_rel(ri(probe - probe0), sel(g["probe"])[:, 5:7].ravel()) < 2e-12
