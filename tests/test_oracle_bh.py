"""The BH oracle (oracle/bh.py) on the reference's seeded far-field scenario
(`dm_scenario(32, 40, 2, 2e5, 4.0)` after `scale_obj_probe`, redrawn by oracle/scenario.py):
its gradient and Hessian against central differences, and two epochs with one batch of every
frame and with batches of 16 against the reference's float64 BH runs
(ptyrs/tests/engine_bh.rs:85-243, `bh_{full,mini}_*_f64.txt`)."""
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
    g_obj, g_probe = b.grads()
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
        g = BhBatch(views, p.obs, p.optics, p.object + t * v[0], p.probe + t * v[1]).grads()
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
