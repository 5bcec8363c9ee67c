"""The oracle's OPR probe variation (oracle/opr.py, `Lsqml(var=...)`) against the reference's
golden OPR sets on the redrawn scenario `dm_scenario(32, 40, 2, 2e5, 4.0)` after
`scale_obj_probe` (ptyrs/tests/engine_opr.rs): the costs and LSQML's LLK of every frame's own
probe, the weight gradients, one OPR step alone (one eigenmode) and inside an LSQML step (three
eigenmodes, with and without the main mode's weights), to the reference's own bounds."""
import functools
import os

import numpy as np
import pytest

from oracle import ops
from oracle.lsqml import Lsqml
from oracle.opr import ProbeVariation, opr_weight_grad, unique_views
from oracle.ptycho import Ptycho
from oracle.scenario import dm_scenario

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
N = 32

# columns of each reference's tables (engine_opr.rs:88-118): `u` the re columns of U, U''
# Gaussian, U'' Poisson; `w` the first of the k columns of w, dL/dw, dF/dw, w' Gaussian,
# w' Poisson; `c` the main mode's weights c, c' Gaussian, c' Poisson
REFS = {
    "opr": dict(k=1, u=(2, 4, 6), w=(1, 2, 3, 4, 5), c=None),
    "lsqml_opr": dict(k=3, u=(3, 5, 7), w=(1, 4, 7, 10, 13), c=None),
    "lsqml_opr_int": dict(k=3, u=(3, 5, 7), w=(2, 5, 8, 12, 16), c=(1, 11, 15)),
}


@functools.lru_cache(maxsize=None)
def golden(name):
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@functools.lru_cache(maxsize=None)
def _scenario():
    return dm_scenario(32, 40, 2, 2e5, 4.0)


def state():
    s = _scenario()
    p = Ptycho(s["counts"], s["y"], s["x"], s["optics"], s["object"], s["probe"])
    p.scale_obj_probe()
    return p


def max_rel(a, b):
    a, b = np.ravel(a), np.ravel(b)
    if np.iscomplexobj(a) or np.iscomplexobj(b):
        a = np.stack([np.real(a), np.imag(a)], 1).ravel()
        b = np.stack([np.real(b), np.imag(b)], 1).ravel()
    return float(np.abs(a - b).max() / np.abs(b).max())


def eigenmodes(name, re):
    r, t = REFS[name], golden(name)["eigen"]
    return (t[:, re] + 1j * t[:, re + 1]).reshape(r["k"], N, N)


def weights(name, c):
    return golden(name)["weights"][:, c:c + REFS[name]["k"]].ravel()


def column(name, c):
    return golden(name)["weights"][:, c].copy()


def variation(name, w=None):
    r = REFS[name]
    w = weights(name, r["w"][0]) if w is None else w
    intensity = column(name, r["c"][0]) if r["c"] else None
    return ProbeVariation(eigenmodes(name, r["u"][0]), w, intensity=intensity)


def all_views(p, frames):
    return np.concatenate([p.addr.frame_views(f) for f in frames])


def per_frame_llk(p, var, frames):
    views = all_views(p, frames)
    np_, nmode = p.probe.shape[0], p.addr.nmode
    planes = var.planes(frames, p.probe)
    uviews = unique_views(views, len(frames), np_, nmode)
    psi = p.optics.exit_forward(ops.obj_probe_to_psi(uviews, p.object, planes, p.optics.quad))
    return ops.llk(p.obs, frames, nmode, psi)


@pytest.mark.parametrize("name", sorted(REFS))
def test_costs_of_every_frames_own_probe(name):
    """engine_opr.rs:201-222: the Poisson sum and the amplitude cost (Euclidian / 4) over
    every frame, each with its own probe."""
    p = state()
    nb, L, F = golden(name)["values"][0]
    assert p.obs.nb_obs == nb
    l = per_frame_llk(p, variation(name), list(range(40)))
    assert abs(l.poisson - L) < 1e-13 * abs(L)
    assert abs(l.euclidian / 4.0 - F) < 1e-13 * abs(F)


@pytest.mark.parametrize("name", sorted(REFS))
def test_lsqml_llk_reads_every_frames_own_probe(name):
    p = state()
    nb, L, F = golden(name)["values"][0]
    got = Lsqml(40, "poisson", 0, var=variation(name)).llk(p.addr, p.obs, p.optics, p.object,
                                                            p.probe)
    assert abs(got.poisson * nb - L) < 1e-13 * abs(L)
    assert abs(got.euclidian * nb / 4.0 - F) < 1e-13 * abs(F)


@pytest.mark.parametrize("name", sorted(REFS))
@pytest.mark.parametrize("cost", ["poisson", "amplitude"])
def test_weight_gradients(name, cost):
    """engine_opr.rs:311-326: ∂cost/∂w of every frame and eigenmode against the reference's."""
    p = state()
    r = REFS[name]
    g = opr_weight_grad(cost, all_views(p, range(40)), p.obs, p.optics, p.object, p.probe,
                        variation(name))
    want = weights(name, r["w"][1] if cost == "poisson" else r["w"][2])
    assert max_rel(g, want) < 1e-13


def lsqml_step(p, cost, frames, var):
    run = Lsqml(len(frames), cost, 0, var=var)
    run.preconditioner = ops.illumination(p.addr.views, p.object.shape, p.probe)
    obj, probe, rec = run.step(all_views(p, frames), p.obs, p.optics, p.object, p.probe)
    assert list(rec["frames"]) == list(frames)
    return rec, obj - p.object, probe - p.probe


def assert_variation(name, var, frames, noise):
    r = REFS[name]
    assert max_rel(var.eigenmodes, eigenmodes(name, r["u"][1 + noise])) < 1e-13
    start, want = weights(name, r["w"][0]), weights(name, r["w"][3 + noise])
    assert_change(var.weights, start, want, r["k"], frames)
    if r["c"]:
        assert_change(var.intensity, column(name, r["c"][0]), column(name, r["c"][1 + noise]),
                      1, frames)


def assert_change(got, start, want, per, frames):
    moved, expected = [], []
    for f in range(len(start) // per):
        ws = slice(f * per, (f + 1) * per)
        if f in frames:
            moved.append(got[ws] - start[ws])
            expected.append(want[ws] - start[ws])
        else:
            assert np.array_equal(got[ws], start[ws])
    assert max_rel(np.concatenate(moved), np.concatenate(expected)) < 1e-13


@pytest.mark.parametrize("cost,noise", [("amplitude", 0), ("poisson", 1)])
def test_opr_step(cost, noise):
    """engine_opr.rs:451-472: one eigenmode, the step on frames 0–19: Poisson's a_far, the
    eigenmode and the weights."""
    p = state()
    var = variation("opr")
    frames = list(range(20))
    rec, _, _ = lsqml_step(p, cost, frames, var)
    if cost == "poisson":
        assert max_rel(rec["a_far"], column("opr", 6)[:20]) < 1e-13
    assert_variation("opr", var, frames, noise)


@pytest.mark.parametrize("name", ["lsqml_opr", "lsqml_opr_int"])
@pytest.mark.parametrize("cost,noise", [("amplitude", 0), ("poisson", 1)])
def test_lsqml_step_with_opr(name, cost, noise):
    """engine_opr.rs:474-520: three eigenmodes inside an LSQML step on the reference's batch:
    per-frame a_far, a_obj, a_probe, the object and probe changes, the eigenmodes and weights."""
    p = state()
    var = variation(name)
    g = golden(name)
    rows = g["steps"]
    frames = [int(f) for f in rows[:, 0]]
    rec, d_obj, d_probe = lsqml_step(p, cost, frames, var)
    for key, col, tol in [("a_far", 1, 1e-13), ("a_obj", 2, 1e-12), ("a_probe", 3, 1e-12)]:
        assert max_rel(rec[key], rows[:, col + 3 * noise]) < tol, key
    o, c = g["obj"], 2 + 2 * noise
    assert max_rel(d_obj, o[:, c] + 1j * o[:, c + 1]) < 1e-12
    pr, c = g["probe"], 3 + 2 * noise
    assert max_rel(d_probe, pr[:, c] + 1j * pr[:, c + 1]) < 1e-12
    assert_variation(name, var, frames, noise)


@pytest.mark.parametrize("name", sorted(REFS))
def test_one_frame_batch_moves_only_main_mode_weights(name):
    """engine_opr.rs:534-558: a one-frame batch moves no eigenmode or w; refined main-mode
    weights move at that frame as in the reference's batch."""
    p = state()
    var = variation(name)
    start = variation(name)
    rec, _, _ = lsqml_step(p, "amplitude", [3], var)
    assert len(rec["a_far"]) == 1
    assert np.array_equal(var.eigenmodes, start.eigenmodes)
    assert np.array_equal(var.weights, start.weights)
    r = REFS[name]
    if r["c"]:
        assert_change(var.intensity, column(name, r["c"][0]), column(name, r["c"][1]), 1, [3])
