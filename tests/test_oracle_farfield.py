"""The oracle on the reference's seeded far-field scenario against its golden far-field
results: `oracle/scenario.py` redraws `dm_scenario(32, 40, nprobe, 2e5, 4.0)` (ChaCha8 Poisson
counts, tests/common/engine/scenario.rs) and is itself pinned by the scenario's Poisson and
Euclidian sums; then the position gradient (ptyrs/tests/engine_features.rs:56-103), ML with
refined positions (engine_ml_pos.rs), LSQML steps and epochs with and without positions
(engine_lsqml.rs, engine_lsqml_pos.rs), rPIE's LLK trace against pty-chi
(engine_reconstruct.rs:222-236) and DM's and RAAR's against PyNX (engine_reconstruct.rs:186-220),
to the reference's own tolerances."""
import functools
import os

import numpy as np
import pytest

from oracle import ops
from oracle.lsqml import Lsqml
from oracle.ptycho import Ptycho
from oracle.scenario import dm_scenario

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@functools.lru_cache(maxsize=None)
def scenario(nprobe):
    return dm_scenario(32, 40, nprobe, 2e5, 4.0)


def state(nprobe=2):
    """`Ptycho::new` on the scenario, then `scale_obj_probe` (engine_lsqml.rs:24-29)."""
    s = scenario(nprobe)
    p = Ptycho(s["counts"], s["y"], s["x"], s["optics"], s["object"], s["probe"])
    p.scale_obj_probe()
    return p


def max_rel(a, b, scale=None):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.abs(a - b).max() / (np.abs(b).max() if scale is None else scale))


def re_im(a):
    a = np.ravel(a)
    return np.stack([a.real, a.imag], 1).ravel()


def frame_offsets(p, rows, col):
    return np.array([[r[col], r[col + 1]] for r in rows])


def test_scenario_counts_reproduce_the_reference_draw():
    """The redrawn counts give the reference's nb_obs, Poisson sum and a quarter of the
    Euclidian sum at its offsets to 1e-12 (engine_features.rs:42-54, 85-90)."""
    p = state()
    g = golden("pos_grad")
    rows, (nb, L, F) = g["table"], g["values"][0]
    nm = p.addr.nmode
    d = np.array([[r[1] - p.addr.views[f * nm]["oy"], r[2] - p.addr.views[f * nm]["ox"]]
                  for f, r in enumerate(rows)])
    assert np.abs(d).max() < 0.5
    p.set_positions(d)
    l = ops.llk(p.obs, slice(0, p.addr.nframe), nm, p.optics.exit_forward(p.calc_psi()))
    assert p.obs.nb_obs == nb
    assert abs(l.poisson - L) < 1e-12 * abs(L)
    assert abs(l.euclidian / 4.0 - F) < 1e-12 * abs(F)


@pytest.mark.parametrize("cost,col", [("poisson", 3), ("amplitude", 5)])
def test_position_gradient_matches_golden(cost, col):
    p = state()
    rows = golden("pos_grad")["table"]
    nm = p.addr.nmode
    d = np.array([[r[1] - p.addr.views[f * nm]["oy"], r[2] - p.addr.views[f * nm]["ox"]]
                  for f, r in enumerate(rows)])
    got = p.position_grad(cost, d)
    assert max_rel(got, rows[:, col:col + 2]) < 1e-12


def test_ml_with_refined_positions_matches_golden():
    """Four ML cycles refining the offsets from the golden start (engine_ml_pos.rs:53-118)."""
    p = state()
    g = golden("ml_pos")
    start = frame_offsets(p, g["offsets"], 1)
    p.set_positions(start, refine=True)
    o0, p0 = p.object.copy(), p.probe.copy()
    p.ml(4, update_object=True, update_probe=True, calc_llk=1, zero_phase_ramp=False)
    assert max_rel(re_im(p.object - o0), g["obj"][:, 2:4], np.abs(re_im(o0)).max()) < 1e-13
    assert max_rel(re_im(p.probe - p0), g["probe"][:, 3:5], np.abs(re_im(p0)).max()) < 1e-13
    want = frame_offsets(p, g["offsets"], 3) - start
    assert max_rel(p.offsets - start, want) < 1e-12


def views_of(p, frames):
    return np.concatenate([p.addr.frame_views(f) for f in frames])


@pytest.mark.parametrize("cost,name", [("amplitude", "lsqml_gaussian"),
                                       ("poisson", "lsqml_poisson")])
def test_lsqml_step_matches_golden(cost, name):
    """One step on frames 0..20 with the illumination as preconditioner (engine_lsqml.rs:
    196-236)."""
    p = state()
    g = golden(name)
    run = Lsqml(20, cost, 0)
    run.preconditioner = ops.illumination(p.addr.views, p.object.shape, p.probe)
    frames = list(range(20))
    obj, probe, st = run.step(views_of(p, frames), p.obs, p.optics, p.object, p.probe)
    assert st["frames"] == frames
    assert max_rel(st["a_far"], g["steps"][:, 1]) < 1e-13
    assert max_rel(st["a_obj"], g["steps"][:, 2]) < 1e-12
    assert max_rel(st["a_probe"], g["steps"][:, 3]) < 1e-12
    assert max_rel(re_im(obj - p.object), g["obj"][:, 2:4]) < 1e-12
    assert max_rel(re_im(probe - p.probe), g["probe"][:, 3:5]) < 1e-12


@pytest.mark.parametrize("cost,name", [("amplitude", "lsqml_epochs_gaussian"),
                                       ("poisson", "lsqml_epochs_poisson")])
def test_lsqml_epochs_match_golden(cost, name):
    """Three epochs of batches of 16, seed 7 (engine_lsqml.rs:300-350)."""
    p = state()
    g = golden(name)
    rows = g["steps"]
    run = Lsqml(16, cost, 7)
    obj, probe, nxt = p.object, p.probe, 0
    for e in range(3):
        obj, probe, sts = run.epoch(p.addr, p.obs, p.optics, obj, probe)
        for st in sts:
            want = rows[nxt:nxt + len(st["frames"])]
            nxt += len(st["frames"])
            assert (want[:, 0] == e).all()
            assert st["frames"] == [int(v) for v in want[:, 1]]
            assert max_rel(st["a_far"], want[:, 2]) < 1e-13
            assert max_rel(st["a_obj"], want[:, 3]) < 1e-12
            assert max_rel(st["a_probe"], want[:, 4]) < 1e-12
    assert nxt == len(rows)
    assert max_rel(re_im(obj - p.object), g["obj"][:, 2:4]) < 1e-12
    assert max_rel(re_im(probe - p.probe), g["probe"][:, 3:5]) < 1e-12


@pytest.mark.parametrize("cost,noise", [("amplitude", 0), ("poisson", 1)])
def test_lsqml_positions_step_matches_golden(cost, noise):
    """One step refining the offsets from the golden start (engine_lsqml_pos.rs:128-180)."""
    p = state()
    g = golden("lsqml_pos")
    rows = g["steps"]
    frames = [int(v) for v in rows[:, 0]]
    start = frame_offsets(p, g["offsets"], 1)
    run = Lsqml(len(frames), cost, 0, offsets=start.copy(), refine=True)
    run.preconditioner = ops.illumination(p.addr.views, p.object.shape, p.probe)
    obj, probe, st = run.step(views_of(p, frames), p.obs, p.optics, p.object, p.probe)
    col = 1 + 3 * noise
    assert st["frames"] == frames
    assert max_rel(st["a_far"], rows[:, col]) < 1e-13
    assert max_rel(st["a_obj"], rows[:, col + 1]) < 1e-12
    assert max_rel(st["a_probe"], rows[:, col + 2]) < 1e-12
    c = 2 + 2 * noise
    assert max_rel(re_im(obj - p.object), g["obj"][:, c:c + 2]) < 1e-12
    c = 3 + 2 * noise
    assert max_rel(re_im(probe - p.probe), g["probe"][:, c:c + 2]) < 1e-12
    want = frame_offsets(p, g["offsets"], 3 + 2 * noise) - start
    assert max_rel(run.offsets - start, want) < 1e-12


@pytest.mark.parametrize("cost,noise", [("amplitude", 0), ("poisson", 1)])
def test_lsqml_positions_epochs_match_golden(cost, noise):
    """Three epochs of batches of 16 refining the offsets (engine_lsqml_pos.rs:214-264)."""
    p = state()
    g = golden("lsqml_pos_epochs")
    rows = g["steps"]
    start = frame_offsets(p, g["offsets"], 1)
    run = Lsqml(16, cost, 7, offsets=start.copy(), refine=True)
    obj, probe, nxt = p.object, p.probe, 0
    col = 2 + 3 * noise
    for e in range(3):
        obj, probe, sts = run.epoch(p.addr, p.obs, p.optics, obj, probe)
        for st in sts:
            want = rows[nxt:nxt + len(st["frames"])]
            nxt += len(st["frames"])
            assert (want[:, 0] == e).all()
            assert st["frames"] == [int(v) for v in want[:, 1]]
            assert max_rel(st["a_far"], want[:, col]) < 1e-13
            assert max_rel(st["a_obj"], want[:, col + 1]) < 1e-12
            assert max_rel(st["a_probe"], want[:, col + 2]) < 1e-12
    assert nxt == len(rows)
    c = 2 + 2 * noise
    assert max_rel(re_im(obj - p.object), g["obj"][:, c:c + 2]) < 1e-12
    c = 3 + 2 * noise
    assert max_rel(re_im(probe - p.probe), g["probe"][:, c:c + 2]) < 1e-12
    want = frame_offsets(p, g["offsets"], 3 + 2 * noise) - start
    assert max_rel(run.offsets - start, want) < 1e-11


def test_rpie_llk_trace_matches_ptychi():
    """Twenty rPIE epochs (pty-chi's settings: steps 1, alphas 0.5, batches of 4, seed 7) on the
    one-mode scenario, every LLK record to 1e-9 (engine_reconstruct.rs:222-236)."""
    p = state(nprobe=1)
    p.rpie(20, obj_step=1.0, probe_step=1.0, obj_alpha=0.5, probe_alpha=0.5, batch_size=4,
           calc_llk=1, seed=7)
    rows = golden("rpie_ptychi")["table"]
    assert len(p.history) == len(rows)
    for rec, row in zip(p.history, rows):
        assert rec["cycle"] == row[0]
        for key, want in zip(("poisson", "gaussian", "euclidian", "nb_photons_calc"), row[1:]):
            assert abs(rec[key] - want) < 1e-9 * abs(want), (rec["cycle"], key)


@pytest.mark.parametrize("algorithm", ["dm", "raar"])
def test_dm_raar_llk_traces_match_pynx(algorithm):
    """Twenty-one cycles of DM or RAAR at PyNX's defaults recording every cycle on the scaled
    one-mode scenario: record 0 is the start, record c + 1 the PyNX record of cycle c (PyNX
    takes the estimate after the update), every column to 1e-9 (engine_reconstruct.rs:162-220)."""
    p = state(nprobe=1)
    start = p.llk().as_dict()
    getattr(p, algorithm)(21, calc_llk=1)
    first, rest = p.history[0], p.history[1:]
    cols = ("poisson", "gaussian", "euclidian", "nb_photons_calc")
    assert first["cycle"] == 0 and all(first[k] == start[k] for k in cols)
    rows = golden(f"{algorithm}_pynx")["table"]
    assert len(rest) == len(rows)
    for rec, row in zip(rest, rows):
        assert rec["cycle"] == row[0] + 1 and rec["algorithm"] == algorithm
        for key, want in zip(cols, row[1:]):
            assert abs(rec[key] - want) < 1e-9 * abs(want), (rec["cycle"], key)


@pytest.mark.parametrize("name,params,nepoch", [
    ("rpie_pos_step", dict(obj_step=0.9, probe_step=0.8, obj_alpha=0.3, probe_alpha=0.2,
                           batch_size=20), 1),
    ("rpie_pos_epochs", dict(obj_step=1.0, probe_step=1.0, obj_alpha=0.5, probe_alpha=0.5,
                             batch_size=4), 3)])
def test_rpie_with_refined_positions_matches_ptychi(name, params, nepoch):
    """rPIE refining the offsets under PATCH against pty-chi's `RPIEReconstructor`
    (engine_rpie_pos.rs:59-150): object and probe changes to 1e-12, offset changes 3e-12."""
    p = state()
    g = golden(name)
    start = frame_offsets(p, g["offsets"], 1)
    p.set_positions(start, refine=True)
    o0, p0 = p.object.copy(), p.probe.copy()
    p.rpie(nepoch, calc_llk=1, seed=7, **params)
    assert max_rel(re_im(p.object - o0), g["obj"][:, 2:4]) < 1e-12
    assert max_rel(re_im(p.probe - p0), g["probe"][:, 3:5]) < 1e-12
    want = frame_offsets(p, g["offsets"], 3) - start
    assert max_rel(p.offsets - start, want) < 3e-12


@pytest.mark.parametrize("cost,noise", [("amplitude", 0), ("poisson", 1)])
def test_lsqml_positions_with_opr_step_matches_golden(cost, noise):
    """One step refining the offsets with three eigenmodes of probe mode 0 and their weights
    refined (engine_lsqml_pos.rs:121-200 with `opr`): steps, changes, offsets, eigenmodes and
    weights after it."""
    from oracle.opr import ProbeVariation
    p = state()
    g = golden("lsqml_pos_opr")
    rows = g["steps"]
    frames = [int(v) for v in rows[:, 0]]
    start = frame_offsets(p, g["offsets"], 1)
    e, w = g["eigen"], g["weights"]
    u0 = (e[:, 3] + 1j * e[:, 4]).reshape(3, 32, 32)
    w0 = w[:, 1:4].ravel()
    var = ProbeVariation(u0, w0)
    run = Lsqml(len(frames), cost, 0, offsets=start.copy(), refine=True, var=var)
    run.preconditioner = ops.illumination(p.addr.views, p.object.shape, p.probe)
    obj, probe, st = run.step(views_of(p, frames), p.obs, p.optics, p.object, p.probe)
    col = 1 + 3 * noise
    assert st["frames"] == frames
    assert max_rel(st["a_far"], rows[:, col]) < 1e-13
    assert max_rel(st["a_obj"], rows[:, col + 1]) < 1e-12
    assert max_rel(st["a_probe"], rows[:, col + 2]) < 1e-12
    c = 2 + 2 * noise
    assert max_rel(re_im(obj - p.object), g["obj"][:, c:c + 2]) < 1e-12
    c = 3 + 2 * noise
    assert max_rel(re_im(probe - p.probe), g["probe"][:, c:c + 2]) < 1e-12
    want = frame_offsets(p, g["offsets"], 3 + 2 * noise) - start
    assert max_rel(run.offsets - start, want) < 1e-12
    c = 5 + 2 * noise
    u1 = (e[:, c] + 1j * e[:, c + 1]).reshape(3, 32, 32)
    assert max_rel(re_im(var.eigenmodes), re_im(u1)) < 1e-13
    w1 = w[:, 4 + 3 * noise:7 + 3 * noise].ravel()
    assert max_rel(var.weights - w0, w1 - w0) < 1e-13
