"""The f64 oracle against the reference's golden vectors (pty-chi runs in float64 saved by the
reference, converted by `tests/golden/make_golden.py`), to the reference's own bounds:
`ptyrs/tests/engine_rpie_near.rs` (rPIE, LLK trace and changes to 1e-12) and
`ptyrs/tests/engine_lsqml_near.rs` (LSQML forward model, one step, and the epochs)."""
import os

import numpy as np
import pytest

from oracle import ops
from oracle.base import AddrTable, Observed, counts_from_f64, fftshift2
from oracle.lsqml import Lsqml
from oracle.ptycho import Ptycho

HERE = os.path.dirname(os.path.abspath(__file__))
SHAPE, OBJ, NPROBE = (24, 24), (40, 40), 2


def golden(name):
    return dict(np.load(os.path.join(HERE, "golden", f"{name}.npz")))


def max_rel(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    return np.abs(a - b).max() / np.abs(b).max()


def stack(dims, rows, lead):
    return (rows[:, lead] + 1j * rows[:, lead + 1]).reshape(dims)


def change(a, b):
    d = (a - b).ravel()
    return np.stack([d.real, d.imag], axis=1).ravel()


def of_run(rows, run, lead):
    r = rows[rows[:, 0] == run]
    return np.stack([r[:, lead], r[:, lead + 1]], axis=1).ravel()


def near_case(g, c, pixel):
    """Positions from the golden corners (`corner = (OBJ − SHAPE)/2 + position/pixel`), the
    counts of case `c` and its free-space optics."""
    corners = g["corners"]
    ys = (corners[:, 1] - (OBJ[0] - SHAPE[0]) // 2) * pixel
    xs = (corners[:, 2] - (OBJ[1] - SHAPE[1]) // 2) * pixel
    rows = g["counts"][g["counts"][:, 0] == c[0]]
    counts = counts_from_f64(rows[:, 2:].reshape(len(corners), *SHAPE))
    w = ops.Wavefield(SHAPE, c[1], [pixel, pixel], c[3])
    optics = ops.Optics.free_space(w)
    kind = {"fourier": 0, "angular": 1, "fresnel": 2}[optics.propagator.kind]
    assert kind == int(c[4])
    obj = stack((1,) + OBJ, g["obj"], 2)
    probe = stack((NPROBE,) + SHAPE, g["probe"], 3)
    return corners, counts, ys, xs, optics, obj, probe


def test_rpie_matches_ptychi_near_field():
    """engine_rpie_near.rs:92-170: 3 propagators × batches 1/4/16 over 30 epochs."""
    g = golden("rpie_near")
    runs, trace = g["runs"], g["llk"]
    for r in runs:
        c = g["cases"][int(r[1])]
        corners, counts, ys, xs, optics, obj, probe = near_case(g, c, c[2])
        p = Ptycho(counts, ys, xs, optics, obj, probe)
        for f in range(len(corners)):
            v = p.addr.frame_views(f)[0]
            assert [v["oy"], v["ox"]] == [corners[f, 1], corners[f, 2]]
        o0, p0 = p.object.copy(), p.probe.copy()
        llks = [p.llk().poisson]
        p.rpie(int(r[3]), obj_step=r[4], probe_step=r[5], obj_alpha=r[6], probe_alpha=r[7],
               batch_size=int(r[2]), calc_llk=1, seed=7)
        llks += [h["poisson"] for h in p.history]
        want = trace[trace[:, 0] == r[0]][:, 2]
        assert max_rel(llks, want) < 1e-12, f"run {r[0]} LLK trace"
        assert max_rel(change(p.object, o0), of_run(g["run_obj"], r[0], 3)) < 1e-12
        assert max_rel(change(p.probe, p0), of_run(g["run_probe"], r[0], 4)) < 1e-12


def lsqml_state():
    g = golden("lsqml_near")
    corners = g["corners"]
    ys = corners[:, 1] - (OBJ[0] - SHAPE[0]) // 2
    xs = corners[:, 2] - (OBJ[1] - SHAPE[1]) // 2
    addr = AddrTable(ys, xs, [1.0, 1.0], SHAPE, OBJ, NPROBE, 1)
    for f in range(len(corners)):
        v = addr.frame_views(f)[0]
        assert [v["oy"], v["ox"]] == [corners[f, 1], corners[f, 2]]
    obj = stack((1,) + OBJ, g["obj"], 2)
    probe = stack((NPROBE,) + SHAPE, g["probe"], 3)
    cases = []
    for c in g["cases"]:
        w = ops.Wavefield(SHAPE, c[1], [c[2], c[2]], c[3])
        optics = ops.Optics.free_space(w)
        assert abs(optics.intensity_scale() - c[5]) <= 1e-15 * abs(c[5])
        rows = g["counts"][g["counts"][:, 0] == c[0]]
        obs = Observed(counts_from_f64(rows[:, 2:].reshape(len(corners), *SHAPE)))
        cases.append((optics, obs, c[6]))
    return g, addr, obj, probe, cases


def test_lsqml_forward_matches_ptychi():
    """engine_lsqml_near.rs:154-171: pty-chi's `y_pred` of frames 0..4."""
    g, addr, obj, probe, cases = lsqml_state()
    for r in g["icalc"]:
        optics, obs, _ = cases[int(r[0])]
        f = int(r[1])
        psi = optics.exit_forward(ops.obj_probe_to_psi(addr.frame_views(f), obj, probe,
                                                       optics.quad))
        got = (np.abs(psi) ** 2).sum(axis=0)
        want = fftshift2(r[2:].reshape(SHAPE))
        assert max_rel(got, want) < 1e-14


def assert_step(st, rows, col):
    assert st["frames"] == [int(v) for v in rows[:, col]]
    assert max_rel(st["a_far"], rows[:, col + 1]) < 1e-13
    assert max_rel(st["a_obj"], rows[:, col + 2]) < 1e-12
    assert max_rel(st["a_probe"], rows[:, col + 3]) < 1e-12


def test_lsqml_step_matches_ptychi():
    """engine_lsqml_near.rs:300-340: one step on frames 0..8, every case."""
    g, addr, obj, probe, cases = lsqml_state()
    views = addr.views[:8 * addr.nmode]
    for k, (optics, obs, _) in enumerate(cases):
        run = Lsqml(8, "poisson", 0)
        run.preconditioner = ops.illumination(addr.views, obj.shape, probe)
        o, p, st = run.step(views, obs, optics, obj, probe)
        assert_step(st, g["step_steps"][g["step_steps"][:, 0] == k], 1)
        assert max_rel(change(o, obj), of_run(g["step_obj"], k, 3)) < 1e-12
        assert max_rel(change(p, probe), of_run(g["step_probe"], k, 4)) < 1e-12


def test_lsqml_epochs_match_ptychi():
    """engine_lsqml_near.rs:450-510: batches of 8 (seed 7) over the saved epochs."""
    g, addr, obj0, probe0, cases = lsqml_state()
    steps, trace = g["epochs_steps"], g["llk"]
    for k, (optics, obs, truth) in enumerate(cases):
        obj, probe = obj0.copy(), probe0.copy()
        run = Lsqml(8, "poisson", 7)
        want = trace[trace[:, 0] == k]
        rows = steps[steps[:, 0] == k]
        llks = [run.llk(addr, obs, optics, obj, probe).poisson]
        nxt = 0
        for e in range(len(want) - 1):
            obj, probe, sts = run.epoch(addr, obs, optics, obj, probe)
            for st in sts:
                w = rows[nxt:nxt + len(st["frames"])]
                nxt += len(st["frames"])
                assert (w[:, 1] == e).all()
                assert_step(st, w, 2)
            llks.append(run.llk(addr, obs, optics, obj, probe).poisson)
        assert nxt == len(rows)
        assert max_rel(llks, want[:, 2]) < 1e-12
        assert max_rel(change(obj, obj0), of_run(g["epochs_obj"], k, 3)) < 1e-12
        assert max_rel(change(probe, probe0), of_run(g["epochs_probe"], k, 4)) < 1e-12


def pynx_near_start(g):
    """engine_pynx_near.rs:51-96: the case's angular-spectrum optics, positions from the golden
    corners, the counts, the start object and the two-mode probe."""
    c = g["case"][0]
    pixel = c[1]
    corners = g["corners"]
    ys = (corners[:, 1] - (OBJ[0] - SHAPE[0]) // 2) * pixel
    xs = (corners[:, 2] - (OBJ[1] - SHAPE[1]) // 2) * pixel
    counts = counts_from_f64(g["counts"][:, 1:].reshape(len(corners), *SHAPE))
    optics = ops.Optics.free_space(ops.Wavefield(SHAPE, c[0], [pixel, pixel], c[2]))
    assert optics.propagator.kind == "angular"
    obj = stack((1,) + OBJ, g["obj"], 2)
    probe = stack((NPROBE,) + SHAPE, g["probe"], 3)
    return Ptycho(counts, ys, xs, optics, obj, probe)


def unit(a):
    """`a / Σ|a|` as re, im pairs: DM and RAAR balance `Σ|O|` and `Σ|P|` after each recorded
    cycle, PyNX's cpu_operator does not, and the updates commute with that balance
    (engine_pynx_near.rs:43-49)."""
    a = np.ravel(a) / np.abs(a).sum()
    return np.stack([a.real, a.imag], 1)


@pytest.mark.parametrize("algorithm", [0, 1, 2], ids=["ap", "dm", "raar"])
def test_ap_dm_raar_match_pynx_near_field(algorithm):
    """engine_pynx_near.rs:98-205, the exact-kernel AP, DM and RAAR runs (runs 4-6), 30 cycles
    recording every one: every LLK column per record (DM and RAAR from their second record on,
    then the final LLK, as PyNX records after the update) and the final object and probe (DM's
    and RAAR's over their `Σ|·|`) to the reference's 5e-12."""
    g = golden("pynx_near")
    run = g["runs"][4 + algorithm]
    assert run[1] == 1 and run[2] == algorithm
    p = pynx_near_start(g)
    cycles = int(run[3])
    if algorithm == 0:
        p.ap(cycles, probe_inertia=0.001, calc_llk=1, zero_phase_ramp=False)
    elif algorithm == 1:
        p.dm(cycles, calc_llk=1, zero_phase_ramp=False)
    else:
        p.raar(cycles, calc_llk=1, zero_phase_ramp=False)
    cols = ["poisson", "gaussian", "euclidian", "nb_photons_calc"]
    got = [[h[k] for k in cols] for h in p.history]
    if algorithm > 0:
        got = got[1:] + [[p.llk().as_dict()[k] for k in cols]]
    got = np.asarray(got)
    want = g["llk"][g["llk"][:, 0] == run[0]][:, 2:6]
    assert got.shape == want.shape
    err = (np.abs(got - want) / np.abs(want)).max()
    assert err < 5e-12, err
    for arr, rows, lead in [(p.object, g["run_obj"], 3), (p.probe, g["run_probe"], 4)]:
        r = rows[rows[:, 0] == run[0]]
        want = r[:, lead] + 1j * r[:, lead + 1]
        if algorithm > 0:
            assert max_rel(unit(arr), unit(want)) < 5e-12
        else:
            assert max_rel(np.stack([arr.ravel().real, arr.ravel().imag], 1),
                           np.stack([want.real, want.imag], 1)) < 5e-12


def test_ml_matches_pynx_near_field():
    """engine_pynx_near.rs:107-205, the exact-kernel ML run (run 7): 10 AP cycles with probe
    inertia 0.001, then 30 ML cycles updating object and probe; every LLK column per record
    and the final arrays to the reference's 5e-12."""
    g = golden("pynx_near")
    c = g["case"][0]
    pixel = c[1]
    corners = g["corners"]
    ys = (corners[:, 1] - (OBJ[0] - SHAPE[0]) // 2) * pixel
    xs = (corners[:, 2] - (OBJ[1] - SHAPE[1]) // 2) * pixel
    counts = counts_from_f64(g["counts"][:, 1:].reshape(len(corners), *SHAPE))
    optics = ops.Optics.free_space(ops.Wavefield(SHAPE, c[0], [pixel, pixel], c[2]))
    assert optics.propagator.kind == "angular"
    obj = stack((1,) + OBJ, g["obj"], 2)
    probe = stack((NPROBE,) + SHAPE, g["probe"], 3)
    run = g["runs"][7]
    assert run[1] == 1 and run[2] == 3
    p = Ptycho(counts, ys, xs, optics, obj, probe)
    p.ap(10, probe_inertia=0.001, calc_llk=0, zero_phase_ramp=False)
    p.ml(int(run[3]), update_probe=True, calc_llk=1, zero_phase_ramp=False)
    cols = ["poisson", "gaussian", "euclidian", "nb_photons_calc"]
    got = [[h[k] for k in cols] for h in p.history][1:]
    got.append([p.llk().as_dict()[k] for k in cols])
    got = np.asarray(got)
    want = g["llk"][g["llk"][:, 0] == run[0]][:, 2:6]
    err = (np.abs(got - want) / np.abs(want)).max()
    assert err < 5e-12, err
    for arr, rows, lead in [(p.object, g["run_obj"], 3), (p.probe, g["run_probe"], 4)]:
        r = rows[rows[:, 0] == run[0]]
        want = r[:, lead] + 1j * r[:, lead + 1]
        got = arr.ravel()
        assert max_rel(np.stack([got.real, got.imag], 1), np.stack([want.real, want.imag], 1)) < 5e-12


def test_lsqml_step_with_positions_matches_ptychi():
    """engine_lsqml_near.rs:386-440 under PATCH: from the truth object, every frame moved by
    its offset and the positions refined, one step on frames 0..8 of each case the files hold:
    the step sizes, the object and probe changes, and the offset changes (1e-11)."""
    g, addr, obj0, probe, cases = lsqml_state()
    p = golden("lsqml_near_pos")
    start = stack((1,) + OBJ, p["start"], 2)
    views = addr.views[:8 * addr.nmode]
    checked = 0
    for k, (optics, obs, _) in enumerate(cases):
        rows = p["offsets"][p["offsets"][:, 0] == k]
        if len(rows) == 0:
            continue
        checked += 1
        d0, want = rows[:, 2:4], rows[:, 4:6]
        run = Lsqml(8, "poisson", 0, offsets=d0, refine=True)
        run.preconditioner = ops.illumination(addr.views, start.shape, probe)
        o, pr, st = run.step(views, obs, optics, start, probe)
        assert_step(st, p["steps"][p["steps"][:, 0] == k], 1)
        assert max_rel(change(o, start), of_run(p["obj"], k, 3)) < 1e-12
        assert max_rel(change(pr, probe), of_run(p["probe"], k, 4)) < 1e-12
        assert max_rel(run.offsets - d0, want - d0) < 1e-11
    assert checked == 2


NSLICE = 3


def multislice_state():
    """engine_lsqml_multislice.rs:63-145: three slices with unequal angular-spectrum gaps; case
    kind 0 is the far field of a geometry (its q on the last slice), 1 angular spectrum, 2 a
    Fresnel transform."""
    g = golden("lsqml_multislice")
    corners = g["corners"]
    ys = corners[:, 1] - (OBJ[0] - SHAPE[0]) // 2
    xs = corners[:, 2] - (OBJ[1] - SHAPE[1]) // 2
    addr = AddrTable(ys, xs, [1.0, 1.0], SHAPE, OBJ, NPROBE, 1)
    objs = [stack((1,) + OBJ, g["obj"][g["obj"][:, 0] == s], 3) for s in range(NSLICE)]
    probe = stack((NPROBE,) + SHAPE, g["probe"], 3)
    cases = []
    for c in g["cases"]:
        if c[4] == 0.0:
            lz = c[1] * c[3]
            optics = ops.Optics.far_field(c[1], c[3], lz / (SHAPE[0] * c[2]), list(SHAPE))
            pixel = optics.pixel
        else:
            pixel = [c[2], c[2]]
            optics = ops.Optics.free_space(ops.Wavefield(SHAPE, c[1], pixel, c[3]))
        gaps = [ops.Wavefield(SHAPE, c[1], pixel, d) for d in c[7:]]
        optics = optics.with_slices(gaps)
        assert abs(optics.intensity_scale() - c[5]) <= 1e-15 * abs(c[5])
        rows = g["counts"][g["counts"][:, 0] == c[0]]
        obs = Observed(counts_from_f64(rows[:, 2:].reshape(len(corners), *SHAPE)))
        cases.append((optics, obs, c[6]))
    return g, addr, objs, probe, cases


def multislice_changes(objs, objs0):
    return np.concatenate([change(o, o0) for o, o0 in zip(objs, objs0)])


def of_case(rows, k):
    r = rows[rows[:, 0] == k]
    return np.stack([r[:, 4], r[:, 5]], axis=1).ravel()


def assert_ms_step(st, rows, col):
    assert st["frames"] == [int(v) for v in rows[:, col]]
    assert max_rel(st["a_far"], rows[:, col + 1]) < 1e-13
    for i in range(NSLICE):
        assert max_rel(st["a_obj"][i], rows[:, col + 2 + i]) < 1e-12
    assert max_rel(st["a_probe"], rows[:, col + 2 + NSLICE]) < 1e-12


def test_multislice_forward_and_step_match_ptychi():
    """engine_lsqml_multislice.rs:163-181 and 343-372: pty-chi's y_pred through three slices,
    and one LSQML step on frames 0..8 with the joint slice-0 step sizes."""
    g, addr, objs, probe, cases = multislice_state()
    from oracle.lsqml import SliceWaves
    for r in g["icalc"]:
        optics, obs, _ = cases[int(r[0])]
        v = addr.frame_views(int(r[1]))
        w = SliceWaves(optics, v, objs, probe[v["probe"].astype(np.int64)])
        got = (np.abs(optics.exit_forward(w.psi)) ** 2).sum(axis=0)
        assert max_rel(got, fftshift2(r[2:].reshape(SHAPE))) < 1e-14
    views = addr.views[:8 * addr.nmode]
    for k, (optics, obs, _) in enumerate(cases):
        run = Lsqml(8, "poisson", 0)
        run.preconditioner = ops.illumination(addr.views, objs[0].shape, probe)
        o, pr, st = run.step(views, obs, optics, objs, probe)
        assert_ms_step(st, g["step_steps"][g["step_steps"][:, 0] == k], 1)
        assert max_rel(multislice_changes(o, objs), of_case(g["step_obj"], k)) < 1e-12
        assert max_rel(change(pr, probe), of_case(g["step_probe"], k)) < 1e-12


def test_multislice_epochs_match_ptychi():
    """engine_lsqml_multislice.rs:481-540: the epochs (seed 7), every step and the LLK trace."""
    g, addr, objs0, probe0, cases = multislice_state()
    steps, trace = g["epochs_steps"], g["llk"]
    for k, (optics, obs, truth) in enumerate(cases):
        objs, probe = list(objs0), probe0.copy()
        run = Lsqml(8, "poisson", 7)
        want = trace[trace[:, 0] == k]
        rows = steps[steps[:, 0] == k]
        llks = [run.llk(addr, obs, optics, objs, probe).poisson]
        nxt = 0
        for e in range(len(want) - 1):
            objs, probe, sts = run.epoch(addr, obs, optics, objs, probe)
            for st in sts:
                w = rows[nxt:nxt + len(st["frames"])]
                nxt += len(st["frames"])
                assert_ms_step(st, w, 2)
            llks.append(run.llk(addr, obs, optics, objs, probe).poisson)
        assert nxt == len(rows)
        assert max_rel(llks, want[:, 2]) < 1e-12
        assert max_rel(multislice_changes(objs, objs0), of_case(g["epochs_obj"], k)) < 1e-12
        assert max_rel(change(probe, probe0), of_case(g["epochs_probe"], k)) < 1e-12


def test_multislice_step_with_positions_matches_ptychi():
    """engine_lsqml_multislice.rs:374-458 (`step_with_positions_matches_ptychi`): one LSQML
    step on frames 0..8 through the three slices from `lsqml_multislice_pos.py`'s start, every
    frame moved by its offset under Patch and the offsets refined on the middle slice; the
    case whose exit has no plane phase (the only one the reference checks under Patch): the
    steps, the object and probe changes and the offset changes."""
    g, addr, _, probe, cases = multislice_state()
    p = golden("lsqml_multislice_pos")
    start = p["start"]
    objs = [stack((1,) + OBJ, start[start[:, 0] == s], 3) for s in range(NSLICE)]
    views = addr.views[:8 * addr.nmode]
    checked = 0
    for k, (optics, obs, _) in enumerate(cases):
        if not np.all(optics.quad == 1.0):
            continue
        checked += 1
        rows = p["offsets"][p["offsets"][:, 0] == k]
        d0, want = rows[:, 2:4], rows[:, 4:6]
        run = Lsqml(8, "poisson", 0, offsets=d0, refine=True)
        run.preconditioner = ops.illumination(addr.views, objs[0].shape, probe)
        o, pr, st = run.step(views, obs, optics, objs, probe)
        assert_ms_step(st, p["steps"][p["steps"][:, 0] == k], 1)
        assert max_rel(multislice_changes(o, objs), of_case(p["obj"], k)) < 1e-12
        assert max_rel(change(pr, probe), of_case(p["probe"], k)) < 1e-12
        assert max_rel(run.offsets - d0, want - d0) < 1e-11
    assert checked == 1
