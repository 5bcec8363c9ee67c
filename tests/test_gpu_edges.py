"""Edge cases of the CUDA path against the f64 oracle, as the reference's own tests probe them
(engine_gpu.rs, obs.rs, addr.rs): a scan of one frame; a fully masked frame and a frame of zero
counts among the others; u16 counts (65535 masked) against the same values in float32, bit for
bit; calls of zero epochs or cycles; windows on the object's first and last pixels."""
import numpy as np
import pytest

from oracle.lsqml import Lsqml
from ptyrs_b200 import GpuPtycho, Scan, sim
from scenarios import far_field, oracle_state, rel_l2

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-4


def gpu_of(s, counts=None):
    scan = Scan(s["counts"] if counts is None else counts, s["y"], s["x"], sim.WAVELENGTH,
                sim.DISTANCE, sim.DETECTOR_PIXEL)
    return GpuPtycho(scan, s["object"], s["probe"])


def run_both(s, algorithm):
    """The algorithm's two epochs or cycles on the oracle and the GPU from `s`; returns the
    oracle state and the GPU's object, probe and LLK records."""
    cpu = oracle_state(s)
    if algorithm == "lsqml":
        run = Lsqml(4, "poisson", 7)
        for _ in range(2):
            cpu.object, cpu.probe, _ = run.epoch(cpu.addr, cpu.obs, cpu.optics, cpu.object,
                                                 cpu.probe)
    elif algorithm == "rpie":
        cpu.rpie(2, batch_size=4, calc_llk=1, seed=7)
    elif algorithm == "ml":
        cpu.ml(2, update_probe=True, calc_llk=1, zero_phase_ramp=False)
    else:
        getattr(cpu, algorithm)(2, calc_llk=1, zero_phase_ramp=False)
    with gpu_of(s) as g:
        if algorithm == "lsqml":
            g.lsqml(2, batch_size=4, cost="poisson", seed=7)
        elif algorithm == "rpie":
            g.rpie(2, batch_size=4, calc_llk=1, seed=7)
        elif algorithm == "ml":
            g.ml(2, update_probe=True, calc_llk=1, zero_phase_ramp=False)
        else:
            getattr(g, algorithm)(2, calc_llk=1, zero_phase_ramp=False)
        return cpu, (g.object(), g.probe(), g.history()["poisson"])


def assert_close(cpu, got):
    o, p, h = got
    assert rel_l2(o, cpu.object) < RUN_TOL
    assert rel_l2(p, cpu.probe) < RUN_TOL
    want = np.array([r["poisson"] for r in cpu.history])
    assert len(h) == len(want)
    if len(want):
        assert np.abs(h - want).max() <= 3e-4 * np.abs(want).max()


ALGORITHMS = ["rpie", "lsqml", "ml", "dm", "raar", "ap"]


@pytest.mark.parametrize("algorithm", ALGORITHMS)
def test_one_frame(algorithm):
    s = far_field(64, 2, 1, 96, seed=4)
    assert_close(*run_both(s, algorithm))


@pytest.mark.parametrize("algorithm", ALGORITHMS)
def test_masked_and_empty_frames(algorithm):
    """Frame 0 masked everywhere and frame 1 of zero counts: neither enters the LLK's pixel
    count, the projections keep the masked field, the Poisson terms of zero counts hold."""
    s = far_field(64, 2, 12, 160, masked=True, seed=6)
    s["counts"][0] = -1.0
    s["counts"][1] = 0.0
    assert_close(*run_both(s, algorithm))


def test_u16_counts_match_float32():
    s = far_field(64, 2, 12, 160, masked=True, seed=7)
    f32 = np.minimum(s["counts"], 65534.0)
    u16 = np.where(f32 < 0, 65535, f32).astype(np.uint16)
    outs = []
    for counts in (f32, u16):
        with gpu_of(s, counts) as g:
            g.rpie(1, batch_size=4, seed=3)
            g.lsqml(1, batch_size=4, seed=3)
            g.ml(1, update_probe=True, zero_phase_ramp=False)
            g.dm(1, zero_phase_ramp=False)
            outs.append((g.object(), g.probe(), g.llk()["poisson"]))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_zero_epochs_and_cycles_change_nothing():
    s = far_field(64, 1, 12, 160, seed=8)
    with gpu_of(s) as g:
        o, p = g.object(), g.probe()
        g.rpie(0, batch_size=4)
        g.lsqml(0, batch_size=4)
        for run in (g.ap, g.dm, g.raar):
            run(0, calc_llk=1, zero_phase_ramp=False)
        assert np.array_equal(g.object(), o) and np.array_equal(g.probe(), p)
        assert len(g.history()["poisson"]) == 0 and g.cycle() == 0


@pytest.mark.parametrize("algorithm", ["rpie", "dm"])
def test_windows_on_the_object_edges(algorithm):
    """Frames whose windows start at the object's first row and column and end at its last
    (PyNX's centring puts ±(side − n)/2 pixels at the edges)."""
    n, side = 64, 192
    base = far_field(n, 2, 3, side, seed=9)
    d = (side - n) // 2
    pos = np.array([[-d, -d], [0.0, 0.0], [d, d]], np.float64)
    corner = sim.corners(pos, n, side)
    assert corner.min() == 0 and corner.max() == side - n
    probe = sim.hermite_probe(n, n / 4.0, [0.8, 0.2])
    counts = sim.far_field_counts(base["truth"], probe, corner, 1e5, 10)
    px = sim.object_pixel(n)
    s = dict(base, counts=counts, y=pos[:, 0] * px, x=pos[:, 1] * px, corners=corner)
    with gpu_of(s) as g:
        assert (g.corners() == corner).all()
    assert_close(*run_both(s, algorithm))
