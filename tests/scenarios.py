"""Small seeded far-field scans for the parity tests: the oracle and the CUDA path read the same
counts, positions and start arrays."""
import numpy as np

from oracle import ops
from oracle.ptycho import Ptycho
from ptyrs_b200 import sim


def far_field(n, nmode, nframe, side, photons=1e5, seed=0, masked=False, step=None):
    """Counts `[nframe, n, n]` (float32, negative masked), positions in metres and a perturbed
    start (object of ones, probe scaled and dephased) of a Fermat scan of a smooth object."""
    rng = np.random.default_rng(seed)
    truth = sim.smooth_object(side, seed + 1)
    powers = [0.8, 0.15, 0.05, 0.02][:nmode]
    probe = sim.hermite_probe(n, n / 4.0, powers) if nmode > 1 else (
        sim.aperture_probe(n, n / 4.0)[None] * 30.0)
    step = step or n / 8.0
    pos = sim.fermat_positions(nframe, step) + rng.uniform(-0.5, 0.5, (nframe, 2))
    corner = sim.corners(pos, n, side)
    counts = sim.far_field_counts(truth, probe, corner, photons, seed + 2)
    if masked:
        counts[:, n // 2 - 1:n // 2 + 1, :3] = -1.0
        counts[rng.uniform(size=counts.shape) < 0.002] = -1.0
    px = sim.object_pixel(n)
    # the start: the probe scaled to the data's photons through an object of ones, then
    # perturbed in modulus and phase
    probe = probe * np.sqrt(photons / (np.abs(probe) ** 2).sum())
    start_probe = probe * 0.9 * np.exp(0.2j)
    start_obj = np.ones((1, side, side), np.complex128)
    return dict(counts=counts, y=pos[:, 0] * px, x=pos[:, 1] * px, object=start_obj,
                probe=start_probe, corners=corner, n=n, truth=truth)


def oracle_state(s):
    optics = ops.Optics.far_field(sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL,
                                  [s["n"], s["n"]])
    return Ptycho(s["counts"], s["y"], s["x"], optics, s["object"], s["probe"])


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
