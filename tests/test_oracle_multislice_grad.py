"""The oracle's adjoint of the multislice model (three slices, far-field exit, two
angular-spectrum gaps) against central differences of its float64 Poisson sum: every slice's
gradient and the probe's, in the 2·∂L/∂X* packing."""
import numpy as np

from oracle import ops
from oracle.base import fftshift2
from oracle.lsqml import Lsqml, SliceWaves, multislice_grads
from oracle.ptycho import Ptycho
from ptyrs_b200 import sim


def scene(n=32, side=96, nframe=12, gaps=(2e-6, 3e-6)):
    rng = np.random.default_rng(4)
    truth = [sim.smooth_object(side, 5), sim.smooth_object(side, 6, np.pi / 5),
             sim.smooth_object(side, 7, np.pi / 7)]
    probe = sim.hermite_probe(n, n / 4.0, [0.8, 0.2])
    probe = probe * np.sqrt(1e5 / (np.abs(probe) ** 2).sum())
    pos = sim.fermat_positions(nframe, n / 8.0) + rng.uniform(-0.5, 0.5, (nframe, 2))
    px = sim.object_pixel(n)
    optics = ops.Optics.far_field(sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL, [n, n])
    optics = optics.with_slices([ops.Wavefield([n, n], sim.WAVELENGTH, optics.pixel, d)
                                 for d in gaps])
    y, x = pos[:, 0] * px, pos[:, 1] * px
    gen = Ptycho(np.zeros((nframe, n, n), np.float32), y, x, optics, truth[0], probe)
    waves = SliceWaves(optics, gen.addr.views, truth, probe[gen.addr.views["probe"]])
    inten = (np.abs(optics.exit_forward(waves.psi)) ** 2).reshape(nframe, 2, n, n).sum(axis=1)
    counts = rng.poisson(fftshift2(inten)).astype(np.float32)
    p = Ptycho(counts, y, x, optics, truth[0], probe)
    start = [t * 0.95 * np.exp(0.05j) for t in truth]
    return p, start, probe * 0.9 * np.exp(0.2j)


def test_multislice_gradients_match_central_differences():
    p, objs, probe = scene()
    loss, d_objs, d_probe = multislice_grads(p.addr, p.obs, p.optics, objs, probe)
    assert loss == Lsqml(4).llk(p.addr, p.obs, p.optics, objs, probe).poisson * p.obs.nb_obs

    def f(objs_, probe_):
        return multislice_grads(p.addr, p.obs, p.optics, objs_, probe_)[0]

    h = 1e-6
    picks = [(0, (0, 40, 40)), (1, (0, 45, 52)), (2, (0, 38, 47))]
    for s, idx in picks:
        for unit in (1.0, 1j):
            up = [o.copy() for o in objs]
            dn = [o.copy() for o in objs]
            up[s][idx] += h * unit
            dn[s][idx] -= h * unit
            fd = (f(up, probe) - f(dn, probe)) / (2 * h)
            an = d_objs[s][idx].real if unit == 1.0 else d_objs[s][idx].imag
            assert abs(fd - an) < 1e-5 * max(abs(an), 1e-3 * np.abs(d_objs[s]).max()), (s, unit)
    for idx in [(0, 16, 16), (1, 12, 19)]:
        for unit in (1.0, 1j):
            pu, pd = probe.copy(), probe.copy()
            pu[idx] += h * unit
            pd[idx] -= h * unit
            fd = (f(objs, pu) - f(objs, pd)) / (2 * h)
            an = d_probe[idx].real if unit == 1.0 else d_probe[idx].imag
            assert abs(fd - an) < 1e-5 * max(abs(an), 1e-3 * np.abs(d_probe).max()), (idx, unit)
