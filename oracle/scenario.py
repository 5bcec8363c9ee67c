"""The reference's seeded far-field test scenario, rebuilt bit for bit where its golden files
need it (oracle restatement, test infrastructure only).

physwkim/ptyrs `tests/common/engine/scenario.rs:20-77` (`dm_scenario`): the known object and
multi-mode probe of `base/sim.rs:53-127`, a Fermat scan (`base/sim.rs:30-45`, positions
rounded to f32), the far-field intensities of `engine/sim.rs:71-123` scaled to the photons per
frame, Poisson counts drawn by `base/sim.rs:143-175` (`oracle.rng`), and the start: the
object's phases from a xorshift stream, the probe with a quadratic phase.
"""
import math

import numpy as np

from . import ops
from .base import AddrTable, pixel_size_object, pynx_preprocess, required_obj_shape
from .rng import sample_counts

WAVELENGTH, DISTANCE, DETECTOR_PIXEL = 1.5e-10, 1.0, 75e-6


def _smoothstep(e0, e1, v):
    t = np.clip((v - e0) / (e1 - e0), 0.0, 1.0)
    return t * t * (3.0 - 2.0 * t)


def sim_object(shape):
    """`base::sim::object` (base/sim.rs:53-81): `[1, ny, nx]`."""
    ny, nx = shape
    s = min(ny, nx) / 2.0
    iy, ix = np.mgrid[:ny, :nx].astype(np.float64)
    u, v = (ix - nx / 2.0) / s, (iy - ny / 2.0) / s

    def blob(cu, cv, w):
        return np.exp(-((u - cu) ** 2 + (v - cv) ** 2) / (2.0 * w * w))

    r = np.hypot(u, v)
    star = (0.5 * (1.0 + np.tanh(3.0 * np.cos(12.0 * np.arctan2(v, u))))
            * _smoothstep(0.08, 0.12, r) * (1.0 - _smoothstep(0.55, 0.6, r)))
    phase = star + 0.6 * blob(0.55, -0.45, 0.12) - 0.4 * blob(-0.5, 0.5, 0.1)
    amp = 0.95 - 0.3 * blob(-0.45, -0.55, 0.15) - 0.15 * star
    return (amp * np.cos(phase) + 1j * amp * np.sin(phase))[None]


def _hermite(n, t):
    return np.ones_like(t) if n == 0 else (2.0 * t if n == 1 else 4.0 * t * t - 2.0)


def sim_probe(frame, nmode):
    """`base::sim::probe` (base/sim.rs:94-127): `[nmode, ny, nx]`, mode k of power 4^-k."""
    orders = [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (0, 2)]
    ny, nx = frame
    sigma = min(ny, nx) / 12.0
    weights = [0.25 ** k for k in range(nmode)]
    wsum = sum(weights)
    iy, ix = np.mgrid[:ny, :nx].astype(np.float64)
    u, v = (ix - nx / 2.0) / sigma, (iy - ny / 2.0) / sigma
    r2 = u * u + v * v
    out = []
    for k, (a, b) in enumerate(orders[:nmode]):
        amp = _hermite(a, u) * _hermite(b, v) * np.exp(-r2 / 2.0)
        ph = 1.5 * r2 + 0.3 * k
        plane = amp * np.cos(ph) + 1j * amp * np.sin(ph)
        norm = math.sqrt(float((np.abs(plane) ** 2).sum()))
        out.append(plane * (math.sqrt(weights[k] / wsum) / norm))
    return np.array(out)


def fermat(n, step):
    """`base::sim::fermat` (base/sim.rs:30-45): `(y, x)` in metres."""
    golden = math.pi * (3.0 - math.sqrt(5.0))
    c = step / math.sqrt(math.pi)
    y, x = [], []
    for k in range(n):
        r, t = c * math.sqrt(k), k * golden
        y.append(r * math.sin(t))
        x.append(r * math.cos(t))
    return np.array(y), np.array(x)


def dm_scenario(frame, npos, nprobe, photons, step, seed=1):
    """`dm_scenario(frame, npos, nprobe, photons, step)`: a dict with `counts` (float64, detector
    order), `y`, `x` (metres), the start `object` and `probe`, the `truth` object and probe, the
    object `pixel` and the far-field `optics`."""
    shape = [frame, frame]
    pixel = pixel_size_object(WAVELENGTH, DISTANCE, shape, DETECTOR_PIXEL)
    fy, fx = fermat(npos, step * pixel[1])
    y = fy.astype(np.float32).astype(np.float64)
    x = fx.astype(np.float32).astype(np.float64)
    py, px = pynx_preprocess(y, x, pixel)
    obj_shape = required_obj_shape(py, px, pixel, shape, 16)
    truth = sim_object(obj_shape)
    truth_probe = sim_probe(shape, nprobe)
    optics = ops.Optics.far_field(WAVELENGTH, DISTANCE, DETECTOR_PIXEL, shape)
    addr = AddrTable(py, px, pixel, shape, list(obj_shape), nprobe, 1)
    psi = ops.fft2(ops.obj_probe_to_psi(addr.views, truth, truth_probe, optics.quad))
    inten = ops.icalc_of(psi, addr.nmode)                       # FFT order per frame
    inten = np.fft.fftshift(inten, axes=(-2, -1))               # detector order
    total = 0.0
    for v in inten.ravel():
        total += float(v)
    inten = inten * (photons / (total / addr.nframe))
    counts = sample_counts(inten, seed)
    # the start: phases from a xorshift64 stream, the probe under a quadratic phase
    state = 0x9E3779B97F4A7C15
    m64 = (1 << 64) - 1
    ph = np.empty(truth.size)
    for i in range(truth.size):
        state ^= (state << 13) & m64
        state ^= state >> 7
        state ^= (state << 17) & m64
        ph[i] = (state >> 11) / float(1 << 53) - 0.5
    start = (np.cos(ph) + 1j * np.sin(ph)).reshape(truth.shape)
    sigma = frame / 12.0
    i = np.arange(frame * frame)
    u = ((i % frame) - frame / 2.0) / sigma
    w = ((i // frame) - frame / 2.0) / sigma
    q = -0.5 * (u * u + w * w)
    probe = truth_probe * (np.cos(q) + 1j * np.sin(q)).reshape(shape)[None]
    return dict(counts=counts, y=y, x=x, object=start, probe=probe, truth=truth,
                truth_probe=truth_probe, pixel=pixel, optics=optics, frame=frame)
