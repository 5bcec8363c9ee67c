"""Seeded synthetic scans of the shapes the benchmarks and tests use: smooth-noise objects,
defocused-aperture probes (with Hermite-Gauss modes), raster / Fermat scans and Poisson
far-field counts, all in numpy float64 (data generation, not part of the reconstruction path).

The far-field forward model here is the reference's (`obj_probe_to_psi` then the unitary FFT,
physwkim/ptyrs engine/ops.rs:47-71, engine/fft.rs:155-234) on the integer windows that PyNX's
position convention gives (base/addr.rs:123-127): positions are centred on their mean and the
window corner is `round_half_even((nobj − n)//2 + position/pixel)`.
"""
import numpy as np
from scipy.ndimage import gaussian_filter

WAVELENGTH, DISTANCE, DETECTOR_PIXEL = 1.5e-10, 1.0, 75e-6
GOLDEN_ANGLE = np.pi * (3.0 - np.sqrt(5.0))


def object_pixel(n):
    """Object pixel in metres of an n×n far-field frame at the default geometry."""
    return WAVELENGTH * DISTANCE / (n * DETECTOR_PIXEL)


def smooth_object(side, seed, phase_scale=np.pi / 2):
    """`amp = 1 − 0.2·g`, `phase = phase_scale·g`, `g` uniform noise smoothed by a σ = 3 px
    Gaussian (periodic) and normalised to [0, 1]; `[1, side, side]` complex128."""
    rng = np.random.default_rng(seed)
    g = gaussian_filter(rng.uniform(size=(side, side)), 3.0, mode="wrap")
    g = (g - g.min()) / (g.max() - g.min())
    return ((1.0 - 0.2 * g) * np.exp(1j * phase_scale * g))[None]


def aperture_probe(n, radius, edge_phase=2.0):
    """A circular aperture of `radius` px with a quadratic defocus phase reaching `edge_phase`
    rad at the edge (slightly softened edge), `[n, n]` complex128."""
    y, x = np.mgrid[:n, :n] - n / 2.0
    r = np.hypot(y, x)
    amp = np.clip(radius + 0.5 - r, 0.0, 1.0)
    return amp * np.exp(1j * edge_phase * (r / radius) ** 2)


def hermite_probe(n, radius, powers, edge_phase=2.0):
    """Incoherent probe modes: the defocused aperture times Hermite-Gauss factors of orders
    (0,0), (1,0), (0,1), (1,1), … of width radius/2, mode k scaled to power `powers[k]` of a
    total of 1e4 (arbitrary units), `[len(powers), n, n]`."""
    base = aperture_probe(n, radius, edge_phase)
    y, x = (np.mgrid[:n, :n] - n / 2.0) / (radius / 2.0)
    herm = [lambda t: np.ones_like(t), lambda t: 2 * t, lambda t: 4 * t * t - 2]
    orders = [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (0, 2)]
    modes = []
    for k, p in enumerate(powers):
        a, b = orders[k]
        m = base * herm[a](x) * herm[b](y) * np.exp(-(x * x + y * y) / 4.0)
        if k == 0:
            m = base
        modes.append(m * np.sqrt(p * 1e4) / np.linalg.norm(m))
    return np.array(modes)


def raster_positions(ny, nx, step, jitter, seed):
    """`ny × nx` raster of `step` px with uniform ±`jitter` px noise, in pixels `[P, 2]`."""
    rng = np.random.default_rng(seed)
    gy, gx = np.mgrid[:ny, :nx] * float(step)
    p = np.stack([gy.ravel(), gx.ravel()], 1)
    return p + rng.uniform(-jitter, jitter, size=p.shape)


def fermat_positions(count, step):
    """Fermat spiral of `count` points with about `step` px between neighbours, `[P, 2]`."""
    k = np.arange(count, dtype=np.float64)
    c = step / np.sqrt(np.pi)
    r, t = c * np.sqrt(k), k * GOLDEN_ANGLE
    return np.stack([r * np.sin(t), r * np.cos(t)], 1)


def corners(pos_px, n, nobj):
    """Window corners `[P, 2]` of positions in pixels under PyNX's convention (centred on the
    mean, rounded half to even, relative to the object centre)."""
    p = pos_px - pos_px.mean(axis=0)
    c = np.round((nobj - n) // 2 + p).astype(np.int64)
    if (c < 0).any() or (c > nobj - n).any():
        raise ValueError("a window leaves the object")
    return c


def far_field_counts(obj, probe, corner, photons, seed, chunk=64):
    """Poisson counts `[P, n, n]` (float32, detector order: zero frequency at the centre) of
    `Σ_modes |FFT_ortho(P·O_window)|²`, scaled so the mean pattern holds `photons`."""
    n = probe.shape[-1]
    P = len(corner)
    inten = np.empty((P, n, n), np.float64)
    for s in range(0, P, chunk):
        cs = corner[s:s + chunk]
        win = np.stack([obj[0, y:y + n, x:x + n] for y, x in cs])
        psi = probe[None] * win[:, None]
        far = np.fft.fft2(psi, norm="ortho")
        inten[s:s + chunk] = np.fft.fftshift((np.abs(far) ** 2).sum(axis=1), axes=(-2, -1))
    inten *= photons / inten.sum(axis=(1, 2)).mean()
    rng = np.random.default_rng(seed)
    return rng.poisson(inten).astype(np.float32)


def far_field_counts_gpu(obj, probe, corner, offsets, photons, seed, chunk=128,
                         device=None):
    """`far_field_counts` on a CUDA device with torch (data generation only), each frame's
    probe modes moved by its sub-pixel offset `offsets[f]` (dy, dx px) on the periodic frame
    grid before the window multiplies them: the Patch model of the position feature. Counts
    `[P, n, n]` float32, detector order, Poisson-sampled from the seed."""
    import torch
    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    n = probe.shape[-1]
    P = len(corner)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    o = torch.as_tensor(obj[0], dtype=torch.complex64, device=device)
    pr = torch.as_tensor(probe, dtype=torch.complex64, device=device)
    spec = torch.fft.fft2(pr)
    f = torch.fft.fftfreq(n, device=device, dtype=torch.float64)
    d = torch.as_tensor(offsets, dtype=torch.float64, device=device)
    iy = torch.arange(n, device=device)
    inten = torch.empty((P, n, n), dtype=torch.float32, device=device)
    for s0 in range(0, P, chunk):
        cs = torch.as_tensor(corner[s0:s0 + chunk], device=device)
        m = len(cs)
        rows = (cs[:, 0, None] + iy[None]).reshape(m, n, 1)
        cols = (cs[:, 1, None] + iy[None]).reshape(m, 1, n)
        win = o[rows, cols]
        ph = -2.0 * np.pi * (f[None, :, None] * d[s0:s0 + m, 0, None, None]
                             + f[None, None, :] * d[s0:s0 + m, 1, None, None])
        ramp = torch.polar(torch.ones_like(ph), ph).to(torch.complex64)
        moved = torch.fft.ifft2(spec[None] * ramp[:, None])
        far = torch.fft.fft2(moved * win[:, None], norm="ortho")
        inten[s0:s0 + m] = torch.fft.fftshift((far.abs() ** 2).sum(dim=1), dim=(-2, -1))
    inten *= photons / inten.sum(dim=(1, 2)).mean()
    counts = torch.poisson(inten, generator=gen)
    return counts.cpu().numpy()


def multislice_counts_gpu(slices, probe, corner, gaps, wavelength, pixel, photons, seed,
                          chunk=64, device=None):
    """Poisson counts of a multislice object (data generation only, torch): per frame and probe
    mode the wave crosses the slices, `ψ ← O_s[win]·ψ`, with an angular-spectrum propagation
    `exp(2πi·z·√(1/λ² − |f|²))` (evanescent frequencies dropped) over each gap `z` between
    them; the far field of the last product, summed over the modes. Counts `[P, n, n]` float32,
    detector order, scaled so the mean pattern holds `photons`."""
    import torch
    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    n = probe.shape[-1]
    P = len(corner)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    o = torch.as_tensor(np.concatenate(slices), dtype=torch.complex64, device=device)
    pr = torch.as_tensor(probe, dtype=torch.complex64, device=device)
    f = torch.fft.fftfreq(n, d=pixel, device=device, dtype=torch.float64)
    f2 = f[:, None] ** 2 + f[None, :] ** 2
    arg = 1.0 / wavelength ** 2 - f2
    prop = []
    for z in gaps:
        ph = 2.0 * np.pi * z * torch.sqrt(torch.clamp(arg, min=0.0))
        h = torch.polar((arg > 0).to(torch.float64), ph).to(torch.complex64)
        prop.append(h)
    iy = torch.arange(n, device=device)
    inten = torch.empty((P, n, n), dtype=torch.float32, device=device)
    for s0 in range(0, P, chunk):
        cs = torch.as_tensor(corner[s0:s0 + chunk], device=device)
        m = len(cs)
        rows = (cs[:, 0, None] + iy[None]).reshape(m, n, 1)
        cols = (cs[:, 1, None] + iy[None]).reshape(m, 1, n)
        psi = pr[None].expand(m, -1, -1, -1)
        for s in range(o.shape[0]):
            psi = psi * o[s][rows, cols][:, None]
            if s < len(prop):
                psi = torch.fft.ifft2(torch.fft.fft2(psi) * prop[s])
        far = torch.fft.fft2(psi, norm="ortho")
        inten[s0:s0 + m] = torch.fft.fftshift((far.abs() ** 2).sum(dim=1), dim=(-2, -1))
    inten *= photons / inten.sum(dim=(1, 2)).mean()
    counts = torch.poisson(inten, generator=gen)
    return counts.cpu().numpy()


def make_batch(count=32, seed=0, scale=1.0, sides=(64, 96, 128, 192, 256)):
    """`count` independent seeded scans of uneven sizes (the batched configuration, on the frame
    sides the engine has kernels for): per scan a side drawn from `sides`, an object 4–8 times
    the side, 500–5000 Fermat positions (times `scale`) at a step that keeps the scan inside the
    object (at most a quarter of the side), log-uniform 1e4–1e7 photons, the defocused aperture
    probe (one mode); counts made on the CUDA device. Returns a list of `make_scan`-style
    dicts."""
    rng = np.random.default_rng(seed + 100)
    out = []
    for i in range(count):
        n = int(rng.choice(sides))
        side = int(n * rng.uniform(4.0, 8.0))
        npos = max(2, int(rng.uniform(500, 5000) * scale))
        photons = 10.0 ** rng.uniform(4.0, 7.0)
        step = min(n / 4.0, (side - n - 8) * np.sqrt(np.pi) / (2.0 * np.sqrt(npos)))
        pos = fermat_positions(npos, step)
        truth = smooth_object(side, seed + 1000 + i)
        probe = aperture_probe(n, n / 4.0)[None]
        c = corners(pos, n, side)
        counts = far_field_counts_gpu(truth, probe, c, np.zeros((npos, 2)), photons,
                                      seed + 2000 + i)
        px = object_pixel(n)
        out.append(dict(counts=counts, y=pos[:, 0] * px, x=pos[:, 1] * px,
                        object=np.ones_like(truth),
                        probe=probe * np.sqrt(photons / (np.abs(probe) ** 2).sum()),
                        truth=truth, corners=c, n=n, side=side, wavelength=WAVELENGTH,
                        distance=DISTANCE, detector_pixel=DETECTOR_PIXEL,
                        true_offsets=np.zeros((npos, 2)), photons=photons))
    return out


def opr_start(probe, nframe, k=2, seed=3):
    """A seeded start of pty-chi's OPR probe variation of mode 0: `k` smooth eigenmodes at the
    main mode's scale (the mode times smoothed noise), weights uniform in ±0.1 per frame and
    main-mode weights 1; `(eigenmodes [k, ny, nx], weights [nframe, k], intensity [nframe])`."""
    rng = np.random.default_rng(seed)
    p0 = np.asarray(probe)[0]
    scale = np.sqrt((np.abs(p0) ** 2).mean())
    u = []
    for i in range(k):
        g = smooth_object(p0.shape[-1], seed + i)[0] - 1.0
        u.append(p0 * g * scale / np.sqrt((np.abs(p0 * g) ** 2).mean()))
    return np.array(u), rng.uniform(-0.1, 0.1, (nframe, k)), np.ones(nframe)


def make_scan(kind, seed=0, scale=1.0, device=None):
    """Seeded synthetic inputs of a benchmark configuration: returns a dict with counts
    (float32), y, x (metres), object start, probe start, truth object and sizes.

    kind "rpie64": 256² object, 64² aperture probe, 20×20 raster of 8 px ±1 px, 1e5 photons.
    kind "lsqml128": 1024² object, 128² probe with 3 modes (0.8/0.15/0.05), Fermat 4096 at
    6 px, 1e6 photons. kind "ml256": 2048² object, 256² probe with 2 modes (0.8/0.2), Fermat
    10000 at 12 px, 1e7 photons, the frames taken at true positions off the nominal ones by
    seeded N(0, 1.5 px) offsets (`true_offsets`; the solver is given the nominal positions),
    counts generated on the CUDA device (`device`: "cpu" makes them with torch on the host,
    the same counts on every machine of this image). `scale` < 1 keeps that fraction of the
    positions (the same first ones) for small cases. kind "fermat256": 1280² object, 256² probe with 2 modes
    (0.8/0.2), Fermat 4096 at 12 px, 1e7 photons, counts on the CUDA device (the scan of the
    AP / DM / RAAR workloads). kind "ms128": three slices of 1536² (phase scale π/4, independent
    seeds) 10 µm apart, λ = 0.1 nm at a 10 nm object pixel (detector 0.96 m away, 75 µm
    pixels), 128² probe with 2 modes (0.8/0.2), Fermat 6000 at 12 px, 1e6 photons; the start
    is three slices of ones and `gaps` holds the spacings.
    """
    if kind == "ms128":
        n, side, photons, wavelength, distance = 128, 1536, 1e6, 1e-10, 0.96
        pos = fermat_positions(6000, 12.0)
        if scale < 1.0:
            pos = pos[:max(2, int(len(pos) * scale))]
        truth = [smooth_object(side, seed + 2 + k, np.pi / 4) for k in range(3)]
        probe = hermite_probe(n, n / 4.0, [0.8, 0.2])
        c = corners(pos, n, side)
        px = wavelength * distance / (n * DETECTOR_PIXEL)
        gaps = (1e-5, 1e-5)
        counts = multislice_counts_gpu(truth, probe, c, gaps, wavelength, px, photons, seed + 3,
                                       device=device)
        start = np.ones((3, side, side), np.complex128)
        return dict(counts=counts, y=pos[:, 0] * px, x=pos[:, 1] * px, object=start,
                    probe=probe * np.sqrt(photons / (np.abs(probe) ** 2).sum()),
                    truth=np.concatenate(truth), corners=c, n=n, side=side,
                    wavelength=wavelength, distance=distance, detector_pixel=DETECTOR_PIXEL,
                    true_offsets=np.zeros((len(pos), 2)), gaps=gaps)
    if kind == "rpie64":
        n, side, modes, photons = 64, 256, [1.0], 1e5
        pos = raster_positions(20, 20, 8, 1.0, seed + 1)
    elif kind == "lsqml128":
        n, side, modes, photons = 128, 1024, [0.8, 0.15, 0.05], 1e6
        pos = fermat_positions(4096, 6.0)
    elif kind == "ml256":
        n, side, modes, photons = 256, 2048, [0.8, 0.2], 1e7
        pos = fermat_positions(10000, 12.0)
    elif kind == "fermat256":
        n, side, modes, photons = 256, 1280, [0.8, 0.2], 1e7
        pos = fermat_positions(4096, 12.0)
    else:
        raise ValueError(kind)
    if scale < 1.0:
        pos = pos[:max(2, int(len(pos) * scale))]
    truth = smooth_object(side, seed + 2)
    probe = hermite_probe(n, n / 4.0, modes) if len(modes) > 1 else aperture_probe(n, n / 4.0)[None] * 30.0
    c = corners(pos, n, side)
    true_offsets = np.zeros((len(pos), 2))
    if kind == "ml256":
        true_offsets = np.random.default_rng(seed + 4).normal(0.0, 1.5, (len(pos), 2))
        counts = far_field_counts_gpu(truth, probe, c, true_offsets, photons, seed + 3,
                                      device=device)
    elif kind == "fermat256":
        counts = far_field_counts_gpu(truth, probe, c, true_offsets, photons, seed + 3,
                                      device=device)
    else:
        counts = far_field_counts(truth, probe, c, photons, seed + 3)
    px = object_pixel(n)
    start = np.ones_like(truth)
    return dict(counts=counts, y=pos[:, 0] * px, x=pos[:, 1] * px, object=start, probe=probe,
                truth=truth, corners=c, n=n, side=side, wavelength=WAVELENGTH,
                distance=DISTANCE, detector_pixel=DETECTOR_PIXEL, true_offsets=true_offsets)
