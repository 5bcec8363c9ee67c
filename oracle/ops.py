"""Operators of the hot path in float64 (oracle restatement, test infrastructure only).

Follows physwkim/ptyrs `ptyrs/src/engine/{fft,propagate,ops}.rs`. Exit waves are held as
`[nview, ny, nx]` complex128 arrays in the FFT-shifted layout, as the reference holds them.
"""
import numpy as np

from .base import fftshift2


# --------------------------------------------------------------------------------------
# Unitary FFT (engine/fft.rs:155-234): numpy's `norm="ortho"`, no shift. With FFT_WORKERS set,
# scipy's pocketfft splits a batch of planes over that many threads (same transforms).

FFT_WORKERS = None


def fft2(a):
    if FFT_WORKERS:
        import scipy.fft
        return scipy.fft.fft2(a, axes=(-2, -1), norm="ortho", workers=FFT_WORKERS)
    return np.fft.fft2(a, axes=(-2, -1), norm="ortho")


def ifft2(a):
    if FFT_WORKERS:
        import scipy.fft
        return scipy.fft.ifft2(a, axes=(-2, -1), norm="ortho", workers=FFT_WORKERS)
    return np.fft.ifft2(a, axes=(-2, -1), norm="ortho")


def freq(k, n):
    """numpy `fftfreq` value of index `k` (engine/features.rs:337-344)."""
    kk = k if k < (n + 1) // 2 else k - n
    return kk * (1.0 / n)


# --------------------------------------------------------------------------------------
# Propagators (engine/propagate.rs).

class Wavefield:
    """pty-chi wavefield parameters (engine/propagate.rs:216-313)."""

    def __init__(self, shape, wavelength, pixel, distance):
        if any(n == 0 or n % 2 for n in shape):
            raise ValueError(f"plane shape {shape} must be even and non-zero")
        self.shape = list(shape)
        self.wavelength = wavelength
        self.pixel = list(pixel)
        self.distance = distance

    def pixel_width_wlu(self):
        return self.pixel[1] / self.wavelength

    def aspect_ratio(self):
        return self.pixel[1] / self.pixel[0]

    def distance_wlu(self):
        return self.distance / self.wavelength

    def fresnel_number(self):
        w = self.pixel_width_wlu()
        return w * w / self.distance_wlu()

    def prefers_fresnel(self):
        ny, nx = self.shape
        d = abs(self.distance_wlu())
        w = self.pixel_width_wlu()
        h = w / self.aspect_ratio()
        return w * w / d < 1.0 / nx or h * h / d < 1.0 / ny


class Propagator:
    """Unitary free-space propagator in the shifted layout (engine/propagate.rs:316-470).
    kind: "fourier", "angular" or "fresnel"."""

    def __init__(self, kind, shape, tf=None, a=None, b=None, reverse=False, scale=None,
                 plane_quad=(0.0, 0.0)):
        self.kind = kind
        self.shape = list(shape)
        self.tf, self.a, self.b = tf, a, b
        self.reverse = reverse
        self.scale = scale
        self.plane_quad = list(plane_quad)

    @staticmethod
    def free_space(w):
        if np.isinf(w.distance):
            return Propagator("fourier", w.shape)
        if w.prefers_fresnel():
            return Propagator._fresnel(w)
        return Propagator._angular(w)

    @staticmethod
    def _angular(w):
        """Transfer function `exp(2πi z √(1 − r))`, 0 on the evanescent band
        (engine/propagate.rs:505-531)."""
        ny, nx = w.shape
        ar = w.aspect_ratio()
        width = w.pixel_width_wlu()
        i2piz = 2.0 * np.pi * w.distance_wlu()
        tf = np.zeros((ny, nx), np.complex128)
        for y in range(ny):
            fy = freq(y, ny)
            for x in range(nx):
                fx = freq(x, nx)
                ratio = (fx * fx + (ar * fy) * (ar * fy)) / (width * width)
                if ratio < 1.0:
                    ph = i2piz * np.sqrt(1.0 - ratio)
                    tf[y, x] = complex(np.cos(ph), np.sin(ph))
        return Propagator("angular", w.shape, tf=tf)

    @staticmethod
    def _fresnel(w):
        """Fresnel transform `x ↦ a·Fft2(b·x)` (engine/propagate.rs:534-571)."""
        ny, nx = w.shape
        fr = w.fresnel_number()
        ar = w.aspect_ratio()
        ph1 = 2.0 * np.pi * w.distance_wlu()
        c1 = complex(np.cos(ph1), np.sin(ph1))
        c1c0 = c1 * complex(0.0, -np.sign(fr))
        n, m = float(nx), float(ny)
        a = np.zeros(ny * nx, np.complex128)
        b = np.zeros(ny * nx, np.complex128)
        for j in range(ny * nx):
            jy, jx = j // nx, j % nx
            i = ((jy + ny // 2) % ny) * nx + (jx + nx // 2) % nx
            xx = float(i % nx) - float(nx // 2)
            yy = float(i // nx) - float(ny // 2)
            s2 = (xx / n) * (xx / n) + (ar * yy / m) * (ar * yy / m)
            pa = s2 * np.pi / fr
            a[j] = c1c0 * complex(np.cos(pa), np.sin(pa))
            sb = xx * xx + (yy / ar) * (yy / ar)
            pb = np.pi * fr * sb
            b[j] = complex(np.cos(pb), np.sin(pb))
        c0 = fr / ar
        return Propagator("fresnel", w.shape, a=a.reshape(ny, nx), b=b.reshape(ny, nx),
                          reverse=w.distance < 0.0, scale=(ny * nx) * (c0 * c0),
                          plane_quad=(np.pi * fr / (ar * ar), np.pi * fr))

    def intensity_scale(self):
        if self.kind == "fourier":
            return float(self.shape[0] * self.shape[1])
        if self.kind == "angular":
            return 1.0
        return self.scale

    def after_plane(self, planes):
        """Forward of planes that carry the Fresnel `B` already (propagate.rs:405-423)."""
        if self.kind == "fourier":
            return fft2(planes)
        if self.kind == "angular":
            return ifft2(fft2(planes) * self.tf)
        out = ifft2(planes) if self.reverse else fft2(planes)
        return out * self.a

    def before_plane(self, planes):
        """Adjoint of `after_plane` (propagate.rs:435-453)."""
        if self.kind == "fourier":
            return ifft2(planes)
        if self.kind == "angular":
            return ifft2(fft2(planes) * np.conj(self.tf))
        out = planes * np.conj(self.a)
        return fft2(out) if self.reverse else ifft2(out)

    def forward(self, planes):
        if self.kind == "fresnel":
            planes = planes * self.b
        return self.after_plane(planes)

    def adjoint(self, planes):
        out = self.before_plane(planes)
        if self.kind == "fresnel":
            out = out * np.conj(self.b)
        return out


class Optics:
    """Exit-wave model `psi = E(P·O·q)` (engine/propagate.rs:24-207); with `gaps`, the
    angular-spectrum propagators between consecutive object slices (propagate.rs:84-99)."""

    def __init__(self, pixel, quad, propagator, gaps=()):
        self.pixel = list(pixel)
        self.quad = quad  # natural layout [ny, nx]
        self.propagator = propagator
        self.gaps = list(gaps)

    def with_slices(self, gap_wavefields):
        """This model through len(gaps) + 1 slices, each gap angular spectrum
        (propagate.rs:84-99)."""
        return Optics(self.pixel, self.quad, self.propagator,
                      [Propagator._angular(w) for w in gap_wavefields])

    def nslice(self):
        return len(self.gaps) + 1

    def slice_quad(self, s):
        """The plane phase slice `s` applies: `quad` on the last slice, none before
        (propagate.rs:143-148)."""
        return self.quad if s + 1 == self.nslice() else None

    @staticmethod
    def far_field(wavelength, distance, detector_pixel, frame):
        """PyNX far field: `quad_phase` and the unitary FFT (propagate.rs:44-53)."""
        from .base import pixel_size_object
        pixel = pixel_size_object(wavelength, distance, frame, detector_pixel)
        return Optics(pixel, quad_phase(wavelength, distance, pixel, frame),
                      Propagator("fourier", frame))

    @staticmethod
    def free_space(w):
        """pty-chi planar model (propagate.rs:57-76)."""
        ny, nx = w.shape
        prop = Propagator.free_space(w)
        quad = np.ones((ny, nx), np.complex128)
        if prop.kind == "fresnel":
            quad = fftshift2(prop.b)  # B is in the shifted layout, quad natural
        return Optics(w.pixel, quad, prop)

    def exit_forward(self, planes):
        return self.propagator.after_plane(planes)

    def exit_adjoint(self, planes):
        return self.propagator.before_plane(planes)

    def intensity_scale(self):
        return self.propagator.intensity_scale()

    def near_field(self):
        return self.propagator.kind != "fourier"


def quad_phase(wavelength, distance, pixel, frame):
    """Far-field quadratic phase, natural layout (engine/ops.rs:17-33)."""
    ny, nx = frame
    py, px = pixel
    f = np.pi / (wavelength * distance)
    dy = np.arange(ny, dtype=np.float64) - float(ny // 2)
    dx = np.arange(nx, dtype=np.float64) - float(nx // 2)
    ph = f * (dx[None, :] * dx[None, :] * px * px + dy[:, None] * dy[:, None] * py * py)
    return np.cos(ph) + 1j * np.sin(ph)


# --------------------------------------------------------------------------------------
# PyNX / pty-chi operators (engine/ops.rs).

def windows(views, obj_planes, ny, nx):
    """Object window of every view, natural layout `[nview, ny, nx]`."""
    out = np.empty((len(views), ny, nx), np.complex128)
    for k, v in enumerate(views):
        oy, ox = int(v["oy"]), int(v["ox"])
        out[k] = obj_planes[int(v["obj"])][oy:oy + ny, ox:ox + nx]
    return out


def obj_probe_to_psi(views, obj, probe, quad):
    """ObjProbe2Psi: `psi[k] = shift(P[probe_k]·O[obj_k, win_k]·q)` (engine/ops.rs:47-71)."""
    ny, nx = probe.shape[-2:]
    win = windows(views, obj, ny, nx)
    p = probe[views["probe"].astype(np.int64)]
    return fftshift2(p * win * quad)


def icalc_of(psi, nmode):
    """`Σ_modes |psi|²` per frame pixel for frame-major, mode-minor planes."""
    nv, ny, nx = psi.shape
    return (np.abs(psi.reshape(nv // nmode, nmode, ny, nx)) ** 2).sum(axis=1)


def apply_amplitude(obs, frames, nmode, psi):
    """ApplyAmplitude (engine/ops.rs:77-107)."""
    nv, ny, nx = psi.shape
    b = psi.reshape(nv // nmode, nmode, ny, nx)
    calc = np.sqrt(icalc_of(psi, nmode))
    iobs, mask = obs.iobs[frames], obs.mask[frames]
    r = np.where(mask, 1.0, np.sqrt(iobs) / np.maximum(calc, 1e-12))
    return (b * r[:, None]).reshape(psi.shape)


class Llk:
    def __init__(self, poisson=0.0, gaussian=0.0, euclidian=0.0, nb_photons_calc=0.0):
        self.poisson, self.gaussian = poisson, gaussian
        self.euclidian, self.nb_photons_calc = euclidian, nb_photons_calc

    def normalised(self, nb_obs):
        """engine/ops.rs:265-277."""
        n = float(nb_obs)
        return Llk(self.poisson / n, self.gaussian / n, self.euclidian / n,
                   self.nb_photons_calc)

    def as_dict(self):
        return dict(poisson=self.poisson, gaussian=self.gaussian, euclidian=self.euclidian,
                    nb_photons_calc=self.nb_photons_calc)


def llk(obs, frames, nmode, psi):
    """PyNX LLK sums over unmasked pixels (engine/ops.rs:119-154)."""
    icalc = icalc_of(psi, nmode)
    iobs, keep = obs.iobs[frames], ~obs.mask[frames]
    with np.errstate(divide="ignore", invalid="ignore"):
        pois = np.where(iobs > 0, icalc - iobs + iobs * np.log(iobs / icalc), icalc)
    ic, io = icalc[keep], iobs[keep]
    return Llk(float(pois[keep].sum()), float(((io - ic) ** 2 / (io + 1.0)).sum()),
               float((4.0 * (np.sqrt(io) - np.sqrt(ic)) ** 2).sum()), float(ic.sum()))


def poisson_grad(obs, frames, nmode, psi):
    """GradPoissonFourier: `psi *= 2(1 − iobs/max(1e-12, icalc))`, masked → 0
    (engine/ops.rs:161-195)."""
    nv, ny, nx = psi.shape
    icalc = icalc_of(psi, nmode)
    iobs, mask = obs.iobs[frames], obs.mask[frames]
    r = np.where(mask, 0.0, 2.0 * (1.0 - iobs / np.maximum(icalc, 1e-12)))
    return (psi.reshape(nv // nmode, nmode, ny, nx) * r[:, None]).reshape(psi.shape)


def cg_poisson_gamma(obs, frames, nmode, po, a, b):
    """PyNX CG_Poisson_Gamma numerator and denominator (engine/ops.rs:206-253)."""
    nv, ny, nx = po.shape
    sh = (nv // nmode, nmode, ny, nx)
    po, a, b = po.reshape(sh), a.reshape(sh), b.reshape(sh)
    calc = (np.abs(po) ** 2).sum(axis=1)
    r = (np.conj(po) * a).real.sum(axis=1)
    s = (np.abs(a) ** 2 + 2.0 * (np.conj(po) * b).real).sum(axis=1)
    iobs, keep = obs.iobs[frames], ~obs.mask[frames]
    calc = np.maximum(calc, 1e-32)
    d = 1.0 - iobs / calc
    num = -(2.0 * r * d)[keep].sum()
    den = (2.0 * s * d + iobs * (2.0 * r / calc) ** 2)[keep].sum()
    return float(num), float(den)


def accumulate_obj(views, obj_shape, probe, quad, psi):
    """Object back-projection over views in order (engine/ops.rs:282-310): returns
    `(num, norm)` shaped `obj_shape` `[nobj, nyo, nxo]`."""
    ny, nx = probe.shape[-2:]
    num = np.zeros(obj_shape, np.complex128)
    norm = np.zeros(obj_shape, np.float64)
    w = fftshift2(psi)
    cq = np.conj(quad[None] * probe)
    p2 = np.abs(probe) ** 2
    for k, v in enumerate(views):
        oy, ox, o, p = int(v["oy"]), int(v["ox"]), int(v["obj"]), int(v["probe"])
        num[o, oy:oy + ny, ox:ox + nx] += w[k] * cq[p]
        norm[o, oy:oy + ny, ox:ox + nx] += p2[p]
    return num, norm


def accumulate_probe(views, obj, probe_shape, quad, psi):
    """Probe back-projection over views in order (engine/ops.rs:315-345)."""
    ny, nx = probe_shape[-2:]
    num = np.zeros(probe_shape, np.complex128)
    norm = np.zeros(probe_shape, np.float64)
    w = fftshift2(psi)
    win = windows(views, obj, ny, nx)
    for k, v in enumerate(views):
        p = int(v["probe"])
        num[p] += w[k] * np.conj(quad * win[k])
        norm[p] += np.abs(win[k]) ** 2
    return num, norm


# --------------------------------------------------------------------------------------
# The position model under Patch sampling (engine/features.rs:337-527).

POSITION_STEP = 0.3
POSITION_LIMIT = 0.1
EPS_POSITION = 1e-6


def _freqs(n):
    return np.array([freq(k, n) for k in range(n)])


def translation(shape, offset):
    """`exp(−2πi f·offset)` on the unshifted DFT grid (engine/features.rs:364-369)."""
    ny, nx = shape
    fy, fx = _freqs(ny), _freqs(nx)
    ph = -2.0 * np.pi * (fy[:, None] * offset[0] + fx[None, :] * offset[1])
    return np.cos(ph) + 1j * np.sin(ph), (fy, fx)


def move_planes(planes, quad, offset, axes=()):
    """Natural-layout planes moved by `offset` as pty-chi moves its probe, `conj(q)·T(q·p)`,
    with the derivative over the listed offset components (engine/features.rs:393-441)."""
    shape = planes.shape[-2:]
    e, (fy, fx) = translation(shape, offset)
    for a in axes:
        f = fy[:, None] if a == 0 else fx[None, :]
        e = e * (-2j * np.pi * f)
    q = 1.0 if quad is None else quad
    out = ifft2(fft2(planes * q) * e)
    return out * (np.conj(quad) if quad is not None else 1.0)


def gradient_sums(patch, w, chi):
    """Per axis `num = Σ Re(conj(∂O·w)·chi)`, `den = Σ |∂O·w|²` with ∂O the periodic Fourier
    derivative of the natural-layout window (engine/features.rs:459-492); `w`, `chi` shifted."""
    ny, nx = patch.shape
    fy, fx = _freqs(ny), _freqs(nx)
    g = fft2(patch)
    grads = [ifft2(g * (2j * np.pi * fy[:, None])), ifft2(g * (2j * np.pi * fx[None, :]))]
    num, den = [0.0, 0.0], [0.0, 0.0]
    for axis in range(2):
        u = fftshift2(grads[axis]) * w
        num[axis] = float((np.conj(u) * chi).real.sum())
        den[axis] = float((np.abs(u) ** 2).sum())
    return [num, den]


def gradient_directions(sums, eps):
    """`num / (den + max(max_batch den, eps))` per axis (engine/features.rs:496-501)."""
    mx = [max([eps] + [s[1][a] for s in sums]) for a in range(2)]
    return [[s[0][a] / (s[1][a] + mx[a]) for a in range(2)] for s in sums]


def batch_position_step(d, frames, delta):
    """pty-chi's SGD position step with the per-axis clip `min(10·MAD, 0.1)` over every frame
    (engine/features.rs:507-521); `d` `[P, 2]` is updated in place."""
    dx = np.zeros_like(d)
    for f, dl in zip(frames, delta):
        dx[f] = [POSITION_STEP * dl[0], POSITION_STEP * dl[1]]
    n = float(len(d))
    for axis in range(2):
        s = 0.0
        for v in dx[:, axis]:
            s += v
        mean = s / n
        s = 0.0
        for v in dx[:, axis]:
            s += abs(v - mean)
        limit = min(10.0 * (s / n), POSITION_LIMIT)
        d[:, axis] += np.clip(dx[:, axis], -limit, limit)


def position_step(d, sums):
    """The position step of AP, DM and ML (engine/features.rs:1028-1047): per axis, with `max`
    the largest `den` over every frame, `step = clip(0.3·num / (den + max), ±0.1)` (0 where the
    denominator is not positive), then `d += step − mean(step)` over every frame. `sums`
    `[P][2][2]` holds each frame's `[num, den]`; `d` `[P, 2]` is updated in place."""
    n = len(d)
    for axis in range(2):
        mx = 0.0
        for s in sums:
            mx = max(mx, float(s[1][axis]))
        step = []
        for s in sums:
            den = float(s[1][axis]) + mx
            step.append(min(max(POSITION_STEP * float(s[0][axis]) / den, -POSITION_LIMIT),
                            POSITION_LIMIT) if den > 0.0 else 0.0)
        total = 0.0
        for v in step:
            total += v
        mean = total / n
        for f in range(n):
            d[f, axis] += step[f] - mean


def illumination(views, obj_shape, probe):
    """pty-chi illumination map `Σ|P[probe_k]|²` on each window (engine/lsqml.rs:374-388)."""
    ny, nx = probe.shape[-2:]
    out = np.zeros(obj_shape, np.float64)
    p2 = np.abs(probe) ** 2
    for v in views:
        oy, ox = int(v["oy"]), int(v["ox"])
        out[int(v["obj"]), oy:oy + ny, ox:ox + nx] += p2[int(v["probe"])]
    return out
