"""Data model of the hot path (oracle restatement, test infrastructure only).

Follows physwkim/ptyrs `ptyrs/src/base`: positions preprocessing, window corners, the
address table of views, the counts with their mask sentinel and the FFT-shifted observed
intensities, plus `engine/batch.rs`'s seeded mini-batches.
"""
import math

import numpy as np

# ptyrs/src/base/counts.rs:3-4
MASKED = 65535
MAX_COUNT = 65534

M64 = (1 << 64) - 1


def pixel_size_object(wavelength, distance, frame, detector_pixel):
    """Object pixel `[py, px]` = `λz / (n·pitch)` per axis (base/geometry.rs:120-126)."""
    lz = wavelength * distance
    return [lz / (frame[0] * detector_pixel), lz / (frame[1] * detector_pixel)]


def _round_half_even(v):
    return float(np.round(v))  # numpy rounds half to even


def _pynx_axis(v, px):
    """One axis of `Positions::pynx_preprocess` (base/positions.rs:289-315)."""
    v = [float(a) for a in v]
    if not v:
        return []
    n = float(len(v))
    s = 0.0
    for a in v:
        s += a  # sequential sum, as Rust's Iterator::sum
    mean = s / n
    pos = [p - mean for p in v]
    frac = [math.fmod(p / px, 1.0) for p in pos]
    frac = [f + 1.0 if f < 0 else f for f in frac]  # f64::rem_euclid(1.0)
    if all(abs(min(d, 1.0 - d)) < 0.1 for d in frac):
        frac = []
        for p in pos:
            r = math.fmod(p + 0.5, 1.0)
            if r < 0:
                r += 1.0
            frac.append(r - 0.5)
    s = 0.0
    for f in frac:
        s += f
    fmean = s / n
    if all(abs(d - fmean) <= 0.02 + 1e-5 * abs(fmean) for d in frac):
        pos = [_round_half_even((p - fmean * px) / px) * px for p in pos]
    return pos


def pynx_preprocess(y, x, pixel):
    """PyNX position preprocessing: centre, remove a shared sub-pixel offset and snap
    (base/positions.rs:274-277)."""
    return np.array(_pynx_axis(y, pixel[0])), np.array(_pynx_axis(x, pixel[1]))


def view_corner(obj, frame, shift):
    """Window corner along one axis: `round_half_even((obj − frame)//2 + shift)`, or None when
    the window leaves the object (base/addr.rs:123-127)."""
    if obj < frame:
        return None
    span = obj - frame
    if not math.isfinite(shift):
        return None
    c = _round_half_even((span // 2) + shift)
    if 0.0 <= c <= span:
        return int(c)
    return None


def required_obj_shape(y, x, pixel, frame, margin):
    """PyNX `calc_obj_shape(..., multiple=4)` (base/addr.rs:131-149)."""
    def axis(v, p, n):
        ext = 0.0
        for a in v:
            ext = max(ext, abs(math.ceil(a / p)) + 1.0)
        length = int(2.0 * ext) + n + margin
        return -(-length // 4) * 4
    return [axis(y, pixel[0], frame[0]), axis(x, pixel[1], frame[1])]


# View fields, frame-major and mode-minor (base/addr.rs:6-13, 32-81).
VIEW_DTYPE = np.dtype([("frame", np.uint32), ("mode", np.uint32), ("probe", np.uint32),
                       ("obj", np.uint32), ("oy", np.uint32), ("ox", np.uint32)])


class AddrTable:
    """Address table of every (frame, mode) view (base/addr.rs:22-116). `y`, `x` are
    preprocessed positions in metres, `pixel` `[py, px]`."""

    def __init__(self, y, x, pixel, frame, obj, nprobe, nobj):
        if nprobe == 0 or nobj == 0:
            raise ValueError("nprobe and nobj must be >= 1")
        if obj[0] < frame[0] or obj[1] < frame[1]:
            raise ValueError(f"object {obj} smaller than frame {frame}")
        nmode = nprobe * nobj
        views = np.zeros(len(y) * nmode, VIEW_DTYPE)
        for f, (py, px) in enumerate(zip(y, x)):
            dy, dx = py / pixel[0], px / pixel[1]
            oy, ox = view_corner(obj[0], frame[0], dy), view_corner(obj[1], frame[1], dx)
            if oy is None or ox is None:
                raise ValueError(f"frame {f} at ({dy:.2f}, {dx:.2f}) object pixels leaves "
                                 f"object {obj}")
            for m in range(nmode):
                views[f * nmode + m] = (f, m, m % nprobe, m // nprobe, oy, ox)
        self.views = views
        self.nframe = len(y)
        self.nprobe = nprobe
        self.nobj = nobj
        self.nmode = nmode
        self.frame = list(frame)
        self.obj = list(obj)

    def frame_views(self, f):
        return self.views[f * self.nmode:(f + 1) * self.nmode]


def _mix(z):
    """SplitMix64 output function (engine/batch.rs:8-12)."""
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def random_batches(nframe, size, seed, epoch):
    """Seeded shuffled mini-batches, each sorted (engine/batch.rs:18-38)."""
    assert size > 0, "batch size must be positive"
    state = (seed ^ _mix(epoch)) & M64
    order = list(range(nframe))
    for i in range(nframe - 1, 0, -1):
        state = (state + 0x9E3779B97F4A7C15) & M64
        j = (_mix(state) * (i + 1)) >> 64
        order[i], order[j] = order[j], order[i]
    return [sorted(order[s:s + size]) for s in range(0, nframe, size)]


def counts_from_f64(values, detector_mask=None, limit=True):
    """`Counts::from_f64` (base/counts.rs): negative or masked → MASKED. With `limit` the
    reference's u16 range and integer checks apply; without, values are kept as float
    counts (the wide-count path the configs above 65534 photons need)."""
    values = np.asarray(values, np.float64)
    masked = values < 0
    if detector_mask is not None:
        masked = masked | np.broadcast_to(np.asarray(detector_mask, bool), values.shape[-2:])
    if limit:
        bad = (~masked) & (~np.isfinite(values) | (values > MAX_COUNT))
        if bad.any():
            raise ValueError("count out of range")
        if ((~masked) & (np.mod(values, 1.0) != 0)).any():
            raise ValueError("non-integer count")
        out = values.astype(np.uint16)
        out[masked] = MASKED
        return out
    out = values.copy()
    out[masked] = -1.0
    return out


def shift_index(j, ny, nx):
    """Natural index of shifted index `j` (engine/obs.rs:44-48); its own inverse."""
    y, x = j // nx, j % nx
    return ((y + ny // 2) % ny) * nx + (x + nx // 2) % nx


def fftshift2(a):
    """`shift` applied to every plane: even frames, so its own inverse."""
    return np.fft.fftshift(a, axes=(-2, -1))


class Observed:
    """Measured intensities in the FFT-shifted layout (engine/obs.rs:52-109). `counts` is
    u16 (MASKED sentinel) or float (negative masked). `iobs` holds float64 values with the
    mask in `mask` (True = masked)."""

    def __init__(self, counts):
        counts = np.asarray(counts)
        if counts.dtype == np.uint16:
            mask = counts == MASKED
            vals = counts.astype(np.float64)
        else:
            mask = counts < 0
            vals = counts.astype(np.float64)
        vals[mask] = 0.0
        self.iobs = fftshift2(vals)
        self.mask = fftshift2(mask)
        self.nframe = counts.shape[0]
        self.frame = list(counts.shape[1:])
        self.nb_obs = int((~mask).sum())

    def total(self):
        return float(self.iobs[~self.mask].sum())
