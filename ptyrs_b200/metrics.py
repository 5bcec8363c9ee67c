"""Reconstruction error of an object against a reference object.

`object_nrmse` is the figure the accuracy targets are stated in: over the illuminated pixels
(a weight > 0), the global phase and a linear phase ramp of `a` relative to `b` are removed —
the ambiguities a far-field ptychographic reconstruction cannot fix (the ramp is what PyNX's
ZeroPhaseRamp removes, reference engine/ptycho.rs:1134-1180) — and the scale is kept, so a
uniform amplitude error counts in full: ‖a·e^{-iθ} − b‖ / ‖b‖ with θ = φ0 + gy·y + gx·x.
"""
import numpy as np


def phase_ramp_fit(a, b, weight, rounds=3):
    """(φ0, gy, gx) of the phase of a·conj(b) over the pixels where `weight` > 0: weighted
    least squares on the wrapped phase difference, weights |a|·|b|·weight, refined `rounds`
    times on what the previous fit leaves (so a ramp of many radians across the object is
    followed without unwrapping)."""
    a = np.asarray(a)
    b = np.asarray(b)
    ny, nx = a.shape[-2:]
    yy, xx = np.meshgrid(np.arange(ny, dtype=float), np.arange(nx, dtype=float), indexing="ij")
    yy = np.broadcast_to(yy, a.shape)
    xx = np.broadcast_to(xx, a.shape)
    m = weight > 0
    w = (np.abs(a) * np.abs(b) * weight)[m]
    cross = (a * np.conj(b))[m]
    y, x = yy[m] - ny / 2.0, xx[m] - nx / 2.0
    theta = np.zeros(3)
    if w.sum() <= 0:
        return theta
    # start from the ramp at the peak of the weighted cross product's spectrum (4× padded),
    # so the first least-squares round sees less than a cycle across the object
    field = np.zeros((4 * ny, 4 * nx), complex)
    field[:ny, :nx] = np.where(weight > 0, a * np.conj(b) * weight, 0).reshape(
        -1, ny, nx).sum(axis=0)
    ky, kx = np.unravel_index(np.argmax(np.abs(np.fft.fft2(field))), field.shape)
    theta[1] = 2 * np.pi * ((ky + 2 * ny) % (4 * ny) - 2 * ny) / (4 * ny)
    theta[2] = 2 * np.pi * ((kx + 2 * nx) % (4 * nx) - 2 * nx) / (4 * nx)
    theta[0] = np.angle(np.sum(w * np.exp(1j * np.angle(cross)) *
                               np.exp(-1j * (theta[1] * y + theta[2] * x))))
    design = np.stack([np.ones_like(y), y, x], axis=1) * np.sqrt(w)[:, None]
    for _ in range(rounds):
        rest = np.angle(cross * np.exp(-1j * (theta[0] + theta[1] * y + theta[2] * x)))
        step, *_ = np.linalg.lstsq(design, rest * np.sqrt(w), rcond=None)
        theta = theta + step
    # back to the origin of the array's own pixel grid
    return np.array([theta[0] - theta[1] * ny / 2.0 - theta[2] * nx / 2.0, theta[1], theta[2]])


def object_nrmse(a, b, weight):
    """‖a·e^{-iθ} − b‖ / ‖b‖ over the pixels where `weight` > 0, θ the global phase and linear
    phase ramp of `a` against `b` (phase_ramp_fit); no scale is divided out. `a`, `b` and
    `weight` share a shape whose last two axes are the object's (several slices share one
    ramp)."""
    a = np.asarray(a)
    b = np.asarray(b)
    weight = np.broadcast_to(weight, a.shape)
    p0, gy, gx = phase_ramp_fit(a, b, weight)
    ny, nx = a.shape[-2:]
    yy, xx = np.meshgrid(np.arange(ny, dtype=float), np.arange(nx, dtype=float), indexing="ij")
    aligned = a * np.exp(-1j * (p0 + gy * yy + gx * xx))
    m = weight > 0
    return float(np.linalg.norm((aligned - b)[m]) / np.linalg.norm(b[m]))
