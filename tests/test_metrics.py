"""The accuracy figure: global phase and linear phase ramp removed, scale kept."""
import numpy as np

from ptyrs_b200.metrics import object_nrmse


def _object(seed=0, n=96):
    rng = np.random.default_rng(seed)
    return (1.0 - 0.2 * rng.random((n, n))) * np.exp(1j * rng.random((n, n)))


def test_phase_and_ramp_are_removed():
    b = _object()
    y, x = np.mgrid[:96, :96]
    a = b * np.exp(1j * (0.7 + 0.31 * y - 0.17 * x))  # several radians across the object
    assert object_nrmse(a, b, np.ones(b.shape)) < 1e-12


def test_scale_is_kept():
    b = _object(1)
    assert abs(object_nrmse(1.01 * b, b, np.ones(b.shape)) - 0.01) < 1e-12


def test_noise_is_measured_outside_the_mask_ignored():
    b = _object(2)
    rng = np.random.default_rng(3)
    noise = 1e-3 * (rng.standard_normal(b.shape) + 1j * rng.standard_normal(b.shape)) / np.sqrt(2)
    a = b + noise * np.abs(b)
    w = np.zeros(b.shape)
    w[10:80, 5:90] = 1.0
    a[w == 0] = 0.0  # dark pixels do not count
    e = object_nrmse(a * np.exp(0.4j), b, w)
    assert 0.8e-3 < e < 1.2e-3


def test_slices_share_the_ramp():
    b = np.stack([_object(4), _object(5)])
    y, x = np.mgrid[:96, :96]
    a = b * np.exp(1j * (0.2 + 0.05 * y + 0.01 * x))
    assert object_nrmse(a, b, np.ones(b.shape[-2:])) < 1e-12
