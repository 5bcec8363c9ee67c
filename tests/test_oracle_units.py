"""The oracle against the reference's own known-answer unit tests: window corners and the
address table (ptyrs/src/base/addr.rs:155-214), position preprocessing
(base/positions.rs:329-358), the shifted layout and mask (engine/obs.rs:117-127), the FFT
(engine/fft.rs:251-285), the quadratic phase and the LLK hand values (engine/ops.rs:409-502)."""
import numpy as np
import pytest

from oracle import ops
from oracle.base import (AddrTable, MASKED, Observed, pynx_preprocess, required_obj_shape,
                         shift_index, view_corner)


def test_corner_rounds_half_even_and_rejects_windows_outside():
    assert view_corner(40, 16, 0.5) == 12
    assert view_corner(40, 16, 1.5) == 14
    assert view_corner(40, 16, -0.4) == 12
    assert view_corner(40, 16, -12.5) == 0
    assert view_corner(40, 16, 12.0) == 24
    for s in (-12.6, 12.6, -20.0, 30.0, float("nan")):
        assert view_corner(40, 16, s) is None
    assert view_corner(15, 16, 0.0) is None


def test_table_rejects_a_frame_outside_the_object():
    AddrTable([0.0, 6.0], [0.0, 0.0], [1.0, 1.0], [8, 8], [20, 20], 1, 1)
    with pytest.raises(ValueError):
        AddrTable([0.0, 6.6], [0.0, 0.0], [1.0, 1.0], [8, 8], [20, 20], 1, 1)


def test_required_shape_holds_every_view_and_its_neighbour():
    y, x = [-3.2, 1.0, 9.49], [0.0, 5.1, -7.5]
    for margin in (0, 1, 4, 16):
        obj = required_obj_shape(y, x, [1.0, 1.0], [16, 16], margin)
        for a, b in zip(y, x):
            for axis, d in ((0, a), (1, b)):
                c = view_corner(obj[axis], 16, d)
                assert c is not None and c + 16 < obj[axis]
    assert required_obj_shape([-3.2, 1.0], [0.0, 5.1], [1.0, 1.0], [16, 16], 8) == [32, 40]


def test_table_orders_frame_major_and_maps_modes():
    t = AddrTable([0.0, 2.0], [0.0, -3.0], [1.0, 1.0], [8, 8], [20, 20], 2, 1)
    assert len(t.views) == 4
    v = t.frame_views(1)
    assert (v[0]["frame"], v[0]["mode"], v[0]["probe"], v[0]["obj"]) == (1, 0, 0, 0)
    assert (v[1]["mode"], v[1]["probe"]) == (1, 1)
    assert (v[0]["oy"], v[0]["ox"]) == (8, 3)


def snapped(pixels, px):
    x = [v * px for v in pixels]
    _, p = pynx_preprocess(x, x, [px, px])
    return [v / px for v in p]


def test_positions_snap_and_offsets():
    for got, want in zip(snapped([0.0, 2.02, 4.0, 6.0], 1e-8), [-3.0, -1.0, 1.0, 3.0]):
        assert abs(got - want) < 1e-9
    for got, want in zip(snapped([0.0, 3.01, 6.0, 8.99], 1e-8), [-5.0, -2.0, 1.0, 4.0]):
        assert abs(got - want) < 1e-9
    x = [0.0, 1.3, 2.71, 4.05]
    _, p = pynx_preprocess(x, x, [1.0, 1.0])
    mean = sum(x) / 4
    for a, b in zip(p, x):
        assert abs(a - (b - mean)) < 1e-12


def test_shift_moves_centre_to_origin_and_masks():
    assert shift_index(0, 4, 6) == 2 * 6 + 3
    assert shift_index(shift_index(7, 4, 6), 4, 6) == 7
    raw = np.arange(24, dtype=np.uint16)
    raw[2 * 6 + 3] = MASKED
    o = Observed(raw.reshape(1, 4, 6))
    assert o.mask[0].ravel()[0] and o.iobs[0].ravel()[1] == 16.0 and o.nb_obs == 23


def test_fft_matches_direct_dft_with_ortho_scale():
    ny, nx = 4, 6
    t = np.arange(ny * nx, dtype=float)
    x = (np.sin(0.37 * t) + 0.1 * np.cos(t) + 1j * (np.cos(1.3 * t) - 0.2)).reshape(ny, nx)
    got = ops.fft2(x)
    ky, kx, y, xx = np.ogrid[:ny, :nx, :ny, :nx]
    w = np.exp(-2j * np.pi * (ky * y / ny + kx * xx / nx))
    want = (w * x[None, None]).sum(axis=(2, 3)) / np.sqrt(ny * nx)
    assert np.abs(got - want).max() < 1e-12
    assert np.abs(ops.ifft2(got) - x).max() < 1e-13


def test_quad_phase_is_one_at_centre_and_symmetric():
    px = 1e-10 * 2.0 / (8 * 5e-5)
    q = ops.quad_phase(1e-10, 2.0, [px, px], [8, 8])
    assert q[4, 4] == 1.0
    assert abs(q[3, 4] - q[5, 4]) < 1e-15
    want = np.exp(1j * np.pi / 2e-10 * 2.0 * px * px)
    assert abs(q[3, 5] - want) < 1e-14


def test_llk_matches_hand_values_and_skips_masked():
    raw = np.array([9, MASKED, 0, 4], np.uint16).reshape(1, 2, 2)
    obs = Observed(raw)
    assert list(obs.iobs.ravel()) == [4.0, 0.0, 0.0, 9.0] and list(obs.mask.ravel()) == [
        False, False, True, False]
    psi = (1j * np.array([2.0, 1.0, 5.0, 2.0])).reshape(1, 2, 2)
    l = ops.llk(obs, slice(0, 1), 1, psi)
    p = 0.0 + 1.0 + (4.0 - 9.0 + 9.0 * np.log(9.0 / 4.0))
    assert abs(l.poisson - p) < 1e-14
    assert abs(l.gaussian - (0.0 + 1.0 + 25.0 / 10.0)) < 1e-14
    assert abs(l.euclidian - 4.0 * (0.0 + 1.0 + 1.0)) < 1e-14
    assert l.nb_photons_calc == 9.0
