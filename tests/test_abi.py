"""The C ABI without a GPU: the library loads and exports every function include/ptyb200.h
declares, and its native host logic (seeded batches, PyNX position preprocessing and window
corners) is bit-exact with the oracle's restatement of the reference."""
import os
import re

import numpy as np
import pytest

from oracle.base import AddrTable, pynx_preprocess, random_batches
from ptyrs_b200 import _lib, build
from ptyrs_b200.engine import PtybError, random_batches as native_batches, view_corners

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def declared():
    text = open(os.path.join(ROOT, "include", "ptyb200.h")).read()
    return sorted(set(re.findall(r"\b(ptyb_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    names = declared()
    assert "ptyb_create" in names and "ptyb_rpie" in names and len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES)


def test_kernel_kinds_are_named(lib):
    """Every kernel kind of the per-kernel timing has its own name (the names key the bench's
    kernel table)."""
    k = lib.ptyb_kernel_kinds()
    names = [lib.ptyb_kernel_name(i).decode() for i in range(k)]
    assert all(names) and len(set(names)) == k
    assert {"frame_carry", "object_blend", "frame_ml_grad", "opr_step"} <= set(names)
    assert lib.ptyb_kernel_name(k).decode() == ""


@pytest.mark.parametrize("nframe,size,seed,epoch", [(0, 3, 7, 0), (1, 1, 7, 0), (30, 4, 7, 0),
                                                    (30, 4, 7, 5), (400, 100, 7, 3),
                                                    (4096, 256, 123456789, 99),
                                                    (17, 100, 2**64 - 1, 2**63)])
def test_random_batches_bit_exact(lib, nframe, size, seed, epoch):
    assert native_batches(nframe, size, seed, epoch) == random_batches(nframe, size, seed, epoch)


def oracle_corners(y, x, pixel, frame, obj):
    py, px = pynx_preprocess(y, x, pixel)
    t = AddrTable(py, px, pixel, frame, obj, 1, 1)
    return np.stack([t.views["oy"], t.views["ox"]], 1).astype(np.int32)


@pytest.mark.parametrize("case", range(6))
def test_view_corners_bit_exact(lib, case):
    rng = np.random.default_rng(case)
    px = 3.1e-8
    n, obj = 64, [256, 240]
    if case == 0:      # scattered sub-pixel positions: only centred
        p = rng.uniform(-40, 40, size=(50, 2))
    elif case == 1:    # near-integer positions: snapped
        p = np.round(rng.uniform(-40, 40, size=(50, 2))) + rng.uniform(-0.05, 0.05, (50, 2))
    elif case == 2:    # a shared half-pixel offset: removed, then snapped
        p = np.round(rng.uniform(-40, 40, size=(50, 2))) + 0.5 + rng.uniform(-0.01, 0.01, (50, 2))
    elif case == 3:    # exact ties of the rounding
        p = np.array([[0.5, -0.5], [1.5, 2.5], [-3.5, 4.0], [7.0, -7.5]])
    elif case == 4:    # a raster with jitter, as the benchmarks scan
        g = np.stack(np.mgrid[:20, :20], -1).reshape(-1, 2) * 8.0
        p = g + rng.uniform(-1, 1, g.shape)
    else:              # a Fermat spiral
        k = np.arange(300)
        r, t = 3.0 * np.sqrt(k), k * np.pi * (3 - np.sqrt(5))
        p = np.stack([r * np.sin(t), r * np.cos(t)], 1)
    y, x = p[:, 0] * px, p[:, 1] * px
    want = oracle_corners(y, x, [px, px], [n, n], obj)
    got = view_corners(y, x, [px, px], [n, n], obj)
    assert (got == want).all()


def test_view_corners_rejects_a_window_outside(lib):
    px = 1e-8
    y = np.array([0.0, 200.0]) * px
    with pytest.raises(PtybError):
        view_corners(y, y, [px, px], [64, 64], [128, 128])


def test_live_ring_refuses_bad_parameters_before_any_device_call():
    from ptyrs_b200.live import LiveRing
    from ptyrs_b200 import PtybError
    for kw in (dict(n=100), dict(n=64, slots=0), dict(n=64, capacity=0), dict(n=64, batch=-1),
               dict(n=64, pos_wait_s=-1.0)):
        n = kw.pop("n")
        with pytest.raises(PtybError, match="invalid: live"):
            LiveRing(n, 1.5e-10, 1.0, 75e-6, **kw)
    with pytest.raises(PtybError, match="invalid: live"):
        LiveRing(64, 0.0, 1.0, 75e-6)
