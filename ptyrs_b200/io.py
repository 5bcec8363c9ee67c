"""Scan and reconstruction files through the library's HDF5 reader (C ABI `ptyb_read_cxi`,
`ptyb_read_ptyr`), mirroring the reference's `ptyrs::io::{read_cxi, read_ptyr}`
(physwkim/ptyrs ptyrs/src/io/cxi.rs, ptyr.rs)."""
import ctypes

import numpy as np

from . import _lib
from .engine import STATUS, PtybError, Scan


def _error(rc, lib):
    # the reason may quote names out of a damaged file: undecodable bytes are replaced
    return PtybError(STATUS.get(rc, rc), lib.ptyb_io_last_error().decode(errors="replace"))


def read_cxi(path):
    """The `Scan` of a CXI file in PyNX's layout: counts `uint16 [nframe, ny, nx]` in detector
    order with 65535 masked, positions in metres from the translation rows, the geometry from
    the energy, distance and pixel size."""
    lib = _lib.load()
    s = _lib.CxiScan()
    rc = lib.ptyb_read_cxi(str(path).encode(), ctypes.byref(s))
    if rc != 0:
        raise _error(rc, lib)
    try:
        n, ny, nx = s.nframe, s.ny, s.nx
        counts = np.ctypeslib.as_array(s.counts, shape=(n * ny * nx,)).reshape(n, ny, nx).copy()
        y = np.ctypeslib.as_array(s.y, shape=(n,)).copy()
        x = np.ctypeslib.as_array(s.x, shape=(n,)).copy()
        return Scan(counts, y, x, s.wavelength, s.distance, s.detector_pixel)
    finally:
        lib.ptyb_free_cxi(ctypes.byref(s))


def read_ptyr(path):
    """The object and probe of a PtyPy `.ptyr` reconstruction: a dict of `object`
    `complex128 [nobj, ny, nx]`, `probe` `complex128 [nprobe, ny, nx]`, `psize` and `origin`
    ([y, x] of the object storage)."""
    lib = _lib.load()
    r = _lib.Ptyr()
    rc = lib.ptyb_read_ptyr(str(path).encode(), ctypes.byref(r))
    if rc != 0:
        raise _error(rc, lib)
    try:
        def arr(p, shape):
            n = int(np.prod(shape))
            a = np.ctypeslib.as_array(p, shape=(2 * n,)).copy()
            return a.view(np.complex128).reshape(tuple(shape))
        return dict(object=arr(r.object, list(r.obj_shape)), probe=arr(r.probe, list(r.probe_shape)),
                    psize=tuple(r.psize), origin=tuple(r.origin))
    finally:
        lib.ptyb_free_ptyr(ctypes.byref(r))
