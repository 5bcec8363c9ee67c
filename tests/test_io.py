"""The library's HDF5 reader on files libhdf5 wrote, as the reference's I/O tests read them
(ptyrs/tests/io_pynx_fixture.rs, io_ptypy_fixture.rs): PyNX's `save_ptycho_data_cxi` output
(float32 counts in gzip + shuffle chunks, an h5py bool detector mask, f32 translations, a soft
link to the data) and PtyPy's `.ptyr` storages (complex64 and complex128), every value against
the closed forms the fixtures were made from; and the refusals."""
import os

import numpy as np
import pytest

from ptyrs_b200 import PtybError
from ptyrs_b200.io import read_cxi, read_ptyr

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MASKED = 65535


def test_reads_pynx_written_cxi():
    s = read_cxi(os.path.join(GOLDEN, "pynx_small.cxi"))
    nz, ny, nx = 4, 4, 6
    assert s.counts.shape == (nz, ny, nx) and s.counts.dtype == np.uint16
    for i, v in enumerate(s.counts.ravel()):
        f, p = i // (ny * nx), i % (ny * nx)
        want = MASKED if p == nx + 2 or (f, p) == (2, 3 * nx + 1) else i * 37 % 500
        assert v == want, i
    assert (s.distance, s.detector_pixel) == (1.2, 75e-6)
    assert abs(s.wavelength / 1.5e-10 - 1.0) < 1e-12
    for i in range(nz):
        x = float(np.float32(i * 1.1e-7 + 1e-9 / 3.0))
        y = float(np.float32(-i * 0.7e-7))
        assert (s.x[i], s.y[i]) == (x, y)


@pytest.mark.parametrize("kind", ["single", "double"])
def test_reads_ptypy_written_ptyr(kind):
    r = read_ptyr(os.path.join(GOLDEN, f"ptypy_small_{kind}.ptyr"))
    assert r["object"].shape == (1, 10, 11) and r["probe"].shape == (2, 8, 8)
    y, x = np.mgrid[:10, :11].astype(float)
    np.testing.assert_array_equal(r["object"][0], (y - 0.25 * x) + 1j * (0.5 * y + x))
    m, y, x = np.mgrid[:2, :8, :8].astype(float)
    np.testing.assert_array_equal(r["probe"], (m + 0.5 * y) + 1j * (0.25 * m - x))
    assert (r["psize"], r["origin"]) == ((1.5e-8, 2.5e-8), (-3e-7, 4e-7))


def test_refuses_what_it_cannot_read(tmp_path):
    with pytest.raises(PtybError, match="cannot open"):
        read_cxi(tmp_path / "absent.cxi")
    junk = tmp_path / "junk.cxi"
    junk.write_bytes(b"not an hdf5 file" * 64)
    with pytest.raises(PtybError, match="not an HDF5 file"):
        read_cxi(junk)
    # a file of the other layout: the PtyPy file has no CXI entry
    with pytest.raises(PtybError, match="no member entry_1"):
        read_cxi(os.path.join(GOLDEN, "ptypy_small_single.ptyr"))
    # a truncated file: every address is checked against its end
    cut = tmp_path / "cut.cxi"
    cut.write_bytes(open(os.path.join(GOLDEN, "pynx_small.cxi"), "rb").read()[:4096])
    with pytest.raises(PtybError):
        read_cxi(cut)
