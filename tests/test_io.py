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


FUZZ = r"""
import sys
import numpy as np
from ptyrs_b200 import PtybError
from ptyrs_b200.io import read_cxi, read_ptyr
src, out, seed, n = sys.argv[1], sys.argv[2], int(sys.argv[3]), int(sys.argv[4])
reader = read_ptyr if src.endswith(".ptyr") else read_cxi
blob = open(src, "rb").read()
rng = np.random.default_rng(seed)
for it in range(n):
    b = bytearray(blob)
    if it % 3 == 0:
        b = b[: rng.integers(8, len(b))]
    for _ in range(rng.integers(1, 12)):
        b[rng.integers(0, len(b))] = rng.integers(0, 256)
    open(out, "wb").write(bytes(b))
    try:
        reader(out)
    except PtybError:
        pass
"""


@pytest.mark.parametrize("name", ["pynx_small.cxi", "ptypy_small_double.ptyr"])
def test_damaged_files_are_refused_not_crashed(tmp_path, name):
    """Seeded truncations and byte flips of the fixtures, read in a child process: each read
    returns its scan or raises PtybError, and the process ends normally within the time limit
    (a fault, an unbounded allocation or a cycle in the file's structure would fail here)."""
    import subprocess
    import sys
    env = dict(os.environ, PYTHONPATH=os.path.dirname(GOLDEN.rstrip("/")).rsplit("/", 1)[0])
    r = subprocess.run([sys.executable, "-c", FUZZ, os.path.join(GOLDEN, name),
                        str(tmp_path / "damaged"), "7", "400"], env=env, timeout=300,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
