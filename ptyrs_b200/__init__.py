"""ptyrs_b200: the per-iteration ptychography reconstruction hot path of physwkim/ptyrs
(rPIE, LSQML, ML with their FFT projections and object/probe updates) as hand-written sm_100a
CUDA kernels behind a C ABI (`include/ptyb200.h`, `libptyb200.so`), with a numpy front end that
mirrors the reference's `ptyrs.Scan` / `ptyrs.GpuPtycho` binding."""
from .engine import GpuPtycho, PtybError, Scan, batch_run  # noqa: F401
