"""Live ingestion into the device: the reference's pinned host ring and uploader
(physwkim/ptyrs ptyrs/src/live/ring.rs:1-31) with its position table by uid
(ptyrs/src/live/pos.rs), through the C ABI's ptyb_live_* entry points.

Workers `reserve` a ring slot, fill the returned pinned frame (detector order) and `commit`
it with the frame's uid; positions come by uid through `position`, in any order with the
frames. The library's uploader thread lands frames in sequence order once their positions are
in, into a device store (converted there as `GpuPtycho` converts counts); `gpu_ptycho` makes a
reconstruction state over the frames landed so far."""
import ctypes

import numpy as np

from . import _lib
from .engine import STATUS, GpuPtycho, PtybError, _dptr

KINDS = {"u16": (0, np.uint16, ctypes.c_uint16), "f32": (1, np.float32, ctypes.c_float)}


class LiveRing:
    """A ring of `slots` frames of `n`×`n` counts (`counts` "u16", 65535 masked, or "f32",
    negative masked) feeding a device store of `capacity` frames on CUDA device `device`.
    A frame without its position is dropped `pos_wait_s` after its commit, or as soon as a
    worker needs its slot; runs of at most `batch` frames go to the device in one copy."""

    def __init__(self, n, wavelength, distance, detector_pixel, slots=64, capacity=4096,
                 counts="u16", pos_wait_s=1.0, batch=32, device=0):
        self._lib = _lib.load()
        kind, self._dtype, self._ctype = KINDS[counts]
        self.n, self.capacity = n, capacity
        p = _lib.LiveParams(device, n, kind, slots, capacity, batch, wavelength, distance,
                            detector_pixel, int(round(pos_wait_s * 1e9)))
        h = ctypes.c_void_p()
        rc = self._lib.ptyb_live_create(ctypes.byref(p), ctypes.byref(h))
        if rc != 0:
            raise PtybError(STATUS.get(rc, rc), self._lib.ptyb_live_last_error(None).decode())
        self._h = h

    def _check(self, rc):
        if rc != 0:
            raise PtybError(STATUS.get(rc, rc), self._lib.ptyb_live_last_error(self._h).decode())

    def reserve(self):
        """(seq, frame): the next sequence number and its pinned host frame `[n, n]` to fill;
        blocks while the ring is full."""
        seq, ptr = ctypes.c_int64(), ctypes.c_void_p()
        self._check(self._lib.ptyb_live_reserve(self._h, ctypes.byref(seq), ctypes.byref(ptr)))
        buf = (self._ctype * (self.n * self.n)).from_address(ptr.value)
        return seq.value, np.ctypeslib.as_array(buf).reshape(self.n, self.n)

    def commit(self, seq, uid):
        self._check(self._lib.ptyb_live_commit(self._h, seq, uid))

    def put(self, uid, frame):
        """Reserve, copy `frame` in and commit it as `uid`."""
        seq, buf = self.reserve()
        buf[...] = frame
        self.commit(seq, uid)
        return seq

    def position(self, uid, y, x):
        """The position (metres) of frame `uid`; a coordinate that is not finite or exceeds
        1e10 in magnitude marks the frame as having no scan position."""
        self._check(self._lib.ptyb_live_position(self._h, uid, y, x))

    def flush(self, timeout_s=10.0):
        """Waits until every committed frame has landed or dropped and its copy completed."""
        self._check(self._lib.ptyb_live_flush(self._h, int(timeout_s * 1000)))

    def stats(self):
        st = _lib.LiveStats()
        self._check(self._lib.ptyb_live_get_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.LiveStats._fields_}

    def landed(self):
        """(uids, y, x) of the landed frames in landing order."""
        n = self.stats()["landed"]
        uids = np.empty(max(n, 1), np.int64)
        y, x = np.empty(max(n, 1)), np.empty(max(n, 1))
        got = self._lib.ptyb_live_landed(self._h, uids.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                         _dptr(y), _dptr(x), n)
        if got < 0:
            self._check(got)
        return uids[:got], y[:got], x[:got]

    def gpu_ptycho(self, obj, probe, stack_size=0, cluster=0):
        """A `GpuPtycho` over the frames landed and converted so far (object `[1, nyo, nxo]`,
        probe `[nprobe, n, n]`), frames in landing order."""
        obj = np.ascontiguousarray(obj, dtype=np.complex128)
        probe = np.ascontiguousarray(probe, dtype=np.complex128)
        if obj.ndim != 3 or obj.shape[0] != 1 or probe.ndim != 3:
            raise ValueError("object must be [1, nyo, nxo] and probe [nprobe, n, n]")
        opts = _lib.Options(0, stack_size, cluster)
        h, nframe = ctypes.c_void_p(), ctypes.c_int32()
        self._check(self._lib.ptyb_live_handle(self._h, _dptr(obj.view(np.float64)), obj.shape[1],
                                               obj.shape[2], _dptr(probe.view(np.float64)),
                                               probe.shape[0], ctypes.byref(opts),
                                               ctypes.byref(h), ctypes.byref(nframe)))
        return GpuPtycho._adopt(h, obj.shape, probe.shape, nframe.value)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ptyb_live_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
