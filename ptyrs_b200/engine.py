"""Python face of the B200 engine, mirroring the reference binding `ptyrs.Scan` and
`ptyrs.GpuPtycho` (physwkim/ptyrs ptyrs-py/src/lib.rs:435-463, ptyrs-py/src/gpu.rs:28-267):
numpy arrays in and out, every call through the C ABI of `libptyb200.so`."""
import ctypes

import numpy as np

from . import _lib

STATUS = {0: "ok", 1: "invalid", 2: "gpu", 3: "aborted"}
ALGORITHMS = {0: "ap", 1: "dm", 2: "raar", 3: "rpie", 4: "ml", 5: "bh", 6: "lsqml"}
COSTS = {"poisson": 0, "amplitude": 1, "gaussian": 1}


class PtybError(RuntimeError):
    """A refused or failed engine call: `status` is "invalid", "gpu" or "aborted"."""

    def __init__(self, status, message):
        super().__init__(f"{status}: {message}")
        self.status = status


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Scan:
    """A far-field scan: counts `[nframe, ny, nx]` in detector order (uint16 with 65535 masked,
    or float32/float64 with negative values masked), positions `y`, `x` in metres, geometry in
    metres."""

    def __init__(self, counts, y, x, wavelength, distance, detector_pixel):
        counts = np.asarray(counts)
        if counts.ndim != 3:
            raise ValueError("counts must be [nframe, ny, nx]")
        if counts.dtype == np.uint16:
            kind = 0
        elif counts.dtype == np.float32:
            kind = 1
        else:
            counts, kind = counts.astype(np.float64), 2
        self.counts = np.ascontiguousarray(counts)
        self.kind = kind
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        if self.y.shape != (counts.shape[0],) or self.x.shape != (counts.shape[0],):
            raise ValueError("one y and one x position per frame")
        self.wavelength, self.distance, self.detector_pixel = wavelength, distance, detector_pixel

    def _struct(self):
        n, ny, nx = self.counts.shape
        return _lib.Scan(n, ny, nx, self.kind, self.counts.ctypes.data_as(ctypes.c_void_p),
                         _dptr(self.y), _dptr(self.x), self.wavelength, self.distance,
                         self.detector_pixel)


class GpuPtycho:
    """The GPU reconstruction state of a scan on CUDA device `device`: `object` complex
    `[1, nyo, nxo]`, `probe` complex `[nprobe, ny, nx]`.

    With `gaps` (the nslice - 1 slice spacings in metres, reference `Optics::with_slices`),
    `obj` is pty-chi's multislice object `[nslice, nyo, nxo]` in the order the wave crosses the
    slices; `object()` / `set_object()` then read and replace slice 0 and `objects()` returns
    every slice, as the reference's `GpuPtycho::with_slices` does."""

    def __init__(self, scan, obj, probe, device=0, stack_size=0, cluster=0, gaps=None):
        self._lib = _lib.load()
        obj = np.ascontiguousarray(obj, dtype=np.complex128)
        probe = np.ascontiguousarray(probe, dtype=np.complex128)
        if obj.ndim != 3 or probe.ndim != 3:
            raise ValueError("object must be [nobj, nyo, nxo] and probe [nprobe, ny, nx]")
        self._nslice = 1 if gaps is None else obj.shape[0]
        if gaps is not None and len(gaps) != self._nslice - 1:
            raise ValueError(f"{obj.shape[0]} slices need {obj.shape[0] - 1} gaps, got {len(gaps)}")
        self._obj_shape = (1,) + obj.shape[1:] if gaps is not None else obj.shape
        self._probe_shape = probe.shape
        self._nframe = scan.counts.shape[0]
        st = scan._struct()
        opts = _lib.Options(device, stack_size, cluster)
        h = ctypes.c_void_p()
        if gaps is None:
            rc = self._lib.ptyb_create(ctypes.byref(st), _dptr(obj.view(np.float64)),
                                       obj.shape[0], obj.shape[1], obj.shape[2],
                                       _dptr(probe.view(np.float64)), probe.shape[0],
                                       ctypes.byref(opts), ctypes.byref(h))
        else:
            g = np.ascontiguousarray(gaps, dtype=np.float64).reshape(-1)
            rc = self._lib.ptyb_create_slices(ctypes.byref(st), _dptr(obj.view(np.float64)),
                                              obj.shape[0], _dptr(g) if len(g) else None,
                                              obj.shape[1], obj.shape[2],
                                              _dptr(probe.view(np.float64)), probe.shape[0],
                                              ctypes.byref(opts), ctypes.byref(h))
        if rc != 0:
            raise PtybError(STATUS.get(rc, rc), self._lib.ptyb_last_error(None).decode())
        self._h = h

    @classmethod
    def _adopt(cls, h, obj_shape, probe_shape, nframe):
        """A GpuPtycho that owns the single-slice handle `h` made by another entry point (the
        live ring's ptyb_live_handle)."""
        self = cls.__new__(cls)
        self._lib = _lib.load()
        self._nslice = 1
        self._obj_shape = tuple(obj_shape)
        self._probe_shape = tuple(probe_shape)
        self._nframe = nframe
        self._h = h
        return self

    def _check(self, rc):
        if rc != 0:
            raise PtybError(STATUS.get(rc, rc), self._lib.ptyb_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ptyb_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # Algorithms ---------------------------------------------------------------------------
    def rpie(self, nepoch, obj_step=1.0, probe_step=1.0, obj_alpha=0.1, probe_alpha=0.1,
             batch_size=100, calc_llk=0, seed=7):
        """rPIE epochs (reference `RpieParams` keywords; a step of None holds that array)."""
        p = _lib.RpieParams(obj_step is not None, probe_step is not None,
                            0.0 if obj_step is None else obj_step,
                            0.0 if probe_step is None else probe_step, obj_alpha, probe_alpha,
                            batch_size, calc_llk, seed)
        self._check(self._lib.ptyb_rpie(self._h, ctypes.byref(p), nepoch))

    def lsqml(self, nepoch, calc_llk=0, batch_size=256, cost="poisson", seed=7):
        """LSQML epochs without probe variation, fresh preconditioner per call."""
        p = _lib.LsqmlParams(batch_size, COSTS[cost], seed)
        self._check(self._lib.ptyb_lsqml(self._h, ctypes.byref(p), nepoch, calc_llk))

    def ml(self, ncycle, update_object=True, update_probe=False, calc_llk=0,
           zero_phase_ramp=True):
        """Poisson ML conjugate-gradient cycles (reference `MlParams`)."""
        p = _lib.MlParams(update_object, update_probe, calc_llk, zero_phase_ramp)
        self._check(self._lib.ptyb_ml(self._h, ctypes.byref(p), ncycle))

    def bh(self, nepoch, batch_size, probe_rho=0.01, seed=7, calc_llk=0, position_rho=0.1):
        """pty-chi's BH on the amplitude cost (reference `GpuPtycho::bh`): `nepoch` epochs from
        a fresh run; one batch of every frame runs conjugate directions across epochs. With
        `set_positions` every frame's probe is moved by its offset; refined offsets are BH
        variables too (their gradient scaled by `position_rho²`, stepped by 0.3·α·D_d)."""
        p = _lib.BhParams(batch_size, 0, probe_rho, position_rho, seed)
        self._check(self._lib.ptyb_bh(self._h, ctypes.byref(p), nepoch, calc_llk))

    def bh_steps(self):
        """The last BH epoch's steps: dicts of batch, count, beta, alpha, top, bottom."""
        n = self._lib.ptyb_bh_steps_len(self._h)
        out = (_lib.BhStep * max(n, 1))()
        self._check(self._lib.ptyb_bh_steps(self._h, out, n))
        return [dict(batch=s.batch, count=s.count, beta=s.beta, alpha=s.alpha, top=s.top,
                     bottom=s.bottom) for s in out[:n]]

    @staticmethod
    def _inertia(x):
        return (0, 0.0) if x is None else (1, float(x))

    def ap(self, ncycle, obj_inertia=0.01, probe_inertia=None, calc_llk=0, zero_phase_ramp=True):
        """PyNX AP cycles (reference `ApParams`); an inertia of None leaves that array fixed."""
        (uo, oi), (up, pi) = self._inertia(obj_inertia), self._inertia(probe_inertia)
        p = _lib.ApParams(uo, up, oi, pi, calc_llk, zero_phase_ramp)
        self._check(self._lib.ptyb_ap(self._h, ctypes.byref(p), ncycle))

    def dm(self, ncycle, obj_inertia=0.01, probe_inertia=0.001, alpha=0.02, loop_obj_probe=1,
           calc_llk=0, zero_phase_ramp=True):
        """PyNX DM cycles (reference `DmParams`)."""
        (uo, oi), (up, pi) = self._inertia(obj_inertia), self._inertia(probe_inertia)
        p = _lib.DmParams(uo, up, oi, pi, alpha, loop_obj_probe, calc_llk, zero_phase_ramp)
        self._check(self._lib.ptyb_dm(self._h, ctypes.byref(p), ncycle))

    def raar(self, ncycle, obj_inertia=0.01, probe_inertia=0.001, beta=0.9, loop_obj_probe=1,
             calc_llk=0, zero_phase_ramp=True):
        """PyNX RAAR cycles (reference `RaarParams`)."""
        (uo, oi), (up, pi) = self._inertia(obj_inertia), self._inertia(probe_inertia)
        p = _lib.RaarParams(uo, up, oi, pi, beta, loop_obj_probe, calc_llk, zero_phase_ramp)
        self._check(self._lib.ptyb_raar(self._h, ctypes.byref(p), ncycle))

    # State --------------------------------------------------------------------------------
    def llk(self):
        out = _lib.Llk()
        self._check(self._lib.ptyb_get_llk(self._h, ctypes.byref(out)))
        return dict(poisson=out.poisson, gaussian=out.gaussian, euclidian=out.euclidian,
                    nb_photons_calc=out.nb_photons_calc)

    def gradients(self, obj=True, probe=True, positions=True):
        """The Poisson LLK sum `loss` of the current estimate and its gradients through the
        hand-written adjoint: `object` and `probe` as 2·∂L/∂X* (the complex gradient torch
        uses; on a multislice handle `object` holds every slice's), `positions` ∂L/∂d
        `[nframe, 2]` (needs `set_positions`, single slice); a dict, None for what is not
        asked."""
        loss = ctypes.c_double()
        oshape = ((self._nslice,) + tuple(self._obj_shape[1:]) if self._nslice > 1
                  else self._obj_shape)
        go = np.empty(oshape, np.complex128) if obj else None
        gp = np.empty(self._probe_shape, np.complex128) if probe else None
        gd = np.empty((self._nframe, 2), np.float64) if positions else None
        ptr = lambda a, view=True: None if a is None else _dptr(a.view(np.float64) if view else a)
        self._check(self._lib.ptyb_gradients(self._h, ctypes.byref(loss), ptr(go), ptr(gp),
                                             ptr(gd, False)))
        return dict(loss=loss.value, object=go, probe=gp, positions=gd)

    def gradients_device(self, d_obj, d_probe, positions=False):
        """`gradients` with the object and probe gradients written as complex64 into device
        buffers (`data_ptr()` of contiguous complex64 CUDA tensors of the handle's device, or
        None to skip): returns `(loss, positions gradient or None)`."""
        loss = ctypes.c_double()
        gd = np.empty((self._nframe, 2), np.float64) if positions else None
        self._check(self._lib.ptyb_gradients_device(
            self._h, ctypes.byref(loss), d_obj, d_probe, None if gd is None else _dptr(gd)))
        return loss.value, gd

    def set_object_device(self, ptr, nobj, nyo, nxo):
        """The object (slice 0) from complex64 device memory `ptr` of the handle's device,
        `[nobj, nyo, nxo]` (reference `GpuPtycho::set_object_device`)."""
        self._check(self._lib.ptyb_set_object_device(self._h, nobj, nyo, nxo, ptr))

    def set_objects_device(self, ptr, nslice, nyo, nxo):
        """Every slice from complex64 device memory `ptr`, `[nslice, nyo, nxo]`."""
        self._check(self._lib.ptyb_set_objects_device(self._h, nslice, nyo, nxo, ptr))

    def set_probe_device(self, ptr, nprobe, ny, nx):
        """The probe from complex64 device memory `ptr`, `[nprobe, ny, nx]`."""
        self._check(self._lib.ptyb_set_probe_device(self._h, nprobe, ny, nx, ptr))

    def forward_intensity(self, frames=None):
        """Model intensity `Σ_modes |Ψ|²` `[len(frames), ny, nx]` of the current estimate, in the
        FFT-shifted detector layout (zero frequency at [0, 0])."""
        frames = np.arange(self._nframe, dtype=np.int32) if frames is None else np.ascontiguousarray(frames, np.int32)
        n = self._probe_shape[-1]
        out = np.empty((len(frames), n, n), np.float32)
        self._check(self._lib.ptyb_forward_intensity(
            self._h, frames.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(frames),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def forward_intensity_noalloc(self, frames=None):
        """`forward_intensity` through the entry point that allocates no device memory (its
        scratch is a fixed 32 MiB device array shared by every call in the process; calls that
        run on the GPU at the same time race on it)."""
        frames = np.arange(self._nframe, dtype=np.int32) if frames is None else np.ascontiguousarray(frames, np.int32)
        n = self._probe_shape[-1]
        out = np.empty((len(frames), n, n), np.float32)
        self._check(self._lib.ptyb_forward_intensity_noalloc(
            self._h, frames.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(frames),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def object(self):
        out = np.empty(self._obj_shape, np.complex128)
        self._check(self._lib.ptyb_get_object(self._h, _dptr(out.view(np.float64))))
        return out

    def nslice(self):
        """The handle's object slices."""
        return self._lib.ptyb_nslice(self._h)

    def objects(self):
        """Every object slice `[nslice, nyo, nxo]` (reference `GpuPtycho::objects`)."""
        out = np.empty((self._nslice,) + tuple(self._obj_shape[1:]), np.complex128)
        self._check(self._lib.ptyb_get_objects(self._h, _dptr(out.view(np.float64))))
        return out

    def set_objects(self, objs):
        """Replaces every object slice `[nslice, nyo, nxo]`."""
        objs = np.ascontiguousarray(objs, dtype=np.complex128).reshape(
            (self._nslice,) + tuple(self._obj_shape[1:]))
        self._check(self._lib.ptyb_set_objects(self._h, _dptr(objs.view(np.float64))))

    def probe(self):
        out = np.empty(self._probe_shape, np.complex128)
        self._check(self._lib.ptyb_get_probe(self._h, _dptr(out.view(np.float64))))
        return out

    def set_object(self, obj):
        obj = np.ascontiguousarray(obj, dtype=np.complex128).reshape(self._obj_shape)
        self._check(self._lib.ptyb_set_object(self._h, _dptr(obj.view(np.float64))))

    def set_probe(self, probe):
        probe = np.ascontiguousarray(probe, dtype=np.complex128).reshape(self._probe_shape)
        self._check(self._lib.ptyb_set_probe(self._h, _dptr(probe.view(np.float64))))

    def set_positions(self, offsets=None, refine=True):
        """Per-frame sub-pixel offsets `[nframe, 2]` (dy, dx) in object pixels, modelled by
        moving each frame's probe and refined by LSQML and ML when `refine`; None clears
        them."""
        if offsets is None:
            self._check(self._lib.ptyb_set_positions(self._h, None, 0))
            return
        d = np.ascontiguousarray(offsets, np.float64).reshape(self._nframe, 2)
        self._check(self._lib.ptyb_set_positions(self._h, _dptr(d), int(refine)))

    def positions(self):
        """The offsets `[nframe, 2]` as the last step left them (zeros when none are set)."""
        out = np.empty((self._nframe, 2), np.float64)
        self._check(self._lib.ptyb_get_positions(self._h, _dptr(out)))
        return out

    def corners(self):
        out = np.empty((self._nframe, 2), np.int32)
        self._check(self._lib.ptyb_corners(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return out

    def history(self):
        n = self._lib.ptyb_history_len(self._h)
        recs = (_lib.LlkRecord * max(n, 1))()
        self._check(self._lib.ptyb_history(self._h, recs, n))
        recs = recs[:n]
        return dict(cycle=np.array([r.cycle for r in recs], np.int64),
                    algorithm=[ALGORITHMS[r.algorithm] for r in recs],
                    poisson=np.array([r.llk.poisson for r in recs]),
                    gaussian=np.array([r.llk.gaussian for r in recs]),
                    euclidian=np.array([r.llk.euclidian for r in recs]),
                    nb_photons_calc=np.array([r.llk.nb_photons_calc for r in recs]))

    def cycle(self):
        return int(self._lib.ptyb_cycle(self._h))

    def lsqml_steps(self):
        """The last LSQML epoch's steps: per batch, its frames and their a_far, a_obj, a_probe."""
        n = self._lib.ptyb_lsqml_steps_len(self._h)
        buf = (_lib.LsqmlStep * max(n, 1))()
        self._check(self._lib.ptyb_lsqml_steps(self._h, buf, n))
        extra = np.zeros((n, self._nslice - 1))
        if self._nslice > 1 and n:
            self._check(self._lib.ptyb_lsqml_slice_steps(self._h, _dptr(extra)))
        steps = []
        for i, s in enumerate(buf[:n]):
            if not steps or steps[-1]["batch"] != s.batch:
                steps.append(dict(batch=s.batch, frames=[], a_far=[], a_probe=[],
                                  a_obj=[] if self._nslice == 1 else
                                  [[] for _ in range(self._nslice)]))
            st = steps[-1]
            st["frames"].append(s.frame)
            st["a_far"].append(s.a_far)
            st["a_probe"].append(s.a_probe)
            if self._nslice == 1:
                st["a_obj"].append(s.a_obj)
            else:
                st["a_obj"][0].append(s.a_obj)
                for k in range(1, self._nslice):
                    st["a_obj"][k].append(extra[i, k - 1])
        return steps

    def synchronize(self):
        self._check(self._lib.ptyb_synchronize(self._h))

    def set_probe_variation(self, eigenmodes, weights, refine_weights=True, intensity=None,
                            refine_intensity=True):
        """pty-chi's OPR probe variation of mode 0 for the LSQML calls that follow (reference
        `ProbeVariation`): eigenmodes `[k, ny, nx]`, weights `[nframe, k]`, optional main-mode
        weights `[nframe]`; `eigenmodes=None` returns to the shared probe."""
        if eigenmodes is None:
            self._check(self._lib.ptyb_set_probe_variation(self._h, None, 0, None, 0, None, 0))
            self._opr = None
            return
        u = np.ascontiguousarray(eigenmodes, np.complex128)
        w = np.ascontiguousarray(weights, np.float64).reshape(self._nframe, len(u))
        c = None if intensity is None else np.ascontiguousarray(intensity, np.float64)
        self._check(self._lib.ptyb_set_probe_variation(
            self._h, _dptr(u.view(np.float64)), len(u), _dptr(w), int(refine_weights),
            None if c is None else _dptr(c), int(refine_intensity)))
        self._opr = (u.shape, c is not None)

    def probe_variation(self):
        """`(eigenmodes, weights, intensity)` of the probe variation (intensity None when not
        modelled), or None without one."""
        if getattr(self, "_opr", None) is None:
            return None
        shape, has_c = self._opr
        u = np.empty(shape, np.complex128)
        w = np.empty((self._nframe, shape[0]), np.float64)
        c = np.empty(self._nframe, np.float64) if has_c else None
        self._check(self._lib.ptyb_get_probe_variation(
            self._h, _dptr(u.view(np.float64)), _dptr(w), None if c is None else _dptr(c)))
        return u, w, c

    def set_timing(self, on=True):
        """Per-kernel device timing of every later launch (resets the totals)."""
        self._check(self._lib.ptyb_set_timing(self._h, int(on)))

    def kernel_times(self):
        """`{kernel: (total ms, launches)}` of the launches timed since `set_timing`."""
        k = self._lib.ptyb_kernel_kinds()
        ms = (ctypes.c_double * k)()
        n = (ctypes.c_int64 * k)()
        self._check(self._lib.ptyb_kernel_times(self._h, ms, n, k))
        return {self._lib.ptyb_kernel_name(i).decode(): (ms[i], n[i]) for i in range(k) if n[i]}

    def kernel_frames(self):
        """`{kernel: frames}` the launches timed since `set_timing` processed (per-frame
        kernels only)."""
        k = self._lib.ptyb_kernel_kinds()
        f = (ctypes.c_int64 * k)()
        self._check(self._lib.ptyb_kernel_frames(self._h, f, k))
        return {self._lib.ptyb_kernel_name(i).decode(): f[i] for i in range(k) if f[i]}

    def last_call_ms(self):
        """Device time of the last algorithm call (CUDA events on the engine's stream)."""
        return float(self._lib.ptyb_last_call_ms(self._h))

    def launches(self):
        """Kernels this handle has launched since it was made."""
        return int(self._lib.ptyb_launches(self._h))


def batch_run(handles, rpie_epochs=30, lsqml_epochs=30, calc_llk=0, rpie=None, lsqml=None):
    """Independent scans at once (`ptyb_batch_run`): `rpie_epochs` rPIE epochs then
    `lsqml_epochs` LSQML epochs on every `GpuPtycho` of `handles`, each on its own stream from
    its own host thread. `rpie` / `lsqml` hold the keywords of `GpuPtycho.rpie` / `.lsqml`
    (steps, alphas, batch size, cost, seed). Returns the batch's device time in ms; raises
    PtybError with the first failing handle's message (the others keep their results)."""
    if not handles:
        raise ValueError("no handles")
    r = dict(obj_step=1.0, probe_step=1.0, obj_alpha=0.1, probe_alpha=0.1, batch_size=100,
             seed=7)
    r.update(rpie or {})
    q = dict(batch_size=256, cost="poisson", seed=7)
    q.update(lsqml or {})
    rp = _lib.RpieParams(r["obj_step"] is not None, r["probe_step"] is not None,
                         0.0 if r["obj_step"] is None else r["obj_step"],
                         0.0 if r["probe_step"] is None else r["probe_step"], r["obj_alpha"],
                         r["probe_alpha"], r["batch_size"], calc_llk, r["seed"])
    lp = _lib.LsqmlParams(q["batch_size"], COSTS[q["cost"]], q["seed"])
    n = len(handles)
    hs = (ctypes.c_void_p * n)(*[h._h for h in handles])
    status = (ctypes.c_int32 * n)()
    ms = ctypes.c_float(-1.0)
    lib = handles[0]._lib
    rc = lib.ptyb_batch_run(hs, n, ctypes.byref(rp), rpie_epochs, ctypes.byref(lp), lsqml_epochs,
                            calc_llk, status, ctypes.byref(ms))
    if rc != 0:
        bad = next((i for i in range(n) if status[i] != 0), None)
        msg = lib.ptyb_last_error(hs[bad]).decode() if bad is not None else "invalid batch"
        raise PtybError(STATUS.get(rc, rc), f"handle {bad}: {msg}")
    return float(ms.value)


def random_batches(nframe, size, seed, epoch):
    """The reference's seeded mini-batches of one epoch from the native host code, as a list of
    sorted frame lists."""
    lib = _lib.load()
    order = np.empty(nframe, np.int32)
    rc = lib.ptyb_random_batches(nframe, size, seed, epoch,
                                 order.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    if rc != 0:
        raise PtybError(STATUS.get(rc, rc), "random_batches")
    return [order[s:s + size].tolist() for s in range(0, nframe, size)]


def view_corners(y, x, pixel, frame, obj):
    """Window corners `[P, 2]` (oy, ox) of positions in metres from the native host code."""
    lib = _lib.load()
    y = np.ascontiguousarray(y, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty((len(y), 2), np.int32)
    rc = lib.ptyb_view_corners(_dptr(y), _dptr(x), len(y), pixel[0], pixel[1], frame[0],
                               frame[1], obj[0], obj[1],
                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    if rc != 0:
        raise PtybError(STATUS.get(rc, rc), lib.ptyb_last_error(None).decode())
    return out
