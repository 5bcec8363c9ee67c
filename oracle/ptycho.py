"""rPIE, ML (Poisson conjugate gradient), AP, DM and RAAR in float64 (oracle restatement, test
infrastructure only).

Follows physwkim/ptyrs `ptyrs/src/engine/ptycho.rs` (`Ptycho`) for the far-field and
planar near-field optics of a single object slice; rPIE, ML, AP, DM and RAAR also under
`Features::position`'s sub-pixel offsets with Patch sampling (`engine/features.rs`, `Shifted`).
"""
import numpy as np

from . import ops
from .base import AddrTable, Observed, fftshift2, pynx_preprocess, random_batches


class Shifted:
    """`Features::position`'s model of `probe` on `views` under Patch sampling
    (engine/features.rs:558-1025): every view's wave `W = T_d(q·P)`, its probe mode with the
    exit phase moved by its frame's offset `d` on the periodic grid, takes the place of `q·P`,
    and the window is the integer one. Planes are kept in the natural layout here; the
    reference's shifted layout commutes with the move."""

    def __init__(self, views, probe, quad, offsets):
        self.views = views
        self.quad = np.ones(probe.shape[-2:]) if quad is None else quad
        self.offsets = np.asarray(offsets, np.float64)
        self.probe = probe
        self.pidx = views["probe"].astype(np.int64)
        self.frames = views["frame"].astype(np.int64)
        moved = {}
        waves = np.empty((len(views),) + probe.shape[-2:], np.complex128)
        for k, (p, f) in enumerate(zip(self.pidx, self.frames)):
            if f not in moved:
                moved[f] = self.quad * ops.move_planes(probe, self.quad, self.offsets[f])
            waves[k] = moved[f][p]
        self.waves = waves

    def _windows(self, obj):
        ny, nx = self.waves.shape[-2:]
        return ops.windows(self.views, obj, ny, nx)

    def to_psi(self, obj):
        """`psi[k] = W[k]·O[win_k]` in the shifted exit layout (features.rs:803-818)."""
        return fftshift2(self.waves * self._windows(obj))

    def derivatives(self, obj, axis):
        """`O[win]·∂W/∂d[axis]` per view, shifted layout (features.rs:964-990)."""
        win = self._windows(obj)
        out = np.empty_like(self.waves)
        cache = {}
        for k, (p, f) in enumerate(zip(self.pidx, self.frames)):
            if f not in cache:
                cache[f] = self.quad * ops.move_planes(self.probe, self.quad, self.offsets[f],
                                                       axes=(axis,))
            out[k] = win[k] * cache[f][p]
        return fftshift2(out)

    def accumulate_obj(self, obj_shape, psi):
        """`num += psi·conj(W)`, `norm += |W|²` on each window in view order
        (features.rs:855-890)."""
        ny, nx = self.waves.shape[-2:]
        num = np.zeros(obj_shape, np.complex128)
        norm = np.zeros(obj_shape, np.float64)
        w = fftshift2(psi)
        for k, v in enumerate(self.views):
            oy, ox, o = int(v["oy"]), int(v["ox"]), int(v["obj"])
            num[o, oy:oy + ny, ox:ox + nx] += w[k] * np.conj(self.waves[k])
            norm[o, oy:oy + ny, ox:ox + nx] += np.abs(self.waves[k]) ** 2
        return num, norm

    def accumulate_probe(self, obj, probe_shape, psi):
        """Through the move's adjoint (features.rs:897-957): per probe mode
        `num = conj(q)·Σ_f IDFT(DFT(Y_f)·conj(exp(−2πi f·d_f)))`, `Y_f = Σ conj(O[win])·psi`
        over frame f's views of that mode, the spectra summed frame by frame;
        `norm = Σ|O[win]|²`."""
        w = fftshift2(psi)
        win = self._windows(obj)
        spectrum = np.zeros(probe_shape, np.complex128)
        norm = np.zeros(probe_shape, np.float64)
        k = 0
        nv = len(self.views)
        while k < nv:
            f = self.frames[k]
            y = np.zeros(probe_shape, np.complex128)
            while k < nv and self.frames[k] == f:
                p = self.pidx[k]
                y[p] += np.conj(win[k]) * w[k]
                norm[p] += np.abs(win[k]) ** 2
                k += 1
            e, _ = ops.translation(probe_shape[-2:], self.offsets[f])
            spectrum += ops.fft2(y) * np.conj(e)
        return np.conj(self.quad) * ops.ifft2(spectrum), norm

    def psi_to_obj_probe(self, obj, probe, psi, obj_inertia, probe_inertia):
        """psi_to_obj_probe under the move (features.rs:653-725), both from the arrays on entry;
        returns `(object, probe)`. The probe takes the first conjugate-gradient step of
        `min ‖psi − A·P'‖² + reg·‖P' − P‖²` preconditioned by `D = Σ|O|² + reg` per mode:
        `s = g / D` with `g = A^H(psi − A·P)`, `P += α·s`, `α = <g, s> / (‖A·s‖² + reg·‖s‖²)`
        where `<g, s> > 0`; the object takes `blend` of its sums under this (old) probe's
        waves."""
        new_obj, new_probe = obj, probe
        if probe_inertia is not None:
            residual = psi - self.to_psi(obj)
            num, norm = self.accumulate_probe(obj, probe.shape, residual)
            reg = max(0.0, float(norm.max())) * probe_inertia
            d = np.maximum(norm + reg, 1e-12)
            slope = (np.abs(num) ** 2 / d).sum(axis=(1, 2))
            step = num / d
            curvature = reg * (np.abs(step) ** 2).sum(axis=(1, 2))
            moved = fftshift2(Shifted(self.views, step, self.quad, self.offsets).to_psi(obj))
            for k, p in enumerate(self.pidx):
                curvature[p] += float((np.abs(moved[k]) ** 2).sum())
            new_probe = probe.copy()
            for m in range(probe.shape[0]):
                if slope[m] > 0.0:
                    new_probe[m] = probe[m] + step[m] * (slope[m] / curvature[m])
        if obj_inertia is not None:
            num, norm = self.accumulate_obj(obj.shape, psi)
            new_obj = _blend(obj, num, norm, obj_inertia)
        return new_obj, new_probe

    def position_sums(self, obj, psi, nframe):
        """Per frame `[num, den]` (features.rs:992-1025): `num[a] = Re Σ conj(x − O·W)·∂psi_a`,
        `den[a] = Σ|∂psi_a|²` over the frame's views and pixels, `x` the new exit waves."""
        c = psi - self.to_psi(obj)
        sums = np.zeros((nframe, 2, 2))
        for axis in range(2):
            dpsi = self.derivatives(obj, axis)
            num = (np.conj(c) * dpsi).real.sum(axis=(1, 2))
            den = (np.abs(dpsi) ** 2).sum(axis=(1, 2))
            for k, f in enumerate(self.frames):
                sums[f, 0, axis] += num[k]
                sums[f, 1, axis] += den[k]
        return sums


def llk_due(calc_llk, ic, ncycle):
    """engine/ptycho.rs:44-46."""
    return calc_llk > 0 and (ic % calc_llk == 0 or ic + 1 == ncycle)


class Ptycho:
    """Reconstruction state of one scan (engine/ptycho.rs:198-285).

    counts: `[nframe, ny, nx]` detector order (u16 with MASKED, or float with negative masked);
    y, x: positions in metres; object `[nobj, nyo, nxo]`, probe `[nprobe, ny, nx]` complex.
    """

    def __init__(self, counts, y, x, optics, obj, probe):
        counts = np.asarray(counts)
        frame = list(counts.shape[1:])
        if list(probe.shape[1:]) != frame:
            raise ValueError("probe plane differs from frame")
        self.optics = optics
        py, px = pynx_preprocess(y, x, optics.pixel)
        self.addr = AddrTable(py, px, optics.pixel, frame, list(obj.shape[1:]),
                              probe.shape[0], obj.shape[0])
        self.obs = Observed(counts)
        self.object = np.array(obj, np.complex128)
        self.probe = np.array(probe, np.complex128)
        self.cycle = 0
        self.history = []
        self.offsets = None
        self.refine = False

    def set_positions(self, offsets, refine=False):
        """`Features::position` with Patch sampling: per-frame offsets `[P, 2]` (dy, dx) in
        object pixels, refined by ML when `refine` (engine/features.rs:20-130)."""
        self.offsets = None if offsets is None else np.array(offsets, np.float64)
        self.refine = bool(refine) and offsets is not None

    def shifted(self, probe=None):
        """`Ptycho::shifted` (engine/ptycho.rs:373-386): the position model of every view, or
        None without offsets."""
        if self.offsets is None:
            return None
        return Shifted(self.addr.views, self.probe if probe is None else probe,
                       self.optics.quad, self.offsets)

    # exit waves -------------------------------------------------------------------------
    def calc_psi(self, views=None, obj=None, probe=None):
        if views is None and obj is None and probe is None and self.offsets is not None:
            return self.shifted().to_psi(self.object)
        views = self.addr.views if views is None else views
        obj = self.object if obj is None else obj
        probe = self.probe if probe is None else probe
        return ops.obj_probe_to_psi(views, obj, probe, self.optics.quad)

    def llk(self):
        """Normalised LLK of the current estimate (engine/ptycho.rs:454-466)."""
        psi = self.optics.exit_forward(self.calc_psi())
        return ops.llk(self.obs, slice(0, self.addr.nframe), self.addr.nmode,
                       psi).normalised(self.obs.nb_obs)

    def record(self, algorithm, l):
        self.history.append(dict(cycle=self.cycle, algorithm=algorithm, **l.as_dict()))

    # ML ---------------------------------------------------------------------------------
    def grad_psi(self):
        """Object-plane `2·∂L/∂psi*` (engine/ptycho.rs:548-561)."""
        psi = self.optics.exit_forward(self.calc_psi())
        psi = ops.poisson_grad(self.obs, slice(0, self.addr.nframe), self.addr.nmode, psi)
        return self.optics.exit_adjoint(psi)

    def grads(self, obj=True, probe=True):
        """Numerators of the back-projections of `grad_psi` (engine/ptycho.rs:429-450,
        511-513)."""
        g = self.grad_psi()
        views, q = self.addr.views, self.optics.quad
        s = self.shifted()
        if s is not None:
            go = (s.accumulate_obj(self.object.shape, g)[0] if obj
                  else np.zeros_like(self.object))
            gp = (s.accumulate_probe(self.object, self.probe.shape, g)[0] if probe
                  else np.zeros_like(self.probe))
            return go, gp
        go = (ops.accumulate_obj(views, self.object.shape, self.probe, q, g)[0] if obj
              else np.zeros_like(self.object))
        gp = (ops.accumulate_probe(views, self.object, self.probe.shape, q, g)[0] if probe
              else np.zeros_like(self.probe))
        return go, gp

    def cg_gamma(self, d_obj, d_probe):
        """engine/ptycho.rs:517-545, under the position model when offsets are set."""
        views, q = self.addr.views, self.optics.quad
        po = self.calc_psi()
        if self.offsets is not None:
            sp, sd = self.shifted(), self.shifted(d_probe)
            a = sp.to_psi(d_obj) + sd.to_psi(self.object)
            b = sd.to_psi(d_obj)
        else:
            a = (ops.obj_probe_to_psi(views, d_obj, self.probe, q)
                 + ops.obj_probe_to_psi(views, self.object, d_probe, q))
            b = ops.obj_probe_to_psi(views, d_obj, d_probe, q)
        po, a, b = (self.optics.exit_forward(x) for x in (po, a, b))
        return ops.cg_poisson_gamma(self.obs, slice(0, self.addr.nframe), self.addr.nmode,
                                    po, a, b)

    def scale_obj_probe(self):
        """PyNX ScaleObjProbe(absolute=True) without background (engine/ptycho.rs:577-591)."""
        calc = self.llk().nb_photons_calc
        self.split_scale(np.sqrt(self.obs.total() / calc))

    def split_scale(self, s):
        """Scale `O·P` by `s` and balance `Σ|O|` and `Σ|P|` (engine/ptycho.rs:593-603); with
        `s = 1` PyNX ScaleObjProbe(absolute=False)."""
        os_ = float(np.abs(self.object).sum())
        ps = float(np.abs(self.probe).sum())
        fp, fo = np.sqrt(os_ / ps * s), np.sqrt(ps / os_ * s)
        self.probe = self.probe * fp
        self.object = self.object * fo

    def position_grad(self, cost="poisson", offsets=None):
        """`position_grad` (engine/features.rs:1055-1100): per frame `[∂C/∂dy, ∂C/∂dx]` of the
        Poisson (or amplitude) cost at `offsets` (the state's when None) under Patch sampling,
        `Σ_views Σ Re(conj(g)·∂psi/∂d)` with `g = 2·IDFT(slope·DFT(psi))`, `slope` =
        `1 − I/Ĩ` (Poisson) or `1 − √(I/Ĩ)` (amplitude), Ĩ floored at 1e-12, 0 where masked."""
        d = self.offsets if offsets is None else np.asarray(offsets, np.float64)
        s = Shifted(self.addr.views, self.probe, self.optics.quad, d)
        nframe, nmode = self.addr.nframe, self.addr.nmode
        psi = ops.fft2(s.to_psi(self.object))
        ny, nx = psi.shape[-2:]
        b = psi.reshape(nframe, nmode, ny, nx)
        icalc = np.maximum((np.abs(b) ** 2).sum(axis=1), 1e-12)
        iobs, mask = self.obs.iobs[:nframe], self.obs.mask[:nframe]
        if cost == "poisson":
            slope = 1.0 - iobs / icalc
        else:
            slope = 1.0 - np.sqrt(np.maximum(iobs, 0.0) / icalc)
        r = np.where(mask, 0.0, 2.0 * slope)
        g = ops.ifft2((b * r[:, None]).reshape(psi.shape))
        grad = np.zeros((nframe, 2))
        for axis in range(2):
            dpsi = s.derivatives(self.object, axis)
            per_view = (np.conj(g) * dpsi).real.sum(axis=(1, 2))
            for k, f in enumerate(s.frames):
                grad[f, axis] += per_view[k]
        return grad

    def projected_position_sums(self, s):
        """`Shifted::position_sums` of the magnitude projection of the current estimate's
        exit waves (engine/ptycho.rs:470-480)."""
        nframe, nmode = self.addr.nframe, self.addr.nmode
        psi = self.optics.exit_forward(s.to_psi(self.object))
        psi = ops.apply_amplitude(self.obs, slice(0, nframe), nmode, psi)
        psi = self.optics.exit_adjoint(psi)
        return s.position_sums(self.object, psi, nframe)

    def ml(self, ncycle, update_object=True, update_probe=False, calc_llk=0,
           zero_phase_ramp=True, after_cycle=None):
        """PyNX ML Poisson CG (engine/ptycho.rs:775-842); refined offsets take AP's and DM's
        position step from the estimate each cycle starts from, after the update.
        `after_cycle(ic)`, if given, runs after cycle ic (a checkpoint hook; the run is the
        same without it)."""
        self.scale_obj_probe()
        last = None
        d_obj = np.zeros_like(self.object)
        d_probe = np.zeros_like(self.probe)
        for ic in range(ncycle):
            l = self.llk() if llk_due(calc_llk, ic, ncycle) else None
            sums = self.projected_position_sums(self.shifted()) if self.refine else None
            go, gp = self.grads(update_object, update_probe)
            if last is None:
                beta = 0.0
            else:
                num = ((np.conj(go) * (go - last[0])).real.sum()
                       + (np.conj(gp) * (gp - last[1])).real.sum())
                den = (np.abs(last[0]) ** 2).sum() + (np.abs(last[1]) ** 2).sum()
                with np.errstate(divide="ignore", invalid="ignore"):
                    beta = num / den
                if not (np.isfinite(beta) and beta >= 0.0):
                    beta = 0.0
            d_obj = d_obj * beta - go
            d_probe = d_probe * beta - gp
            num, den = self.cg_gamma(d_obj, d_probe)
            with np.errstate(divide="ignore", invalid="ignore"):
                gamma = np.float64(num) / np.float64(den)
            if np.isfinite(gamma):
                self.object = self.object + d_obj * gamma
                self.probe = self.probe + d_probe * gamma
            else:
                d_obj, d_probe = -go, -gp
            last = (go, gp)
            if sums is not None:
                ops.position_step(self.offsets, sums)
            if l is not None:
                self.record("ml", l)
            self.cycle += 1
            if after_cycle is not None:
                after_cycle(ic)
        if zero_phase_ramp:
            self.zero_phase_ramp()

    def zero_phase_ramp(self):
        """PyNX ZeroPhaseRamp (engine/ptycho.rs:1134-1170)."""
        self.object, self.probe = zero_phase_ramp(self.object, self.probe)

    # AP ---------------------------------------------------------------------------------
    def ap(self, ncycle, obj_inertia=0.01, probe_inertia=None, calc_llk=0,
           zero_phase_ramp=True):
        """PyNX AP (engine/ptycho.rs:609-641, ops.rs:352-381), under the position model when
        offsets are set."""
        nframe, nmode = self.addr.nframe, self.addr.nmode
        views, q = self.addr.views, self.optics.quad
        for ic in range(ncycle):
            psi = self.optics.exit_forward(self.calc_psi())
            l = None
            if llk_due(calc_llk, ic, ncycle):
                l = ops.llk(self.obs, slice(0, nframe), nmode, psi).normalised(self.obs.nb_obs)
            psi = ops.apply_amplitude(self.obs, slice(0, nframe), nmode, psi)
            psi = self.optics.exit_adjoint(psi)
            s = self.shifted()
            if s is not None:
                # under the move: the position sums against the arrays the projection read,
                # both updates from them, then the position step (engine/ptycho.rs:627-636)
                sums = s.position_sums(self.object, psi, nframe) if self.refine else None
                self.object, self.probe = s.psi_to_obj_probe(self.object, self.probe, psi,
                                                             obj_inertia, probe_inertia)
                if sums is not None:
                    ops.position_step(self.offsets, sums)
                if l is not None:
                    self.record("ap", l)
                self.cycle += 1
                continue
            acc = (ops.accumulate_obj(views, self.object.shape, self.probe, q, psi)
                   if obj_inertia is not None else None)
            if probe_inertia is not None:
                num, norm = ops.accumulate_probe(views, self.object, self.probe.shape, q, psi)
                self.probe = _blend(self.probe, num, norm, probe_inertia)
            if acc is not None:
                self.object = _blend(self.object, acc[0], acc[1], obj_inertia)
            if l is not None:
                self.record("ap", l)
            self.cycle += 1
        if zero_phase_ramp:
            self.zero_phase_ramp()

    # DM and RAAR ------------------------------------------------------------------------
    def _project(self, psi):
        """Object-plane magnitude projection `F⁻¹ Π_F F psi` (engine/ptycho.rs:671-674)."""
        far = self.optics.exit_forward(psi)
        far = ops.apply_amplitude(self.obs, slice(0, self.addr.nframe), self.addr.nmode, far)
        return self.optics.exit_adjoint(far)

    def update_obj_probe(self, psi, obj_inertia, probe_inertia, loops):
        """DM's and RAAR's update (engine/ptycho.rs:732-754): the position sums of `psi` under
        the cycle's model while the positions are refined, `loops` times an object-only then a
        probe-only `psi_to_obj_probe` (engine/ops.rs:352-369; under the move each from the
        current probe's waves), so the probe update sees the new object, then the position
        step."""
        views, q = self.addr.views, self.optics.quad
        s = self.shifted()
        if s is not None:
            sums = s.position_sums(self.object, psi, self.addr.nframe) if self.refine else None
            for _ in range(loops):
                if obj_inertia is not None:
                    self.object, _ = self.shifted().psi_to_obj_probe(
                        self.object, self.probe, psi, obj_inertia, None)
                if probe_inertia is not None:
                    _, self.probe = self.shifted().psi_to_obj_probe(
                        self.object, self.probe, psi, None, probe_inertia)
            if sums is not None:
                ops.position_step(self.offsets, sums)
            return
        for _ in range(loops):
            if obj_inertia is not None:
                num, norm = ops.accumulate_obj(views, self.object.shape, self.probe, q, psi)
                self.object = _blend(self.object, num, norm, obj_inertia)
            if probe_inertia is not None:
                num, norm = ops.accumulate_probe(views, self.object, self.probe.shape, q, psi)
                self.probe = _blend(self.probe, num, norm, probe_inertia)

    def dm(self, ncycle, obj_inertia=0.01, probe_inertia=0.001, alpha=0.02, loop_obj_probe=1,
           calc_llk=0, zero_phase_ramp=True):
        """PyNX DM with `a = alpha` (engine/ptycho.rs:653-691): cycle 0 starts from `psi = PO`,
        later cycles reflect the carried `psi`, `psi ← (2 − a)·PO − (1 − a)·psi`, project it
        and add `(1 − a)·(PO − refl)`; the LLK is of the estimate the cycle starts from, and a
        recorded cycle ends with `split_scale(1)`."""
        a = alpha
        psi = None
        for ic in range(ncycle):
            l = self.llk() if llk_due(calc_llk, ic, ncycle) else None
            po = self.calc_psi()
            if ic == 0:
                psi = po.copy()
                refl = None
            else:
                psi = po * (2.0 - a) - psi * (1.0 - a)
                refl = psi.copy()
            psi = self._project(psi)
            if refl is not None:
                psi = psi + (po - refl) * (1.0 - a)
            self.update_obj_probe(psi, obj_inertia, probe_inertia, loop_obj_probe)
            if l is not None:
                self.record("dm", l)
                self.split_scale(1.0)
            self.cycle += 1
        if zero_phase_ramp:
            self.zero_phase_ramp()

    def raar(self, ncycle, obj_inertia=0.01, probe_inertia=0.001, beta=0.9, loop_obj_probe=1,
             calc_llk=0, zero_phase_ramp=True):
        """PyNX RAAR with `b = beta` (engine/ptycho.rs:698-730): cycle 0 starts from
        `psi = PO`, later cycles mix the carried projection with the carried iterate,
        `psi ← (1 − b/2)·psi + (b/2)·(2·PO − it)`, which becomes the next iterate, then
        project; update, LLK record and balance as DM's."""
        h = 0.5 * beta
        psi = it = None
        for ic in range(ncycle):
            l = self.llk() if llk_due(calc_llk, ic, ncycle) else None
            po = self.calc_psi()
            if ic == 0:
                psi = po.copy()
            else:
                psi = psi * (1.0 - h) + (po * 2.0 - it) * h
            it = psi.copy()
            psi = self._project(psi)
            self.update_obj_probe(psi, obj_inertia, probe_inertia, loop_obj_probe)
            if l is not None:
                self.record("raar", l)
                self.split_scale(1.0)
            self.cycle += 1
        if zero_phase_ramp:
            self.zero_phase_ramp()

    # rPIE -------------------------------------------------------------------------------
    def rpie(self, nepoch, obj_step=1.0, probe_step=1.0, obj_alpha=0.1, probe_alpha=0.1,
             batch_size=100, calc_llk=0, seed=7):
        """pty-chi rPIE on seeded mini-batches (engine/ptycho.rs:874-902)."""
        if self.addr.nobj != 1:
            raise ValueError("rPIE needs exactly one object mode")
        if batch_size == 0:
            raise ValueError("rPIE batch_size must be >= 1")
        nframe = self.addr.nframe
        for ic in range(nepoch):
            for frames in random_batches(nframe, batch_size, seed, self.cycle):
                self.rpie_batch(frames, obj_step, probe_step, obj_alpha, probe_alpha)
            if llk_due(calc_llk, ic, nepoch):
                self.record("rpie", self.llk())
            self.cycle += 1

    def rpie_batch(self, frames, obj_step, probe_step, obj_alpha, probe_alpha):
        """One rPIE batch from the batch-start object, probe and offsets
        (engine/ptycho.rs:904-1085) under Patch sampling: with offsets every view's wave is
        its frame's moved probe, the probe direction of a frame moves back before it adds in,
        and refined offsets take pty-chi's step from mode 0."""
        ny, nx = self.probe.shape[-2:]
        nmode = self.addr.nmode
        nbatch = len(frames)
        views = np.concatenate([self.addr.frame_views(f) for f in frames])
        q = self.optics.quad
        shifted = (None if self.offsets is None else
                   Shifted(views, self.probe, q, self.offsets))
        if shifted is not None:
            psi = shifted.to_psi(self.object)
        else:
            psi = ops.obj_probe_to_psi(views, self.object, self.probe, q)
        delta = self.optics.exit_forward(psi)
        sh = (nbatch, nmode, ny, nx)
        d4 = delta.reshape(sh)
        calc = np.sqrt((np.abs(d4) ** 2).sum(axis=1))
        iobs, mask = self.obs.iobs[frames], self.obs.mask[frames]
        r = np.where(mask, 1.0, np.sqrt(iobs + 1e-7) / (calc + 1e-7))
        delta = (d4 * r[:, None]).reshape(psi.shape)
        delta = self.optics.exit_adjoint(delta) - psi

        pidx = views["probe"].astype(np.int64)
        if shifted is not None:
            wave = fftshift2(shifted.waves)                  # moved W, shifted, per view
            w2 = fftshift2(np.abs(shifted.waves) ** 2)
        else:
            wave = fftshift2(self.probe[pidx] * q)            # shifted, per view
            w2 = fftshift2(np.abs(self.probe[pidx]) ** 2)       # shifted, per view
        nyo, nxo = self.object.shape[-2:]
        new_obj = new_probe = None
        if obj_step is not None:
            # overlap D_m placed on the object per probe mode, read back per view
            # (engine/ptycho.rs:1094-1130)
            dplanes = np.zeros((self.addr.nprobe, nyo, nxo))
            w2n = fftshift2(w2)
            for k, v in enumerate(views):
                oy, ox = int(v["oy"]), int(v["ox"])
                dplanes[pidx[k], oy:oy + ny, ox:ox + nx] += w2n[k]
            dens = np.empty_like(w2)
            for k, v in enumerate(views):
                oy, ox = int(v["oy"]), int(v["ox"])
                dens[k] = fftshift2(dplanes[pidx[k], oy:oy + ny, ox:ox + nx])
            pmax = dens.reshape(sh).sum(axis=1).max()
            a = obj_alpha
            steps = np.conj(wave) / ((1.0 - a) * dens + a * pmax) * delta
            stepn = fftshift2(steps)
            d = np.zeros((nyo, nxo), np.complex128)
            for k, v in enumerate(views):
                oy, ox = int(v["oy"]), int(v["ox"])
                d[oy:oy + ny, ox:ox + nx] += stepn[k]
            new_obj = d
        if probe_step is not None:
            a = probe_alpha
            dp = np.zeros_like(self.probe)
            deltan = fftshift2(delta)
            ob = self.object[0]
            for b in range(nbatch):
                fv = views[b * nmode:(b + 1) * nmode]
                oy, ox = int(fv[0]["oy"]), int(fv[0]["ox"])
                win = ob[oy:oy + ny, ox:ox + nx]
                omax = (np.abs(win) ** 2).max()
                w = np.conj(win * q) / ((1.0 - a) * np.abs(win) ** 2 + a * omax)
                frame = np.zeros_like(self.probe)
                for m, v in enumerate(fv):
                    frame[int(v["probe"])] += w * deltan[b * nmode + m]
                if shifted is not None:
                    # back through the frame's move (engine/ptycho.rs:1027-1035)
                    frame = ops.move_planes(frame, q, -self.offsets[int(fv[0]["frame"])])
                dp += frame
            new_probe = dp
        dirs = None
        if shifted is not None and self.refine:
            # pty-chi's gradient position sums from mode 0 (engine/ptycho.rs:1037-1064)
            sums = []
            for b in range(nbatch):
                k = b * nmode
                v = views[k]
                oy, ox = int(v["oy"]), int(v["ox"])
                patch = self.object[int(v["obj"]), oy:oy + ny, ox:ox + nx]
                sums.append(ops.gradient_sums(patch, fftshift2(shifted.waves[k]), delta[k]))
            dirs = ops.gradient_directions(
                sums, ops.EPS_POSITION * self.optics.intensity_scale())
        if obj_step is not None:
            self.object = self.object + new_obj[None] * obj_step
        if probe_step is not None:
            self.probe = self.probe + new_probe * (probe_step / nbatch)
        if dirs is not None:
            ops.batch_position_step(self.offsets, frames, dirs)


def zero_phase_ramp(obj, probe):
    """engine/ptycho.rs:1134-1170."""
    ny, nx = probe.shape[-2:]
    far = ops.fft2(fftshift2(probe))
    v = (np.abs(fftshift2(far)) ** 2).sum(axis=0)
    w = v.sum()
    iy, ix = np.mgrid[:ny, :nx]
    dy = (v * iy).sum() / w - (ny // 2)
    dx = (v * ix).sum() / w - (nx // 2)

    def ramp(length, half, scale, d, sign):
        return sign * 2.0 * np.pi * d * (np.arange(length) - half) / scale

    ry, rx = ramp(ny, ny // 2, ny, dy, -1.0), ramp(nx, nx // 2, nx, dx, -1.0)
    probe = probe * np.exp(1j * (ry[:, None] + rx[None, :]))
    nyo, nxo = obj.shape[-2:]
    ry, rx = ramp(nyo, nyo // 2, ny, dy, 1.0), ramp(nxo, nxo // 2, nx, dx, 1.0)
    obj = obj * np.exp(1j * (ry[:, None] + rx[None, :]))
    return obj, probe


def _blend(old, num, norm, inertia):
    """`(num + reg·old) / max(norm + reg, 1e-12)`, `reg = max(norm)·inertia`
    (engine/ops.rs:371-381)."""
    reg = max(0.0, float(norm.max())) * inertia
    return (num + old * reg) / np.maximum(norm + reg, 1e-12)
