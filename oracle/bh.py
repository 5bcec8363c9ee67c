"""pty-chi BH (bilinear-Hessian) on the amplitude cost in float64 (oracle restatement, test
infrastructure only), on one object slice, with or without the position model under Patch
sampling.

Follows physwkim/ptyrs `ptyrs/src/engine/bh.rs`: `BhBatch::with_sampling` (bh.rs:168-275: the
exit waves `U psi`, `A = √Σ_m |U psi_m|² + EPS`, `td = U psi·(1 − √iobs / A)`, zero where
masked), `BhBatch::grads` (bh.rs:320-380: `2·∂F/∂x*` as the adjoint of `2·td`),
`BhBatch::hessian` (bh.rs:500-575: pty-chi's bilinear Hessian `H(u, v)`) and `Bh::epoch`
(bh.rs:645-760: seeded batches, the probe preconditioned by `ρ² = probe_rho²·k`, conjugate
directions across epochs with one batch of every frame, steepest descent with smaller batches,
`α = −⟨g, D⟩ / H(D, D) · count / batch_size`).

The cost is F = Σ_frames Σ_unmasked (A − √iobs)² over the batch's views; the displacement
`(u_O, u_P)` of object and probe changes the exit wave by `J u = (u_P·O + P·u_O)·q` and to
second order by `J″(u, v) = (u_P·v_O + v_P·u_O)·q`.

Under the position model (the reference's `Features::position` with Patch sampling, bh.rs:
92-275 and 630-760, and its float64 model `refs/f64/bh_pos.py`) frame b reads the probe moved by
its offset d_b, `M_b(P) = conj(q)·T_d(q·P)` (ops.move_planes). Held offsets only move the probe
and its displacements (`J u = (M_b(u_P)·O + M_b(P)·u_O)·q`). Refined offsets are variables too:
a displacement carries `u_d` per batch frame, `g_d = Σ_m Re⟨Uᴴ(2·td), ∂_a M_b(P)·O·q⟩` per axis,
and with `dW_u = M_b(u_P) + Σ_a u_da·∂_a M_b(P)`,
`J u = (dW_u·O + M_b(P)·u_O)·q` and
`J″(u, v) = ((Σ_a v_da·∂_a M_b(u_P) + u_da·∂_a M_b(v_P) + Σ_ab u_da·v_db·∂_a∂_b M_b(P))·O
+ dW_u·v_O + dW_v·u_O)·q`.
The epoch takes the offsets' part of the gradient times `position_rho²`, keeps the direction's
offsets part per frame for CG and moves the batch's offsets by `0.3·α·D_d` (pty-chi's position
step size, unclipped).
"""
import numpy as np

from . import ops
from .base import fftshift2, random_batches
from .lsqml import SliceWaves, slice_jet

EPS = 1e-8
POSITION_STEP = 0.3  # bh.rs POSITION_STEP, pty-chi's ProbePositionOptions step size


def _dot(a, b):
    """⟨a, b⟩ = Σ Re(conj(a)·b)."""
    return float(np.sum((np.conj(a) * b).real))


class BhBatch:
    """The amplitude cost of `views` (whole frames, in order) at `(obj, probe)` and its
    gradient and Hessian (engine/bh.rs:122-575, one slice); `offsets` `[nb, 2]` (dy, dx in
    object pixels, one per batch frame in order) move each frame's probe, and with `refine` they
    are variables of the cost."""

    def __init__(self, views, obs, optics, obj, probe, offsets=None, refine=False):
        self.views, self.optics, self.obj, self.probe = views, optics, obj, probe
        nmode = 1
        while nmode < len(views) and views[nmode]["frame"] == views[0]["frame"]:
            nmode += 1
        self.nmode = nmode
        self.frames = [int(views[b * nmode]["frame"]) for b in range(len(views) // nmode)]
        ny, nx = probe.shape[-2:]
        self.offsets = None if offsets is None else np.asarray(offsets, np.float64)
        self.refine = bool(refine) and self.offsets is not None
        if self.offsets is not None:
            # each frame's own probe planes: view probe index b·nprobe + mode
            np_ = probe.shape[0]
            self.pviews = views.copy()
            self.pviews["probe"] = (np.repeat(np.arange(len(self.frames)) * np_, nmode)
                                    + views["probe"])
            self.w = self._moved(probe)
            if self.refine:
                self.dw = [self._moved(probe, (a,)) for a in range(2)]
                self.d2w = [[self._moved(probe, (a, b)) for b in range(2)] for a in range(2)]
        else:
            self.pviews, self.w = views, probe
        self.psi = optics.exit_forward(ops.obj_probe_to_psi(self.pviews, obj, self.w,
                                                            optics.quad))
        sh = (len(self.frames), nmode, ny, nx)
        self.amp = np.sqrt((np.abs(self.psi.reshape(sh)) ** 2).sum(axis=1)) + EPS
        iobs, self.mask = obs.iobs[self.frames], obs.mask[self.frames]
        self.root = np.sqrt(iobs)
        w = np.where(self.mask, 0.0, 1.0 - self.root / self.amp)
        self.td = (self.psi.reshape(sh) * w[:, None]).reshape(self.psi.shape)

    def _moved(self, x, axes=()):
        """Every batch frame's `M_b(x)` (or its derivative over the listed offset axes),
        `[nb·nprobe, ny, nx]` frame-major."""
        q = self.optics.quad
        return np.concatenate([ops.move_planes(x, q, d, axes) for d in self.offsets])

    def _per_frame(self, planes, d):
        """`Σ_a d[b, a]·planes[a]` with one coefficient pair per batch frame."""
        np_ = self.probe.shape[0]
        c = np.repeat(np.asarray(d, np.float64), np_, axis=0)
        return c[:, 0, None, None] * planes[0] + c[:, 1, None, None] * planes[1]

    def grads(self):
        """`2·∂F/∂x*` over the object and the probe (engine/bh.rs:320-380), and with refined
        offsets ∂F/∂d `[nb, 2]` (None otherwise)."""
        q = self.optics.quad
        e = self.optics.exit_adjoint(2.0 * self.td)
        g_obj = ops.accumulate_obj(self.pviews, self.obj.shape, self.w, q, e)[0]
        if self.offsets is None:
            g_probe = ops.accumulate_probe(self.views, self.obj, self.probe.shape, q, e)[0]
            return g_obj, g_probe, None
        # each frame's probe-plane gradient, back through its move M_bᴴ = conj(q)·T_−d(q·)
        np_ = self.probe.shape[0]
        per = ops.accumulate_probe(self.pviews, self.obj, self.w.shape, q, e)[0]
        g_probe = sum(ops.move_planes(per[b * np_:(b + 1) * np_], q, -d)
                      for b, d in enumerate(self.offsets))
        if not self.refine:
            return g_obj, g_probe, None
        # Σ_m Re⟨e, shift(∂_a M_b(P)·O·q)⟩ per frame and axis
        nb = len(self.frames)
        g_d = np.zeros((nb, 2))
        for a in range(2):
            t = ops.obj_probe_to_psi(self.pviews, self.obj, self.dw[a], q)
            g_d[:, a] = (np.conj(e) * t).real.reshape(nb, -1).sum(axis=1)
        return g_obj, g_probe, g_d

    def _dw(self, up, ud):
        """`dW_u`: the frames' probe-plane change along the displacement."""
        if self.offsets is None:
            return up
        t = self._moved(up)
        if self.refine and ud is not None:
            t = t + self._per_frame(self.dw, ud)
        return t

    def _tangent(self, u_obj, dw_u):
        """`U·J u` per view: the exit waves' first-order change."""
        q = self.optics.quad
        t = (ops.obj_probe_to_psi(self.pviews, self.obj, dw_u, q)
             + ops.obj_probe_to_psi(self.pviews, u_obj, self.w, q))
        return self.optics.exit_forward(t)

    def hessian(self, u, v):
        """pty-chi's bilinear Hessian (engine/bh.rs:500-575) along `u = (u_O, u_P[, u_d])` and
        `v`: Σ 2·Re(conj(td)·L_uv) + 2·Σ_unmasked [(1 − d/a)·Σ_m Re(conj(L_u)·L_v)
        + d·c_u·c_v/a³], `L_u = U·J u`, `L_uv = U·J″(u, v)`, `c_u = Σ_m Re(conj(U psi)·L_u)`,
        `d = √iobs`, `a` the modelled amplitude plus EPS."""
        uo, up, ud = (tuple(u) + (None,))[:3]
        vo, vp, vd = (tuple(v) + (None,))[:3]
        q = self.optics.quad
        dwu, dwv = self._dw(up, ud), self._dw(vp, vd)
        lu, lv = self._tangent(uo, dwu), self._tangent(vo, dwv)
        t2 = (ops.obj_probe_to_psi(self.pviews, vo, dwu, q)
              + ops.obj_probe_to_psi(self.pviews, uo, dwv, q))
        if self.refine and ud is not None and vd is not None:
            d2 = (self._per_frame([self._moved(up, (a,)) for a in range(2)], vd)
                  + self._per_frame([self._moved(vp, (a,)) for a in range(2)], ud))
            np_ = self.probe.shape[0]
            cu = np.repeat(np.asarray(ud, np.float64), np_, axis=0)
            cv = np.repeat(np.asarray(vd, np.float64), np_, axis=0)
            for a in range(2):
                for b in range(2):
                    d2 = d2 + (cu[:, a] * cv[:, b])[:, None, None] * self.d2w[a][b]
            t2 = t2 + ops.obj_probe_to_psi(self.pviews, self.obj, d2, q)
        luv = self.optics.exit_forward(t2)
        h = 2.0 * _dot(self.td, luv)
        ny, nx = self.probe.shape[-2:]
        sh = (len(self.frames), self.nmode, ny, nx)
        lu, lv, psi = lu.reshape(sh), lv.reshape(sh), self.psi.reshape(sh)
        uv = (np.conj(lu) * lv).real.sum(axis=1)
        cu = (np.conj(psi) * lu).real.sum(axis=1)
        cv = (np.conj(psi) * lv).real.sum(axis=1)
        a, d = self.amp, self.root
        terms = 2.0 * ((1.0 - d / a) * uv + d * cu * cv / (a * a * a))
        return float(h + terms[~self.mask].sum())


class BhSlices:
    """BhBatch through pty-chi's multislice object (engine/bh.rs with several slices, no
    position model): the exit waves through the slices (`SliceWaves`), 2·∂F/∂x* over every
    slice and the probe back through the slices' adjoints, and H(u, v) from the quadratic form
    Q(w) = H(w, w) of the second-order expansion of the exit waves along w (`slice_jet`:
    L_w = U ψ′, U J″(w, w) = 2·U ψ″) by polarization, H(u, v) = (Q(u + v) − Q(u − v))/4,
    exact for the symmetric bilinear H."""

    def __init__(self, views, obs, optics, objs, probe):
        self.views, self.optics, self.objs, self.probe = views, optics, list(objs), probe
        nmode = 1
        while nmode < len(views) and views[nmode]["frame"] == views[0]["frame"]:
            nmode += 1
        self.nmode = nmode
        self.frames = [int(views[b * nmode]["frame"]) for b in range(len(views) // nmode)]
        ny, nx = probe.shape[-2:]
        self.waves = SliceWaves(optics, views, self.objs, probe[views["probe"].astype(np.int64)])
        self.psi = optics.exit_forward(self.waves.psi)
        self.sh = (len(self.frames), nmode, ny, nx)
        self.amp = np.sqrt((np.abs(self.psi.reshape(self.sh)) ** 2).sum(axis=1)) + EPS
        iobs, self.mask = obs.iobs[self.frames], obs.mask[self.frames]
        self.root = np.sqrt(iobs)
        w = np.where(self.mask, 0.0, 1.0 - self.root / self.amp)
        self.td = (self.psi.reshape(self.sh) * w[:, None]).reshape(self.psi.shape)

    def grads(self):
        """2·∂F/∂x* over every slice (a list) and the probe (engine/multislice.rs:266-286,
        399-438 on the amplitude cost's exit-plane field)."""
        e = self.optics.exit_adjoint(2.0 * self.td)
        chis = self.waves.back_propagate(e)
        g_objs = [self.waves.obj_adjoint(s, chis[s]) for s in range(len(self.objs))]
        g_probe = ops.accumulate_probe(self.views, self.objs[0], self.probe.shape,
                                       self.waves.shared(0), chis[0])[0]
        return g_objs, g_probe, None

    def quad(self, w_objs, w_probe):
        """Q(w) = H(w, w): 2·Re⟨td, 2·U ψ″⟩ + 2·Σ_unmasked [(1 − d/a)·Σ_m |U ψ′|²
        + d·c²/a³], c = Σ_m Re(conj(U psi)·U ψ′)."""
        _, p1, p2 = slice_jet(self.optics, self.views, self.objs, self.probe, list(w_objs),
                              w_probe)
        h = 2.0 * _dot(self.td, 2.0 * p2)
        p1 = p1.reshape(self.sh)
        uu = (np.abs(p1) ** 2).sum(axis=1)
        c = (np.conj(self.psi.reshape(self.sh)) * p1).real.sum(axis=1)
        a, d = self.amp, self.root
        terms = 2.0 * ((1.0 - d / a) * uu + d * c * c / (a * a * a))
        return float(h + terms[~self.mask].sum())

    def hessian(self, u, v):
        (uo, up), (vo, vp) = tuple(u)[:2], tuple(v)[:2]
        if uo is vo and up is vp:
            return self.quad(uo, up)
        plus = self.quad([a + b for a, b in zip(uo, vo)], up + vp)
        minus = self.quad([a - b for a, b in zip(uo, vo)], up - vp)
        return (plus - minus) / 4.0


class Bh:
    """BH state across epochs (engine/bh.rs:580-760): the parameters, the epoch count and, with
    one batch per epoch, the last direction; under the position model `offsets` `[nframe, 2]`
    (held, or refined with `refine`, in which case `self.offsets` moves)."""

    def __init__(self, batch_size, probe_rho=0.01, seed=7, position_rho=0.1, offsets=None,
                 refine=False):
        if batch_size < 1:
            raise ValueError("BH batch_size must be >= 1")
        self.batch_size, self.probe_rho, self.seed = batch_size, probe_rho, seed
        self.position_rho = position_rho
        self.offsets = None if offsets is None else np.array(offsets, np.float64)
        self.refine = bool(refine) and self.offsets is not None
        self.epochs = 0
        self.prev = None

    def epoch(self, addr, obs, optics, obj, probe):
        """One epoch over the seeded batches: per batch g, Pg (the probe part times ρ²),
        D = −Pg or, with one batch of every frame after the first epoch,
        D = −Pg + β·D′ with β = H(Pg, D′)/H(D′, D′); α = −⟨g, D⟩/H(D, D)·count/size;
        object and probe += α·D. Returns `(obj, probe, steps)`, a step
        `dict(frames, beta, alpha, top, bottom)`."""
        if isinstance(obj, (list, tuple)):
            return self._epoch_slices(addr, obs, optics, list(obj), probe)
        nframe = addr.nframe
        size = min(self.batch_size, nframe)
        full = size == nframe
        rho2 = self.probe_rho ** 2 * optics.intensity_scale()
        pos_rho2 = self.position_rho ** 2
        epoch = self.epochs
        self.epochs += 1
        steps = []
        for frames in random_batches(nframe, size, self.seed, epoch):
            views = np.concatenate([addr.frame_views(f) for f in frames])
            d_b = None if self.offsets is None else self.offsets[list(frames)]
            b = BhBatch(views, obs, optics, obj, probe, d_b, self.refine)
            g_obj, g_probe, g_d = b.grads()
            pg = (g_obj, g_probe * rho2, None if g_d is None else g_d * pos_rho2)
            if full and self.prev is not None:
                d_obj, d_probe, by_frame = self.prev
                prev = (d_obj, d_probe, None if g_d is None else by_frame[list(frames)])
                beta = b.hessian(pg, prev) / b.hessian(prev, prev)
                direction = (beta * d_obj - pg[0], beta * d_probe - pg[1],
                             None if g_d is None else beta * prev[2] - pg[2])
            else:
                beta = 0.0
                direction = (-pg[0], -pg[1], None if g_d is None else -pg[2])
            top = -(_dot(g_obj, direction[0]) + _dot(g_probe, direction[1]))
            if g_d is not None:
                top -= float((g_d * direction[2]).sum())
            bottom = b.hessian(direction, direction)
            alpha = top / bottom * len(frames) / size
            obj = obj + alpha * direction[0]
            probe = probe + alpha * direction[1]
            by_frame = None
            if g_d is not None:
                by_frame = np.zeros((nframe, 2))
                by_frame[list(frames)] = direction[2]
                self.offsets[list(frames)] += POSITION_STEP * alpha * direction[2]
            if full:
                self.prev = (direction[0], direction[1], by_frame)
            steps.append(dict(frames=list(frames), beta=beta, alpha=alpha, top=top,
                              bottom=bottom))
        return obj, probe, steps

    def _epoch_slices(self, addr, obs, optics, objs, probe):
        """`epoch` through a multislice object (`objs` a list of slices; no position model):
        every slice and the probe are the variables, the probe's part preconditioned by ρ²."""
        if self.offsets is not None:
            raise ValueError("BH through slices runs without the position model")
        nframe = addr.nframe
        size = min(self.batch_size, nframe)
        full = size == nframe
        rho2 = self.probe_rho ** 2 * optics.intensity_scale()
        epoch = self.epochs
        self.epochs += 1
        steps = []
        for frames in random_batches(nframe, size, self.seed, epoch):
            views = np.concatenate([addr.frame_views(f) for f in frames])
            b = BhSlices(views, obs, optics, objs, probe)
            g_objs, g_probe, _ = b.grads()
            pg = (g_objs, g_probe * rho2)
            if full and self.prev is not None:
                prev = self.prev
                beta = b.hessian(pg, prev) / b.hessian(prev, prev)
                direction = ([beta * d - g for d, g in zip(prev[0], pg[0])],
                             beta * prev[1] - pg[1])
            else:
                beta = 0.0
                direction = ([-g for g in pg[0]], -pg[1])
            top = -(sum(_dot(g, d) for g, d in zip(g_objs, direction[0]))
                    + _dot(g_probe, direction[1]))
            bottom = b.hessian(direction, direction)
            alpha = top / bottom * len(frames) / size
            objs = [o + alpha * d for o, d in zip(objs, direction[0])]
            probe = probe + alpha * direction[1]
            if full:
                self.prev = direction
            steps.append(dict(frames=list(frames), beta=beta, alpha=alpha, top=top,
                              bottom=bottom))
        return objs, probe, steps


def amplitude_cost(views, obs, optics, obj, probe, offsets=None):
    """F without the amplitude offset: Σ_unmasked (|U psi| − √iobs)², a quarter of PyNX's
    Euclidian sum (the reference test's `cost`); `offsets` move each batch frame's probe."""
    nmode = 1
    while nmode < len(views) and views[nmode]["frame"] == views[0]["frame"]:
        nmode += 1
    frames = slice(int(views[0]["frame"]), int(views[-1]["frame"]) + 1)
    b = BhBatch(views, obs, optics, obj, probe, offsets) if offsets is not None else None
    pviews, w = (views, probe) if b is None else (b.pviews, b.w)
    psi = optics.exit_forward(ops.obj_probe_to_psi(pviews, obj, w, optics.quad))
    return ops.llk(obs, frames, nmode, psi).euclidian / 4.0


__all__ = ["BhBatch", "BhSlices", "Bh", "amplitude_cost", "fftshift2"]
