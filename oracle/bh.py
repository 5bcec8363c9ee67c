"""pty-chi BH (bilinear-Hessian) on the amplitude cost in float64 (oracle restatement, test
infrastructure only), on one object slice without the position model.

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
"""
import numpy as np

from . import ops
from .base import fftshift2, random_batches

EPS = 1e-8


def _dot(a, b):
    """⟨a, b⟩ = Σ Re(conj(a)·b)."""
    return float(np.sum((np.conj(a) * b).real))


class BhBatch:
    """The amplitude cost of `views` (whole frames, in order) at `(obj, probe)` and its
    gradient and Hessian (engine/bh.rs:122-575, one slice, no offsets)."""

    def __init__(self, views, obs, optics, obj, probe):
        self.views, self.optics, self.obj, self.probe = views, optics, obj, probe
        nmode = 1
        while nmode < len(views) and views[nmode]["frame"] == views[0]["frame"]:
            nmode += 1
        self.nmode = nmode
        self.frames = [int(views[b * nmode]["frame"]) for b in range(len(views) // nmode)]
        ny, nx = probe.shape[-2:]
        self.psi = optics.exit_forward(ops.obj_probe_to_psi(views, obj, probe, optics.quad))
        sh = (len(self.frames), nmode, ny, nx)
        self.amp = np.sqrt((np.abs(self.psi.reshape(sh)) ** 2).sum(axis=1)) + EPS
        iobs, self.mask = obs.iobs[self.frames], obs.mask[self.frames]
        self.root = np.sqrt(iobs)
        w = np.where(self.mask, 0.0, 1.0 - self.root / self.amp)
        self.td = (self.psi.reshape(sh) * w[:, None]).reshape(self.psi.shape)

    def _adjoint(self, y):
        """`Jᴴ Uᴴ y`: the object's and the probe's back-projections (engine/ops.rs:282-345)."""
        e = self.optics.exit_adjoint(y)
        g_obj = ops.accumulate_obj(self.views, self.obj.shape, self.probe, self.optics.quad, e)[0]
        g_probe = ops.accumulate_probe(self.views, self.obj, self.probe.shape, self.optics.quad,
                                       e)[0]
        return g_obj, g_probe

    def grads(self):
        """`2·∂F/∂x*` over the object and the probe (engine/bh.rs:320-380)."""
        return self._adjoint(2.0 * self.td)

    def _tangent(self, u_obj, u_probe):
        """`U·J u` per view: the exit waves' first-order change along `(u_O, u_P)`."""
        q = self.optics.quad
        t = (ops.obj_probe_to_psi(self.views, self.obj, u_probe, q)
             + ops.obj_probe_to_psi(self.views, u_obj, self.probe, q))
        return self.optics.exit_forward(t)

    def hessian(self, u, v):
        """pty-chi's bilinear Hessian (engine/bh.rs:500-575) along `u = (u_O, u_P)` and
        `v = (v_O, v_P)`: Σ 2·Re(conj(td)·L_uv) + 2·Σ_unmasked [(1 − d/a)·Σ_m Re(conj(L_u)·L_v)
        + d·c_u·c_v/a³], `L_u = U·J u`, `L_uv = U·J″(u, v)`, `c_u = Σ_m Re(conj(U psi)·L_u)`,
        `d = √iobs`, `a` the modelled amplitude plus EPS."""
        (uo, up), (vo, vp) = u, v
        q = self.optics.quad
        lu, lv = self._tangent(uo, up), self._tangent(vo, vp)
        luv = self.optics.exit_forward(ops.obj_probe_to_psi(self.views, vo, up, q)
                                       + ops.obj_probe_to_psi(self.views, uo, vp, q))
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


class Bh:
    """BH state across epochs (engine/bh.rs:580-760): the parameters, the epoch count and, with
    one batch per epoch, the last direction."""

    def __init__(self, batch_size, probe_rho=0.01, seed=7):
        if batch_size < 1:
            raise ValueError("BH batch_size must be >= 1")
        self.batch_size, self.probe_rho, self.seed = batch_size, probe_rho, seed
        self.epochs = 0
        self.prev = None

    def epoch(self, addr, obs, optics, obj, probe):
        """One epoch over the seeded batches: per batch g, Pg (the probe part times ρ²),
        D = −Pg or, with one batch of every frame after the first epoch,
        D = −Pg + β·D′ with β = H(Pg, D′)/H(D′, D′); α = −⟨g, D⟩/H(D, D)·count/size;
        object and probe += α·D. Returns `(obj, probe, steps)`, a step
        `dict(frames, beta, alpha, top, bottom)`."""
        nframe = addr.nframe
        size = min(self.batch_size, nframe)
        full = size == nframe
        rho2 = self.probe_rho ** 2 * optics.intensity_scale()
        epoch = self.epochs
        self.epochs += 1
        steps = []
        for frames in random_batches(nframe, size, self.seed, epoch):
            views = np.concatenate([addr.frame_views(f) for f in frames])
            b = BhBatch(views, obs, optics, obj, probe)
            g_obj, g_probe = b.grads()
            pg = (g_obj, g_probe * rho2)
            if full and self.prev is not None:
                d_obj, d_probe = self.prev
                beta = b.hessian(pg, (d_obj, d_probe)) / b.hessian((d_obj, d_probe),
                                                                    (d_obj, d_probe))
                direction = (beta * d_obj - pg[0], beta * d_probe - pg[1])
            else:
                beta = 0.0
                direction = (-pg[0], -pg[1])
            top = -(_dot(g_obj, direction[0]) + _dot(g_probe, direction[1]))
            bottom = b.hessian(direction, direction)
            alpha = top / bottom * len(frames) / size
            obj = obj + alpha * direction[0]
            probe = probe + alpha * direction[1]
            if full:
                self.prev = direction
            steps.append(dict(frames=list(frames), beta=beta, alpha=alpha, top=top,
                              bottom=bottom))
        return obj, probe, steps


def amplitude_cost(views, obs, optics, obj, probe):
    """F without the amplitude offset: Σ_unmasked (|U psi| − √iobs)², a quarter of PyNX's
    Euclidian sum (the reference test's `cost`)."""
    nmode = 1
    while nmode < len(views) and views[nmode]["frame"] == views[0]["frame"]:
        nmode += 1
    frames = slice(int(views[0]["frame"]), int(views[-1]["frame"]) + 1)
    psi = optics.exit_forward(ops.obj_probe_to_psi(views, obj, probe, optics.quad))
    return ops.llk(obs, frames, nmode, psi).euclidian / 4.0


__all__ = ["BhBatch", "Bh", "amplitude_cost", "fftshift2"]
