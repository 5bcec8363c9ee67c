"""pty-chi LSQML in float64 (oracle restatement, test infrastructure only).

Follows physwkim/ptyrs `ptyrs/src/engine/lsqml.rs`, with or without OPR probe variation
(`ProbeVariation`, oracle/opr.py), with the position feature under Patch sampling and pty-chi's
multislice object (`SliceWaves`, engine/multislice.rs:87-438): `LsqmlBatch::new` (lsqml.rs:102-179),
`obj_directions`, `frame_probe_directions`, `probe_direction` (lsqml.rs:194-229),
`step_sizes` (lsqml.rs:286-350), `trim_mean` (lsqml.rs:392-398), `Lsqml::step`
(lsqml.rs:581-643) and `Lsqml::epoch` (lsqml.rs:663-714).
"""
import math

import numpy as np

from . import ops
from .base import fftshift2, random_batches

EPS_AMPLITUDE = 1e-9
EPS_POISSON = 1e-6
EPS_XI = 1e-5
LAMBDA0 = 1.2e-7


def trim_mean(x):
    """MATLAB `trimmean(x, 10)` (engine/lsqml.rs:392-398)."""
    s = sorted(float(v) for v in x)
    k = int(math.ceil(len(s) * 0.1 / 2.0 - 0.5))
    kept = s[k:len(s) - k]
    total = 0.0
    for v in kept:
        total += v
    return total / len(kept)


def _unit(shape):
    return np.ones(shape, np.complex128)


class SliceWaves:
    """The waves of `views` (each with its own probe plane, natural layout `planes[k]`)
    through the slices of `optics` (engine/multislice.rs:87-173): `incident[s]` the wave
    entering slice s (natural, one plane per view), `psi` the exit waves (shifted)."""

    def __init__(self, optics, views, objects, planes):
        self.optics, self.views, self.objects = optics, views, objects
        ny, nx = planes.shape[-2:]
        self.own = views.copy()
        self.own["probe"] = np.arange(len(views))
        self.incident = [planes]
        for s, gap in enumerate(optics.gaps):
            psi = ops.obj_probe_to_psi(self.own, objects[s], self.incident[s], _unit((ny, nx)))
            psi = gap.forward(psi)
            self.incident.append(fftshift2(psi))
        last = len(objects) - 1
        self.psi = ops.obj_probe_to_psi(self.own, objects[last], self.incident[last],
                                        self.shared(last))

    def shared(self, s):
        q = self.optics.slice_quad(s)
        return q if q is not None else _unit(self.optics.quad.shape)

    def back_propagate(self, chi):
        """Per slice, its change of psi_s (engine/multislice.rs:266-286)."""
        out = [chi]
        n = len(self.objects)
        dims = self.incident[0].shape
        for s in range(n - 2, -1, -1):
            up = out[-1]
            h, _ = ops.accumulate_probe(self.own, self.objects[s + 1], dims, self.shared(s + 1),
                                        up)
            g = self.optics.gaps[s].adjoint(fftshift2(h))
            out.append(g)
        out.reverse()
        return out

    def obj_adjoint(self, s, chi_s):
        """Σ conj(q_s·in_s)·chi_s on the slice (engine/multislice.rs:399-428)."""
        return ops.accumulate_obj(self.own, self.objects[s].shape, self.incident[s],
                                  self.shared(s), chi_s)[0]

    def obj_tangent(self, s, d):
        """q_s·d·in_s per view, the change of psi_s along d (engine/multislice.rs:375-392)."""
        return ops.obj_probe_to_psi(self.own, d, self.incident[s], self.shared(s))


def multislice_grads(addr, obs, optics, objs, probe):
    """The Poisson LLK sum through the slices and its gradients 2·∂L/∂O_s* per slice and
    2·∂L/∂P*: the exit wave's `poisson_grad` back through the exit transform and the slices'
    adjoints (engine/multislice.rs:266-286, 399-438), each slice's Σ conj(q_s·in_s)·g_s and
    the probe's Σ conj(O_0)·g_0. Returns `(loss, [d_obj per slice], d_probe)`."""
    views, nmode, nframe = addr.views, addr.nmode, addr.nframe
    waves = SliceWaves(optics, views, objs, probe[views["probe"].astype(np.int64)])
    psi = optics.exit_forward(waves.psi)
    loss = ops.llk(obs, slice(0, nframe), nmode, psi).poisson
    g = optics.exit_adjoint(ops.poisson_grad(obs, slice(0, nframe), nmode, psi))
    chis = waves.back_propagate(g)
    d_objs = [waves.obj_adjoint(s, chis[s]) for s in range(len(objs))]
    d_probe = ops.accumulate_probe(views, objs[0], probe.shape, waves.shared(0), chis[0])[0]
    return loss, d_objs, d_probe


class Lsqml:
    """LSQML state across epochs (engine/lsqml.rs:415-430). cost: "poisson" or "amplitude"."""

    def __init__(self, batch_size, cost="poisson", seed=7, offsets=None, refine=False,
                 var=None):
        if batch_size == 0:
            raise ValueError("LSQML batch_size must be >= 1")
        self.batch_size, self.cost, self.seed = batch_size, cost, seed
        self.epochs = 0
        self.preconditioner = None
        self.a_far_all = {}
        # Features::position under Patch sampling: per-frame offsets [P, 2] in object pixels
        self.offsets = None if offsets is None else np.array(offsets, np.float64)
        self.refine = refine
        # ProbeVariation (oracle/opr.py): OPR of probe mode 0, or None for the shared probe
        self.var = var

    def frame_probes(self, frames, probe, quad):
        """`ProbeVariation::unique` planes moved by each frame's offset (engine/lsqml.rs:
        474-499): `[len(frames)·nprobe, ny, nx]`."""
        planes = (self.var.planes(frames, probe) if self.var is not None
                  else np.concatenate([probe] * len(frames)))
        if self.offsets is None:
            return planes
        np_ = probe.shape[0]
        for b, f in enumerate(frames):
            planes[b * np_:(b + 1) * np_] = ops.move_planes(planes[b * np_:(b + 1) * np_], quad,
                                                            self.offsets[f])
        return planes

    @staticmethod
    def unique_views(views, nb, np_, nmode):
        uv = views.copy()
        uv["probe"] = np.repeat(np.arange(nb) * np_, nmode) + views["probe"]
        return uv

    def a_far(self, f):
        return self.a_far_all.get(f, 0.5)

    def batch(self, views, obs, optics, objs, probe):
        """`LsqmlBatch::new` (engine/lsqml.rs:102-179) without probe variation: returns
        `(frames, nmode, waves, chis, a_far, uprobe, uviews)` with `chis` one per slice."""
        nmode = 1
        while nmode < len(views) and views[nmode]["frame"] == views[0]["frame"]:
            nmode += 1
        frames = [int(views[b * nmode]["frame"]) for b in range(len(views) // nmode)]
        ny, nx = probe.shape[-2:]
        uprobe = self.frame_probes(frames, probe, optics.slice_quad(0))
        uviews = self.unique_views(views, len(frames), probe.shape[0], nmode)
        planes = uprobe[uviews["probe"].astype(np.int64)]
        waves = SliceWaves(optics, uviews, objs, planes)
        psi = waves.psi
        chi = optics.exit_forward(psi)
        sh = (len(frames), nmode, ny, nx)
        icalc = (np.abs(chi.reshape(sh)) ** 2).sum(axis=1)
        iobs, mask = obs.iobs[frames], obs.mask[frames]
        keep = ~mask
        if self.cost == "poisson":
            a_far = [self.a_far(f) for f in frames]
            for _ in range(2):
                prev = sum(a_far) / len(a_far)
                for b in range(len(frames)):
                    yt, yp = iobs[b][keep[b]], icalc[b][keep[b]]
                    xi = 1.0 - yt / (yp + EPS_XI)
                    num = float((xi * (yp - yt / (1.0 - prev * xi))).sum())
                    den = float((xi * xi * yp).sum())
                    ratio = num / den if den > 0.0 else 0.0
                    a_far[b] = min(max(0.5 * prev + 0.5 * ratio, 0.0), 1.0)
            c = np.where(mask, 0.0, 1.0 - iobs / (icalc + EPS_POISSON))
        else:
            a_far = [0.5] * len(frames)
            c = np.where(mask, 0.0,
                         2.0 * (1.0 - np.sqrt(np.maximum(iobs, 0.0))
                                / (np.sqrt(icalc) + EPS_AMPLITUDE)))
        fac = 1.0 - np.asarray(a_far)[:, None, None] * c
        chi = (chi.reshape(sh) * fac[:, None]).reshape(chi.shape)
        chi = optics.exit_adjoint(chi) - psi
        chis = waves.back_propagate(chi)
        return frames, nmode, waves, chis, a_far, uprobe, uviews

    def step(self, views, obs, optics, obj, probe):
        """`Lsqml::step` (engine/lsqml.rs:581-643); `obj` is one slice's array or a list of
        slices. Returns the new object(s) and probe and the step record."""
        single = not isinstance(obj, (list, tuple))
        objs = [obj] if single else list(obj)
        pre = self.preconditioner
        floor = (0.1 * pre.max()) ** 2
        frames, nmode, waves, chis, a_far, uprobe, uviews = self.batch(views, obs, optics, objs,
                                                                       probe)
        ny, nx = probe.shape[-2:]
        np_ = probe.shape[0]
        nb = len(frames)
        d_obj = [waves.obj_adjoint(s, chis[s]) / np.sqrt(pre * pre + floor)
                 for s in range(len(objs))]
        # frame_probe_directions on slice 0 (and |V_b|²), moved back by −offset
        d_raw, vv = ops.accumulate_probe(uviews, objs[0], (nb * np_, ny, nx), waves.shared(0),
                                         chis[0])
        d = d_raw.copy()
        if self.offsets is not None:
            for b, f in enumerate(frames):
                d[b * np_:(b + 1) * np_] = ops.move_planes(d[b * np_:(b + 1) * np_],
                                                           optics.slice_quad(0),
                                                           -self.offsets[f])
        d_probe = np.zeros_like(probe)
        for b in range(nb):
            for m in range(np_):
                d_probe[m] += d[b * np_ + m]
        d_probe = d_probe / float(nb)
        a_obj, a_probe = self.step_sizes(views, nmode, optics, objs, waves, chis, d_obj,
                                         d_probe)
        d_pos = None
        if self.refine and self.offsets is not None:
            d_pos = self.position_directions(frames, nmode, optics, objs, waves, chis, uviews)
        for f, a in zip(frames, a_far):
            self.a_far_all[f] = a
        if self.var is not None:
            # the eigenmodes and refined weights from the state on entry (engine/lsqml.rs:
            # 620-621)
            self.var.step(frames, probe[0], d, d_raw, vv, np_)
        new_objs = [o + trim_mean(a) * dd for o, a, dd in zip(objs, a_obj, d_obj)]
        sp = sum(a_probe) / len(a_probe)
        new_probe = probe + sp * d_probe
        if d_pos is not None:
            ops.batch_position_step(self.offsets, frames, d_pos)
        rec = dict(frames=frames, a_far=a_far, a_obj=a_obj[0] if single else a_obj,
                   a_probe=a_probe)
        return (new_objs[0] if single else new_objs), new_probe, rec

    def position_directions(self, frames, nmode, optics, objs, waves, chis, uviews):
        """pty-chi LSQML's gradient position direction per frame on slice nslice/2, from the
        wave entering it at the frame's first view times the slice's phase, its chi and the
        slice's window (engine/lsqml.rs:237-270)."""
        s = len(objs) // 2
        ny, nx = waves.incident[0].shape[-2:]
        sums = []
        for b in range(len(frames)):
            k = b * nmode
            v = uviews[k]
            w = fftshift2(waves.incident[s][k] * waves.shared(s))
            oy, ox = int(v["oy"]), int(v["ox"])
            patch = objs[s][int(v["obj"]), oy:oy + ny, ox:ox + nx]
            sums.append(ops.gradient_sums(patch, w, chis[s][k]))
        eps = ops.EPS_POSITION * optics.intensity_scale()
        return ops.gradient_directions(sums, eps)

    def step_sizes(self, views, nmode, optics, objs, waves, chis, d_obj, d_probe):
        """pty-chi Eq. 22 on slice 0 jointly with the probe, Eq. 23b on the other slices
        (engine/lsqml.rs:286-350)."""
        ny, nx = d_probe.shape[-2:]
        n = ny * nx
        scale = float(len(objs) * nmode)
        dpo = ops.obj_probe_to_psi(views, objs[0], d_probe, waves.shared(0))
        dop = waves.obj_tangent(0, d_obj[0])
        lambda0 = LAMBDA0 * optics.intensity_scale() / n
        nb = len(views) // nmode
        sh = (nb, nmode * n)
        u, v, c = dop.reshape(sh), dpo.reshape(sh), chis[0].reshape(sh)
        a12 = u * np.conj(v)
        s = np.stack([(np.abs(u) ** 2 + lambda0).sum(axis=1),
                      (np.abs(v) ** 2 + lambda0).sum(axis=1),
                      a12.real.sum(axis=1), a12.imag.sum(axis=1),
                      (np.conj(u) * c).real.sum(axis=1),
                      (np.conj(v) * c).real.sum(axis=1)], axis=1)
        reg11, reg22 = 0.1 * (s[:, 0].sum() / nb), 0.1 * (s[:, 1].sum() / nb)
        a_obj0, a_probe = [], []
        for r in s:
            a11, a22 = r[0] + reg11, r[1] + reg22
            det = a11 * a22 - (r[2] * r[2] + r[3] * r[3])
            x0 = (a22 * r[4] - r[2] * r[5]) / det
            x1 = (a11 * r[5] - r[2] * r[4]) / det
            a_obj0.append(0.9 * max(x0, 0.0) / scale)
            a_probe.append(0.9 * max(x1, 0.0))
        a_obj = [a_obj0]
        for sl in range(1, len(objs)):
            du = waves.obj_tangent(sl, d_obj[sl]).reshape(sh)
            cs = chis[sl].reshape(sh)
            num = (np.conj(du) * cs).real.sum(axis=1)
            den = (np.abs(du) ** 2).sum(axis=1)
            a_obj.append([max(0.5 * nu / de * 0.9 / scale, 0.0) for nu, de in zip(num, den)])
        return a_obj, a_probe

    def epoch(self, addr, obs, optics, obj, probe):
        """`Lsqml::epoch` (engine/lsqml.rs:663-714): preconditioner on pty-chi's schedule, then
        `step` over the epoch's seeded batches. Returns `(obj, probe, steps)`."""
        nframe = addr.nframe
        o0 = obj if not isinstance(obj, (list, tuple)) else obj[0]
        if self.epochs < 10 or self.epochs % 10 == 0:
            illum = ops.illumination(addr.views, o0.shape, probe)
            pre = self.preconditioner
            if pre is None:
                n = float(probe.shape[-1] * probe.shape[-2])
                k = optics.intensity_scale()
                power = 0.0
                for f in range(nframe):
                    power = max(power, float(obs.iobs[f][~obs.mask[f]].sum()))
                pre = illum * (power / (4.0 * n * k))
            self.preconditioner = (pre + illum) / 2.0
        epoch = self.epochs
        self.epochs += 1
        size = min(self.batch_size, nframe)
        steps = []
        for frames in random_batches(nframe, size, self.seed, epoch):
            views = np.concatenate([addr.frame_views(f) for f in frames])
            obj, probe, st = self.step(views, obs, optics, obj, probe)
            steps.append(st)
        return obj, probe, steps

    def llk(self, addr, obs, optics, obj, probe):
        """Normalised LLK of the model the steps update, each frame's own (moved) probe,
        through every slice (engine/lsqml.rs:537-551)."""
        objs = [obj] if not isinstance(obj, (list, tuple)) else list(obj)
        frames = list(range(addr.nframe))
        uprobe = self.frame_probes(frames, probe, optics.slice_quad(0))
        uviews = self.unique_views(addr.views, addr.nframe, probe.shape[0], addr.nmode)
        waves = SliceWaves(optics, uviews, objs, uprobe[uviews["probe"].astype(np.int64)])
        psi = optics.exit_forward(waves.psi)
        return ops.llk(obs, slice(0, addr.nframe), addr.nmode, psi).normalised(obs.nb_obs)


def fftshift_planes(a):
    return fftshift2(a)


def slice_jet(optics, views, objs, probe, d_objs, d_probe):
    """The exit waves through the slices and their first and second Taylor coefficients along
    the displacement (d_objs, d_probe): with every slice O_s + γ·dO_s and the probe P + γ·dP,
    the wave entering slice s is w_s + γ·w′_s + γ²·w″_s + O(γ³), w_0 = P, w′_0 = dP, w″_0 = 0,
    and through slice s and its gap G_s: w_{s+1} = G_s(O_s·w_s),
    w′_{s+1} = G_s(O_s·w′_s + dO_s·w_s), w″_{s+1} = G_s(O_s·w″_s + dO_s·w′_s); the exit
    multiplies by q·(O_last + γ·dO_last) the same way. Returns (ψ, ψ′, ψ″) in the detector
    plane (the exit transform applied), shifted, one plane per view. One slice gives PyNX's
    (po, a, b) of `cg_gamma` (engine/ptycho.rs:517-545)."""
    own = views.copy()
    own["probe"] = np.arange(len(views))
    pk = views["probe"].astype(np.int64)
    w, w1, w2 = probe[pk], d_probe[pk], np.zeros_like(probe[pk])
    ny, nx = w.shape[-2:]
    one = _unit((ny, nx))
    n = len(objs)
    for s in range(n):
        q = optics.slice_quad(s)
        q = one if q is None else q
        t0 = ops.obj_probe_to_psi(own, objs[s], w, q)
        t1 = ops.obj_probe_to_psi(own, objs[s], w1, q) + ops.obj_probe_to_psi(own, d_objs[s], w, q)
        t2 = ops.obj_probe_to_psi(own, objs[s], w2, q) + ops.obj_probe_to_psi(own, d_objs[s], w1, q)
        if s + 1 == n:
            return tuple(optics.exit_forward(t) for t in (t0, t1, t2))
        gap = optics.gaps[s]
        w, w1, w2 = (fftshift2(gap.forward(t)) for t in (t0, t1, t2))


def multislice_ml(addr, obs, optics, objs, probe, ncycle, update_object=True,
                  update_probe=True, calc_llk=0):
    """Poisson ML conjugate gradient through pty-chi's multislice object (this build's
    definition; the reference runs ML on one slice, engine/ptycho.rs:775-842): the opening
    rescale of the probe to the data's photons, per cycle the gradients through the slices
    (`multislice_grads`), the Polak–Ribière β over every slice and the probe, and PyNX's
    Poisson line search `cg_poisson_gamma` on the second-order expansion of the exit waves
    along the direction (`slice_jet`). Returns (objs, probe, llk records)."""
    objs, probe = [o.copy() for o in objs], probe.copy()
    nframe, nmode = addr.nframe, addr.nmode
    views = addr.views
    frames = slice(0, nframe)

    def llk_now():
        waves = SliceWaves(optics, views, objs, probe[views["probe"].astype(np.int64)])
        return ops.llk(obs, frames, nmode, optics.exit_forward(waves.psi))

    calc = llk_now().nb_photons_calc
    probe = probe * np.sqrt(obs.total() / calc)
    last = None
    d_objs = [np.zeros_like(o) for o in objs]
    d_probe = np.zeros_like(probe)
    records = []
    for ic in range(ncycle):
        if calc_llk > 0 and (ic % calc_llk == 0 or ic + 1 == ncycle):
            records.append(llk_now().normalised(obs.nb_obs))
        _, go, gp = multislice_grads(addr, obs, optics, objs, probe)
        if not update_object:
            go = [np.zeros_like(o) for o in objs]
        if not update_probe:
            gp = np.zeros_like(probe)
        if last is None:
            beta = 0.0
        else:
            num = sum((np.conj(g) * (g - l)).real.sum() for g, l in zip(go, last[0]))
            num += (np.conj(gp) * (gp - last[1])).real.sum()
            den = sum((np.abs(l) ** 2).sum() for l in last[0]) + (np.abs(last[1]) ** 2).sum()
            with np.errstate(divide="ignore", invalid="ignore"):
                beta = num / den
            if not (np.isfinite(beta) and beta >= 0.0):
                beta = 0.0
        d_objs = [d * beta - g for d, g in zip(d_objs, go)]
        d_probe = d_probe * beta - gp
        po, a, b = slice_jet(optics, views, objs, probe, d_objs, d_probe)
        num, den = ops.cg_poisson_gamma(obs, frames, nmode, po, a, b)
        with np.errstate(divide="ignore", invalid="ignore"):
            gamma = np.float64(num) / np.float64(den)
        if np.isfinite(gamma):
            objs = [o + d * gamma for o, d in zip(objs, d_objs)]
            probe = probe + d_probe * gamma
        else:
            d_objs, d_probe = [-g for g in go], -gp
        last = (go, gp)
    return objs, probe, records
