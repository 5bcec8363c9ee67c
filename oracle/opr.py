"""pty-chi's orthogonal probe relaxation (OPR) of probe mode 0 in float64 (oracle restatement,
test infrastructure only), following physwkim/ptyrs `ptyrs/src/engine/opr.rs`: with `k`
eigenmodes `U_i`, frame `f` sees `P_f0 = c_f·P_0 + Σ_i w_fi·U_i` and `P_fm = P_m` for `m ≥ 1`;
`c_f` is 1 unless modelled. `Lsqml(var=...)` runs its steps on these per-frame probes and moves
the eigenmodes and the refined weights with each step.
"""
import numpy as np

from . import ops
from .base import fftshift2


def _dot(a, b):
    """`Σ Re(conj(a)·b)` (engine/opr.rs:226-229)."""
    return float((np.conj(a) * b).real.sum())


def _mnorm(x):
    """`√(mean |x|²)` (engine/opr.rs:231-234)."""
    return float(np.sqrt((np.abs(x) ** 2).sum() / x.size))


class ProbeVariation:
    """`ProbeVariation` (engine/opr.rs:17-88): eigenmodes `[k, ny, nx]`, frame-major weights
    `w[f·k + i]` and, when modelled, the main mode's weights `c[f]`, each refined or held."""

    def __init__(self, eigenmodes, weights, refine_weights=True, intensity=None,
                 refine_intensity=True):
        self.eigenmodes = np.array(eigenmodes, np.complex128)
        self.weights = np.array(weights, np.float64)
        self.refine_weights = refine_weights
        self.intensity = None if intensity is None else np.array(intensity, np.float64)
        self.refine_intensity = refine_intensity
        k = len(self.eigenmodes)
        if (k == 0 and len(self.weights)) or (k and len(self.weights) % k):
            raise ValueError(f"{len(self.weights)} weights for {k} eigenmodes")

    @property
    def k(self):
        return len(self.eigenmodes)

    def planes(self, frames, probe):
        """`unique`'s planes (engine/opr.rs:88-120): for each frame in order,
        `c_f·P_0 + w_f0·U_0 + w_f1·U_1 + …`, then `P_1 ..`; `[len(frames)·nprobe, ny, nx]`."""
        out = []
        k = self.k
        for f in frames:
            c = 1.0 if self.intensity is None else self.intensity[f]
            p0 = c * probe[0]
            for i in range(k):
                p0 = p0 + self.weights[f * k + i] * self.eigenmodes[i]
            out.append(p0)
            out.extend(probe[1:])
        return np.array(out)

    def step(self, frames, probe0, moved, d, vv, np_):
        """`ProbeVariation::step` (engine/opr.rs:122-224), pty-chi's
        `update_opr_probe_modes_and_weights`: `d`, `vv` the batch's plane-b·nprobe frame probe
        directions `conj(q·V_b)·chi_b0` and `|V_b|²`, `moved` `d` taken back through the frames'
        moves (`d` itself without offsets), `probe0` the shared probe's mode 0."""
        count = len(frames)
        if self.intensity is not None and self.refine_intensity:
            pp = np.abs(probe0) ** 2
            for b, f in enumerate(frames):
                den = float((pp * vv[b * np_]).sum())
                self.intensity[f] += 0.1 * _dot(probe0, d[b * np_]) / den
        k = self.k
        if k == 0 or count < 2:
            return
        n = float(probe0.size)
        mean = sum(moved[b * np_] for b in range(count)) / count
        r = [moved[b * np_] - mean for b in range(count)]
        a_u = min(0.1, count / (len(self.weights) / k))
        for i in range(k):
            w = [float(self.weights[f * k + i]) for f in frames]
            w2 = sum(x * x for x in w)
            u = self.eigenmodes[i]
            e = np.zeros_like(u)
            for rb, wb in zip(r, w):
                e = e + rb * ((_dot(rb, u) / (n * n) + wb) / w2)
            e = e / count
            u = u + (a_u * np.sqrt(n) / _mnorm(e)) * e
            u = u * (np.sqrt(n) / _mnorm(u))
            if self.refine_weights:
                den = [float((np.abs(u) ** 2 * vv[b * np_]).sum()) for b in range(count)]
                reg = 0.1 * sum(den) / count
                for b, f in enumerate(frames):
                    self.weights[f * k + i] = w[b] + _dot(u, d[b * np_]) / (den[b] + reg)
            if i + 1 < k:
                uu = float((np.abs(u) ** 2).sum())
                for b in range(count):
                    c = (r[b] * np.conj(u)).sum() / uu
                    r[b] = r[b] - c * u
            self.eigenmodes[i] = u


def frame_views(addr, frames):
    return np.concatenate([addr.frame_views(f) for f in frames])


def unique_views(views, nb, np_, nmode):
    uv = views.copy()
    uv["probe"] = np.repeat(np.arange(nb) * np_, nmode) + views["probe"]
    return uv


def opr_weight_grad(cost, views, obs, optics, obj, probe, var):
    """`opr_weight_grad` (engine/opr.rs:236-271): `∂cost/∂w_bi` for every frame of `views`
    (whole frames, in order) and eigenmode `i`, frame-major, as `<U_i, g_b0>` with `g` the
    gradient over each frame's own probe planes, accumulate_probe of `F⁻¹(2·slope·psi)`;
    `slope` 1 − I/Ĩ (Poisson) or 1 − √(I/Ĩ) (amplitude), Ĩ floored at 1e-12."""
    np_ = probe.shape[0]
    nmode = 1
    while nmode < len(views) and views[nmode]["frame"] == views[0]["frame"]:
        nmode += 1
    frames = [int(views[b * nmode]["frame"]) for b in range(len(views) // nmode)]
    uprobe = var.planes(frames, probe)
    uviews = unique_views(views, len(frames), np_, nmode)
    q = optics.quad
    psi = optics.exit_forward(ops.obj_probe_to_psi(uviews, obj, uprobe, q))
    ny, nx = probe.shape[-2:]
    sh = (len(frames), nmode, ny, nx)
    icalc = np.maximum((np.abs(psi.reshape(sh)) ** 2).sum(axis=1), 1e-12)
    iobs, mask = obs.iobs[frames], obs.mask[frames]
    slope = 1.0 - iobs / icalc if cost == "poisson" else 1.0 - np.sqrt(iobs / icalc)
    s = np.where(mask, 0.0, 2.0 * slope)
    psi = optics.exit_adjoint((psi.reshape(sh) * s[:, None]).reshape(psi.shape))
    g, _ = ops.accumulate_probe(uviews, obj, uprobe.shape, q, psi)
    k = var.k
    return np.array([_dot(var.eigenmodes[bi % k], g[(bi // k) * np_])
                     for bi in range(len(frames) * k)])
