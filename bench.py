"""Throughput of the reconstruction hot path on B200: diffraction patterns·iterations per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ml256|lsqml128|opr128|rpie64|ms128|msml128|batch32|dm256|raar256|ap256]

Workload `ml256` (default; the configuration the metric names, a 256² probe): Poisson
maximum-likelihood conjugate gradient with position refinement — a 2048² smooth-noise object,
a 256² probe with 2 incoherent modes (powers 0.8/0.2), a 10000-position Fermat scan at 12 px
whose frames were taken at true positions off the nominal ones by seeded N(0, 1.5 px)
offsets (the solver gets the nominal positions and refines sub-pixel offsets under the Patch
model), Poisson counts at 1e7 photons per pattern, FP32. A step is one ML cycle over all 10000
patterns: the position sums from the magnitude projection, the object and probe gradients,
the Polak–Ribière direction, the Poisson line search, the update and the position step.
`lsqml128`: the LSQML configuration (1024² object, 128² probe × 3 modes, Fermat 4096 at 6 px,
1e6 photons, batches of 256, Poisson cost), a step one epoch; `opr128` the same with pty-chi's
OPR probe variation of mode 0 (2 eigenmodes, their weights and the main mode's refined). `rpie64`: the rPIE
configuration (256² object, 64² probe, 20×20 raster, batch 100), a step one epoch. Inputs
live in HBM before the timed region; the counts of `ml256` (2.6 GB) and `lsqml128` (268 MB)
are larger than the 126 MB L2, so no flush is needed between steps.

The timed region is bracketed by CUDA events on the engine's own stream (its device time of
the K steps) with a synchronize and, for N > 1, a barrier on both sides; N > 1 runs N
independent replicas (one scan per GPU; the path has no exchange step), the time is the max
over ranks and the value the patterns of all ranks over it.

`--impl reference` times the reference's CPU path on the host cores: the reference engine is
Rust and cannot be built in this image, so its numpy float64 restatement (`oracle/`) runs on a
bounded sample of the workload (one ML cycle over the first frames of the scan, or one batch
update of LSQML / rPIE per step), its FFTs on every host thread.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}

WORKLOADS = {
    "ml256": dict(kind="ml256", algorithm="ml", refine=True, sample_frames=48,
                  desc="ML (Poisson CG) with position refinement, 2048^2 object, 256^2 probe x2 "
                       "modes, Fermat 10000 @ 12 px, true positions off the nominal by "
                       "N(0, 1.5 px), 1e7 photons"),
    "lsqml128": dict(kind="lsqml128", algorithm="lsqml", batch=256, cost="poisson",
                     desc="LSQML, 1024^2 object, 128^2 probe x3 modes, Fermat 4096 @ 6 px, "
                          "1e6 photons, batch 256, Poisson"),
    "rpie64": dict(kind="rpie64", algorithm="rpie", batch=100,
                   desc="rPIE, 256^2 object, 64^2 probe, 20x20 raster 8 px +-1 px, "
                        "1e5 photons, batch 100, alpha=beta=0.1"),
    # the LSQML configuration with pty-chi's OPR probe variation of mode 0 (2 eigenmodes, the
    # per-frame weights and main-mode weights refined)
    "opr128": dict(kind="lsqml128", algorithm="lsqml", batch=256, cost="poisson", opr=2,
                   desc="LSQML with OPR probe variation (2 eigenmodes, weights and main-mode "
                        "weights refined), 1024^2 object, 128^2 probe x3 modes, Fermat 4096 @ "
                        "6 px, 1e6 photons, batch 256, Poisson"),
    # pty-chi's multislice object (3 slices) under LSQML, the multislice configuration's shapes
    "ms128": dict(kind="ms128", algorithm="lsqml", batch=256, cost="poisson",
                  desc="multislice LSQML, 3 slices of 1536^2 10 um apart (angular spectrum, "
                       "lambda 0.1 nm, 10 nm pixels), 128^2 probe x2 modes, Fermat 6000 @ "
                       "12 px, 1e6 photons, batch 256, Poisson"),
    # the multislice configuration's ML: Poisson CG through the three slices
    "msml128": dict(kind="ms128", algorithm="ml", sample_frames=48,
                    desc="multislice ML (Poisson conjugate gradient through the slices, object "
                         "and probe), 3 slices of 1536^2 10 um apart (angular spectrum, lambda "
                         "0.1 nm, 10 nm pixels), 128^2 probe x2 modes, Fermat 6000 @ 12 px, 1e6 "
                         "photons"),
    # 32 independent uneven scans at once (ptyb_batch_run), each step one whole reconstruction:
    # 30 rPIE epochs (batches of 100) then 30 LSQML epochs (batches of 256) on every scan
    "batch32": dict(kind="batch32", algorithm="batch", batch=100, lsqml_batch=256,
                    rpie_epochs=30, lsqml_epochs=30,
                    desc="32 independent seeded scans at once (one stream each): sides from "
                         "{64, 96, 128, 192, 256}, objects 4-8x the side, 500-5000 Fermat positions, "
                         "1e4-1e7 photons (log-uniform), one probe mode; per step one whole "
                         "reconstruction of every scan: 30 rPIE epochs (batches of 100, alpha "
                         "0.1) then 30 LSQML epochs (batches of 256, Poisson)"),
    # the reference's own AP / DM benchmark shape: Fermat 4096 frames, 256^2, 2 modes
    "dm256": dict(kind="fermat256", algorithm="dm", sample_frames=48,
                  desc="DM (PyNX defaults: alpha 0.02, object inertia 0.01, probe inertia "
                       "0.001), 1280^2 object, 256^2 probe x2 modes, Fermat 4096 @ 12 px, "
                       "1e7 photons"),
    "raar256": dict(kind="fermat256", algorithm="raar", sample_frames=48,
                    desc="RAAR (PyNX defaults: beta 0.9, object inertia 0.01, probe inertia "
                         "0.001), 1280^2 object, 256^2 probe x2 modes, Fermat 4096 @ 12 px, "
                         "1e7 photons"),
    "ap256": dict(kind="fermat256", algorithm="ap", sample_frames=48,
                  desc="AP (object inertia 0.01, probe inertia 0.001), 1280^2 object, 256^2 "
                       "probe x2 modes, Fermat 4096 @ 12 px, 1e7 photons"),
}

# Algorithms whose step is one cycle over every frame (the bounded CPU sample runs cycles over
# the scan's first frames); the others step through seeded batches.
CYCLES = ("ml", "dm", "raar", "ap")


def dist_env():
    from ptyrs_b200.replicas import env
    return env()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_inputs(workload, seed, scale=1.0):
    from ptyrs_b200 import sim
    return sim.make_scan(WORKLOADS[workload]["kind"], seed=seed, scale=scale)


def prepare(g, s, wl):
    """The workload's features on a fresh state: ML starts at the nominal positions with the
    sub-pixel offsets refined."""
    if wl["algorithm"] == "ml" and "refine" in wl:
        g.set_positions(np.zeros((len(s["counts"]), 2)), refine=wl["refine"])
    if wl.get("opr"):
        u, w, c = opr_start(s, wl)
        g.set_probe_variation(u, w, intensity=c)


def opr_start(s, wl):
    from ptyrs_b200 import sim
    return sim.opr_start(s["probe"], len(s["counts"]), wl["opr"])


def oracle_variation(s, wl):
    """The oracle's copy of the workload's OPR start, or None without one."""
    if not wl.get("opr"):
        return None
    from oracle.opr import ProbeVariation
    u, w, c = opr_start(s, wl)
    return ProbeVariation(u, w.ravel(), intensity=c)


def run_algorithm(g, wl, nepoch):
    if wl["algorithm"] == "ml":
        g.ml(nepoch, update_object=True, update_probe=True, calc_llk=0, zero_phase_ramp=False)
    elif wl["algorithm"] in ("dm", "raar"):
        getattr(g, wl["algorithm"])(nepoch, calc_llk=0, zero_phase_ramp=False)
    elif wl["algorithm"] == "ap":
        g.ap(nepoch, probe_inertia=0.001, calc_llk=0, zero_phase_ramp=False)
    elif wl["algorithm"] == "lsqml":
        g.lsqml(nepoch, batch_size=wl["batch"], cost=wl["cost"], seed=7)
    else:
        g.rpie(nepoch, batch_size=wl["batch"], obj_alpha=0.1, probe_alpha=0.1, seed=7)


def algorithmic_bytes(kind, s, wl):
    """Bytes a launch of `kind` must move from HBM per frame it processes: the unique inputs it
    reads and the outputs it writes (object window 8·N², counts 4·N², per-mode planes 8·K·N²);
    the shared probe, phase and twiddles are L2-resident, the moved per-frame probes of the
    position model are not."""
    n2 = s["n"] ** 2
    K = s["probe"].shape[0]
    S = s["object"].shape[0] if s.get("gaps") else 1
    moved = 8 * K * n2 if wl.get("refine") else 0
    # OPR: every frame's own probe planes, written per batch and read by the frame pass
    planes = 8 * K * n2 if wl.get("opr") else 0
    table = {
        "frame_store": 8 * n2 + 8 * K * n2 + 4 * n2,
        "frame_from_store": 8 * K * n2 + 4 * n2 + 8 * n2 + 8 * K * n2,
        "frame_rpie": 8 * n2 + 4 * n2 + 8 * K * n2,
        "frame_lsqml": 8 * n2 + 4 * n2 + 8 * K * n2 + planes,
        "frame_llk": 8 * n2 + 4 * n2 + moved,
        # gradient pass: object window, counts, (moved probe), Ψ kept and g written
        "frame_ml_grad": 8 * n2 + 4 * n2 + 16 * K * n2 + moved,
        # projection from the kept Ψ: Ψ read, object window, counts, (moved probe), change
        "frame_project": 8 * n2 + 4 * n2 + 16 * K * n2 + moved,
        # line search: object and direction windows, counts, kept Ψ and g, (moved probe and
        # direction); through slices every slice's object and direction windows and the counts
        "ml_gamma": (16 * n2 * S + 4 * n2 if S > 1
                     else 16 * n2 + 4 * n2 + 16 * K * n2 + 2 * moved),
        "move": 8 * K * n2,
        "back_spectrum": 16 * K * n2 + 8 * n2,
        "deriv_sums": 8 * K * n2 + 8 * n2,
        "position_sums": 16 * K * n2 + 8 * n2,
        "probe_partial": 8 * K * n2 + 8 * n2,
        "lsqml_dots": 8 * K * n2 + 16 * n2,
        "object_lsqml": 8 * K * n2,
        "object_rpie": 8 * K * n2,
        "object_ml": 8 * K * n2 + moved,
        # AP / DM / RAAR: object window, counts, the carried waves read and written (RAAR also
        # its iterate)
        "frame_carry": 8 * n2 + 4 * n2 + (32 if wl["algorithm"] == "raar" else 16) * K * n2,
        "object_blend": 8 * K * n2,
        # OPR step per frame of a batch: the frame's object window (|O|² weights) and its
        # mode-0 probe direction read, its own K probe planes written
        "opr_step": 8 * n2 + 8 * n2 + 8 * K * n2,
        # multislice: every slice's window and the counts; forward writes the incident waves
        # of slices 1.. and the detector field, backward reads them and writes every slice's χ
        "slice_forward": 8 * n2 * S + 4 * n2 + 8 * K * n2 * S,
        "slice_backward": 4 * n2 + 8 * n2 * S + 16 * K * n2 * S,
        # ML's gradient through the slices: every slice's window and the counts read, the
        # incident waves of slices 1.. and every slice's gradient field written
        "slice_grad": 8 * n2 * S + 4 * n2 + 8 * K * n2 * (S - 1) + 8 * K * n2 * S,
    }
    return table.get(kind)


# 2-D transforms of one K-plane stack per frame each kernel runs (forward and inverse count one
# each); the FFT's FP32 work is 5·N²·log2(N²) per plane and transform.
FFT_PASSES = {"frame_rpie": 2, "frame_lsqml": 2, "frame_ml_grad": 2, "frame_project": 1,
              "frame_llk": 1, "frame_store": 1, "frame_from_store": 1, "frame_carry": 2,
              "ml_gamma": 1, "move": 1, "back_spectrum": 1, "deriv_sums": 2}
# FP32 lanes × 2 flops × clock: 148 SMs × 128 × 2 × 1.965 GHz
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def fft_flops(kind, s):
    """FP32 flops of a kernel's FFTs per frame, None for kernels without per-frame FFTs."""
    passes = FFT_PASSES.get(kind)
    if passes is None:
        return None
    n2 = s["n"] ** 2
    return passes * s["probe"].shape[0] * 5.0 * n2 * np.log2(n2)


def sample_scan(s, m):
    """The first `m` frames of the scan, its object and probe starts (a bounded sample)."""
    return dict(s, counts=s["counts"][:m], y=s["y"][:m], x=s["x"][:m])


# DRAM bytes per frame of a kernel (ncu dram__bytes_read.sum + dram__bytes_write.sum of one
# launch over its frames) on a cut of the workload's scan: roofline.traffic scales them to the
# launch's frames.
NCU_DRAM_BYTES_PER_FRAME = {
    # the 1000-frame cut of the ml256 scan, one 488-frame launch of each
    "ml256": {"frame_ml_grad": 3.35e6, "deriv_sums": 1.06e6},
    # the carry pass on the 1024-frame cut of the dm256 scan
    "dm256": {"frame_carry": 2.33e6},
}
NCU_PROFILE = {"ml256": "profiles/ml_gradient_and_position_sums_ml256.md (a 1000-frame cut)",
               "dm256": "profiles/dm256_launch_list.md (a 1024-frame cut)"}


def oracle_optics(s):
    """The oracle's optics of the scan: the far field of its geometry, through its slices when
    it has gaps."""
    from oracle import ops
    n = s["n"]
    optics = ops.Optics.far_field(s["wavelength"], s["distance"], s["detector_pixel"], [n, n])
    if s.get("gaps"):
        optics = optics.with_slices([ops.Wavefield([n, n], s["wavelength"], optics.pixel, z)
                                     for z in s["gaps"]])
    return optics


def oracle_objects(s):
    """The start object as the oracle takes it: one array, or a list of [1, ny, nx] slices."""
    if s.get("gaps"):
        return [s["object"][k:k + 1] for k in range(s["object"].shape[0])]
    return s["object"]


def _threads(n):
    """numpy's FFT workers and the BLAS pools limited to `n` threads (None: all)."""
    from oracle import ops
    from threadpoolctl import threadpool_limits
    ops.FFT_WORKERS = n
    return threadpool_limits(limits=n)


def cpu_cycles(s, wl, m, cycles, threads):
    """`cycles` cycles (one call, as the GPU step) of the oracle over the first `m` frames of
    the scan with the full object; returns the seconds and the oracle state."""
    from oracle.ptycho import Ptycho
    t = sample_scan(s, min(m, len(s["counts"])))
    if s.get("gaps"):
        # ML through the slices (oracle.lsqml.multislice_ml); the state keeps every slice
        from oracle.lsqml import multislice_ml
        optics = oracle_optics(s)
        p = Ptycho(t["counts"], t["y"], t["x"], optics, t["object"][:1], t["probe"])
        with _threads(threads):
            t0 = time.perf_counter()
            objs, probe, _ = multislice_ml(p.addr, p.obs, optics, oracle_objects(t), p.probe,
                                           cycles)
            dt = time.perf_counter() - t0
        from oracle import ops
        ops.FFT_WORKERS = None
        p.object, p.probe = np.concatenate(objs), probe
        return dt, p
    p = Ptycho(t["counts"], t["y"], t["x"], oracle_optics(s), t["object"], t["probe"])
    with _threads(threads):
        if wl["algorithm"] == "ml" and "refine" in wl:
            p.set_positions(np.zeros((p.addr.nframe, 2)), refine=wl["refine"])
        t0 = time.perf_counter()
        if wl["algorithm"] == "ml":
            p.ml(cycles, update_object=True, update_probe=True, calc_llk=0,
                 zero_phase_ramp=False)
        elif wl["algorithm"] == "ap":
            p.ap(cycles, probe_inertia=0.001, calc_llk=0, zero_phase_ramp=False)
        else:
            getattr(p, wl["algorithm"])(cycles, calc_llk=0, zero_phase_ramp=False)
        dt = time.perf_counter() - t0
    from oracle import ops
    ops.FFT_WORKERS = None
    return dt, p


def cycle_fit(s, wl, threads, cycles=2, reps=1):
    """The oracle's cycle time over the whole scan, from cycles over its first m/2 and m frames
    (m = wl["sample_frames"]) with the full object: T(m) = a + b·m separates the object-sized
    work of a cycle (a: gradients, conjugate directions, line-search sums and updates over
    every object pixel) from the per-frame work (b), so the sample's few frames do not carry
    the whole object's work. Returns patterns·iter/s over the scan's P frames, P / (a + b·P),
    the fit, and the larger sample's oracle state."""
    m2 = min(wl["sample_frames"], len(s["counts"]))
    m1 = max(1, m2 // 2)
    t1 = t2 = 0.0
    for _ in range(reps):
        t1 += cpu_cycles(s, wl, m1, cycles, threads)[0] / cycles
        d, state = cpu_cycles(s, wl, m2, cycles, threads)
        t2 += d / cycles
    t1, t2 = t1 / reps, t2 / reps
    b = max((t2 - t1) / (m2 - m1), 1e-12)
    a = max(t1 - b * m1, 0.0)
    P = len(s["counts"])
    fit = {"object_s_per_cycle": a, "frame_s": b, "samples": [[m1, t1], [m2, t2]],
           "cycles_per_sample": cycles * reps}
    return P / (a + b * P), fit, state


def cpu_batches(s, wl, seconds, threads):
    """Successive batch updates (`wl["batch"]` frames, the seeded order of the GPU run) of the
    oracle from the same start until `seconds` pass (at least one). Returns patterns·iter/s,
    the pattern-iterations done, the seconds and the oracle state."""
    from oracle import ops
    from oracle.base import random_batches
    from oracle.lsqml import Lsqml
    from oracle.ptycho import Ptycho
    optics = oracle_optics(s)
    p = Ptycho(s["counts"], s["y"], s["x"], optics, s["object"][:1], s["probe"])
    batches = random_batches(p.addr.nframe, wl["batch"], 7, 0)
    done = 0
    obj, probe = oracle_objects(s), p.probe
    with _threads(threads):
        t0 = time.perf_counter()
        if wl["algorithm"] == "lsqml":
            run = Lsqml(wl["batch"], wl["cost"], 7, var=oracle_variation(s, wl))
            run.preconditioner = ops.illumination(p.addr.views, p.object.shape, probe)
        for frames in batches:
            views = np.concatenate([p.addr.frame_views(f) for f in frames])
            if wl["algorithm"] == "lsqml":
                obj, probe, _ = run.step(views, p.obs, optics, obj, probe)
            else:
                p.rpie_batch(frames, 1.0, 1.0, 0.1, 0.1)
            done += len(frames)
            if time.perf_counter() - t0 > seconds:
                break
        dt = time.perf_counter() - t0
    ops.FFT_WORKERS = None
    return done / dt, done, dt, p


def cpu_baseline(s, wl, threads, seconds=15.0):
    """The oracle (numpy float64 restatement of the reference's CPU engine) on the host cores
    for `s`'s workload, like for like with the GPU step: for cycle algorithms the whole-scan
    cycle time from cycle_fit, for batch algorithms batch updates of the run's own size.
    Returns the cpu_baseline object of the bench line and the oracle state of its sample."""
    if wl["algorithm"] in CYCLES:
        v, fit, state = cycle_fit(s, wl, threads)
        what = (f"{wl['algorithm'].upper()} cycles"
                + (" with position refinement" if wl["algorithm"] == "ml" else "")
                + f" over the first {fit['samples'][0][0]} and {fit['samples'][1][0]} frames "
                  f"({fit['cycles_per_sample']} per sample) with the full object, "
                  f"{fit['samples'][0][1]:.2f} s and {fit['samples'][1][1]:.2f} s per cycle; "
                  f"a cycle over all {len(s['counts'])} frames = {fit['object_s_per_cycle']:.2f} "
                  f"s object-sized work + {1e3 * fit['frame_s']:.1f} ms per frame, extrapolated")
        out = {"value": v, "unit": "patterns*iter/s", "cores": threads, "kind": "port",
               "sample": what + f", numpy float64 on {threads} threads", "fit": fit}
        return out, state
    v, done, secs, state = cpu_batches(s, wl, seconds, threads)
    out = {"value": v, "unit": "patterns*iter/s", "cores": threads, "kind": "port",
           "sample": f"{done} pattern-iterations ({done // wl['batch']} batch updates of "
                     f"{wl['batch']} frames of the scan) in {secs:.1f} s, numpy float64 on "
                     f"{threads} threads"}
    return out, state


def object_nrmse(a, b, weight):
    """Object NRMSE with the global phase and a linear phase ramp removed and the scale kept
    (ptyrs_b200.metrics)."""
    from ptyrs_b200.metrics import object_nrmse as nrmse
    return nrmse(a, b, weight)


def accuracy(s, wl, oracle_state, device, cycles=2):
    """The FP32 GPU path against the float64 oracle on the bounded sample of cycles: object
    NRMSE after the global phase and phase ramp, scale kept, over the illuminated pixels
    (illumination ≥ 1e-3 of its max), and for ML the largest difference of the refined
    offsets."""
    from oracle import ops
    from ptyrs_b200 import GpuPtycho, Scan
    t = sample_scan(s, oracle_state.addr.nframe)
    scan = Scan(t["counts"], t["y"], t["x"], t["wavelength"], t["distance"], t["detector_pixel"])
    gaps = s.get("gaps")
    with GpuPtycho(scan, t["object"], t["probe"], device=device, gaps=gaps) as g:
        prepare(g, t, wl)
        run_algorithm(g, wl, cycles)
        obj = g.objects() if gaps else g.object()
        d = g.positions() if wl["algorithm"] == "ml" and "refine" in wl else None
    illum = ops.illumination(oracle_state.addr.views, oracle_state.object[:1].shape,
                             oracle_state.probe)
    w = np.broadcast_to(illum >= 1e-3 * illum.max(), obj.shape).astype(float)
    out = {"object_nrmse_vs_f64": object_nrmse(obj, oracle_state.object, w),
           "sample": f"{cycles} {wl['algorithm'].upper()} cycles over the first "
                     f"{t['counts'].shape[0]} frames, GPU FP32 vs the float64 oracle from the "
                     "same start"}
    if d is not None:
        out["offsets_max_abs_diff_px"] = float(np.abs(d - oracle_state.offsets).max())
    return out


def accuracy_batches(s, wl, device, nbatch=None):
    """rPIE and LSQML: one epoch over the first `nbatch` batches' frames of the scan (the same
    seeded batches) on the GPU in FP32 and in the float64 oracle from the same start; object
    NRMSE after the global phase and phase ramp, scale kept, over the illuminated pixels."""
    from oracle import ops
    from oracle.lsqml import Lsqml
    from oracle.ptycho import Ptycho
    from ptyrs_b200 import GpuPtycho, Scan
    if nbatch is None:
        nbatch = 1 if s.get("gaps") else 2
    t = sample_scan(s, min(len(s["counts"]), nbatch * wl["batch"]))
    optics = oracle_optics(t)
    p = Ptycho(t["counts"], t["y"], t["x"], optics, t["object"][:1], t["probe"])
    if wl["algorithm"] == "lsqml":
        run = Lsqml(wl["batch"], wl["cost"], 7, var=oracle_variation(t, wl))
        ref, _, _ = run.epoch(p.addr, p.obs, optics, oracle_objects(t), p.probe)
    else:
        p.rpie(1, batch_size=wl["batch"], obj_alpha=0.1, probe_alpha=0.1, seed=7)
        ref = p.object
    ref = np.concatenate(ref) if isinstance(ref, list) else ref
    scan = Scan(t["counts"], t["y"], t["x"], t["wavelength"], t["distance"], t["detector_pixel"])
    with GpuPtycho(scan, t["object"], t["probe"], device=device, gaps=t.get("gaps")) as g:
        prepare(g, t, wl)
        run_algorithm(g, wl, 1)
        obj = g.objects()
    illum = ops.illumination(p.addr.views, p.object.shape, p.probe)
    w = np.broadcast_to(illum >= 1e-3 * illum.max(), obj.shape).astype(float)
    return {"object_nrmse_vs_f64": object_nrmse(obj, ref, w),
            "sample": f"one {wl['algorithm']} epoch over the first {len(t['counts'])} frames "
                      f"(batches of {wl['batch']}), GPU FP32 vs the float64 oracle from the "
                      "same start"}


# Time to target (the reference's method, refs/py/time_to_target_ptychi.py): long runs fix an
# LLK target, then timed runs of each algorithm to it from the same start.
TTT_ALGOS = ("rpie", "lsqml", "ml")
TTT_LABELS = {"rpie": "rPIE (alpha = beta = 0.1, batches of 100)",
              "lsqml": "LSQML (Poisson, batches of 100)",
              "ml": "ML (Poisson conjugate gradient, object and probe)"}


def ttt_call(g, algo, n, calc_llk=0):
    """`n` iterations of `algo` in one call from the handle's current state."""
    if algo == "rpie":
        g.rpie(n, batch_size=100, obj_alpha=0.1, probe_alpha=0.1, calc_llk=calc_llk, seed=7)
    elif algo == "lsqml":
        g.lsqml(n, calc_llk=calc_llk, batch_size=100, cost="poisson", seed=7)
    else:
        g.ml(n, update_object=True, update_probe=True, calc_llk=calc_llk, zero_phase_ramp=False)


def llk_after(algo, trace):
    """The Poisson LLK after 1, 2, … iterations from a call's LLK records (rPIE and LSQML record
    the state after each epoch; ML the state a cycle starts from, so its first record is the
    start and the last cycle's result is not recorded): entry i is the LLK after i + 1
    iterations."""
    trace = list(trace)
    return trace[1:] if algo == "ml" else trace


def ttt_targets(traces, margin=1.01):
    """The targets of the long runs' LLK traces (`llk_after` form) and each algorithm's
    iterations to them: the first target is `margin` times the lowest final LLK; when some
    algorithm never reaches it, a second target is `margin` times the highest final among
    those (the reference's rule), which every algorithm then reaches. An algorithm whose long
    run diverged (a non-finite final LLK) sets no target and reaches none. Returns a list of
    (target, {algo: iterations or None})."""
    finals = {a: float(t[-1]) for a, t in traces.items() if np.isfinite(t[-1])}

    def reach(target):
        out = {}
        for a, t in traces.items():
            hit = [i for i, v in enumerate(t) if v <= target]
            out[a] = hit[0] + 1 if hit else None
        return out

    first = margin * min(finals.values())
    targets = [(first, reach(first))]
    missed = [a for a, c in targets[0][1].items() if c is None and a in finals]
    if missed:
        second = margin * max(finals[a] for a in missed)
        targets.append((second, reach(second)))
    return targets


def time_to_target(device, kind="rpie64", long_iters=500, reps=5, check=True, scale=1.0):
    """Each algorithm's time to an LLK target on the scan `kind` (config 0's rPIE scan by
    default), the reference's time-to-target method on this GPU: the long runs (`long_iters`
    iterations, the Poisson LLK recorded after each) fix the targets (ttt_targets); then each
    algorithm runs the iterations it needs in one call on a fresh handle from the common start,
    `reps` times in ABBA order, with no LLK; device time from the engine's events and host wall
    time of the call (handle creation apart). At the headline target (the last: the one every
    algorithm reaches) the FP32 object is checked against the float64 oracle run for the same
    iterations from the same start (object NRMSE, global phase and phase ramp removed, scale
    kept, over the illuminated pixels)."""
    from ptyrs_b200 import GpuPtycho, Scan, sim
    s = sim.make_scan(kind, seed=0, scale=scale)
    scan = Scan(s["counts"], s["y"], s["x"], s["wavelength"], s["distance"], s["detector_pixel"])
    traces, long_ms = {}, {}
    for algo in TTT_ALGOS:
        with GpuPtycho(scan, s["object"], s["probe"], device=device) as g:
            ttt_call(g, algo, long_iters, calc_llk=1)
            traces[algo] = llk_after(algo, g.history()["poisson"])
            long_ms[algo] = g.last_call_ms()
    targets = ttt_targets(traces)
    target, iters = targets[-1]
    timed = {a: {"device_ms": [], "wall_ms": []} for a in TTT_ALGOS}
    objects = {}
    reached = tuple(a for a in TTT_ALGOS if iters[a] is not None)
    for rep in range(reps):
        for algo in (reached if rep % 2 == 0 else reached[::-1]):
            with GpuPtycho(scan, s["object"], s["probe"], device=device) as g:
                g.synchronize()
                t0 = time.perf_counter()
                ttt_call(g, algo, iters[algo])
                g.synchronize()
                timed[algo]["wall_ms"].append(1e3 * (time.perf_counter() - t0))
                timed[algo]["device_ms"].append(g.last_call_ms())
                if rep == 0:
                    objects[algo] = g.object()
    out = {"scan": kind, "scale": scale, "frames": len(s["counts"]),
           "long_iterations": long_iters, "reps": reps,
           "llk": "Poisson, normalised by the unmasked pixels",
           "long_final_llk": {a: float(t[-1]) for a, t in traces.items()},
           "diverged": [a for a, t in traces.items() if not np.isfinite(t[-1])],
           "long_llk_every_10": {a: [float(v) for v in t[9::10]] for a, t in traces.items()},
           "long_call_ms": long_ms,
           "targets": [{"llk": t, "iterations": c} for t, c in targets],
           "target_llk": target, "algorithms": TTT_LABELS, "per_algorithm": {}}
    for algo in TTT_ALGOS:
        if iters[algo] is None:
            out["per_algorithm"][algo] = {"iterations": None, "time_to_target_s": None}
            continue
        out["per_algorithm"][algo] = {
            "iterations": iters[algo],
            "time_to_target_s": statistics.median(timed[algo]["wall_ms"]) / 1e3,
            "device_s": statistics.median(timed[algo]["device_ms"]) / 1e3,
            "wall_ms_runs": [round(v, 3) for v in timed[algo]["wall_ms"]]}
    r = out["per_algorithm"]
    if r["rpie"]["time_to_target_s"]:
        out["rpie_over"] = {a: r["rpie"]["time_to_target_s"] / r[a]["time_to_target_s"]
                            for a in ("lsqml", "ml") if r[a]["time_to_target_s"]}
    if check:
        out["nrmse_vs_f64_at_target"] = ttt_precision(
            s, {a: n for a, n in iters.items() if n is not None}, objects)
    return out


def ttt_precision(s, iters, objects):
    """Object NRMSE of each algorithm's FP32 GPU object after its iterations to the target
    against the float64 oracle run of the same iterations from the same start."""
    from oracle import ops
    from oracle.lsqml import Lsqml
    from oracle.ptycho import Ptycho
    optics = oracle_optics(s)
    out = {}
    with _threads(os.cpu_count() or 1):
        for algo, n in iters.items():
            p = Ptycho(s["counts"], s["y"], s["x"], optics, s["object"], s["probe"])
            if algo == "rpie":
                p.rpie(n, batch_size=100, obj_alpha=0.1, probe_alpha=0.1, seed=7)
                ref = p.object
            elif algo == "lsqml":
                run = Lsqml(100, "poisson", 7)
                obj, probe = p.object, p.probe
                for _ in range(n):
                    obj, probe, _ = run.epoch(p.addr, p.obs, optics, obj, probe)
                ref = obj
            else:
                p.ml(n, update_object=True, update_probe=True, calc_llk=0,
                     zero_phase_ramp=False)
                ref = p.object
            illum = ops.illumination(p.addr.views, p.object.shape, p.probe)
            w = (illum >= 1e-3 * illum.max()).astype(float)
            out[algo] = object_nrmse(objects[algo], ref, w)
    from oracle import ops as _ops
    _ops.FFT_WORKERS = None
    return out


def line_config(args, wl, s, patterns, ws):
    """The `config` of both arms' lines (the same keys, so the two lines name one workload)."""
    counts = sum(x["counts"].nbytes for x in s) if isinstance(s, list) else s["counts"].nbytes
    out = {"workload": args.workload, "description": wl["desc"], "scale": args.scale,
           "patterns_per_step_per_gpu": patterns, "parallelism": f"replicas{ws}",
           "l2": f"inputs larger than L2 (counts {counts / 1e6:.0f} MB)"}
    if isinstance(s, list):
        out["scans"] = len(s)
        out["sides"] = {n: sum(1 for x in s if x["n"] == n) for n in (64, 96, 128, 192, 256)}
    return out


def reference_arm(args, wl):
    """The reference's CPU path for the same workload on the host cores (its numpy float64
    restatement, every host thread), a bounded sample per step: cycle algorithms one cycle over
    the scan's first m/2 and m frames with the full object, extrapolated to the whole scan by
    the fitted object-sized and per-frame costs (cycle_fit); batch algorithms one batch update
    of the run's own batch size."""
    rank, ws, _ = dist_env()
    if rank != 0:
        return
    full_wl = wl
    if wl["algorithm"] == "batch":
        # the batch's first scan (make_batch draws the scans in order), rPIE batch updates
        from ptyrs_b200 import sim
        scans = sim.make_batch(32, seed=0, scale=args.scale)
        s = scans[0]
        patterns = (wl["rpie_epochs"] + wl["lsqml_epochs"]) * sum(len(x["counts"]) for x in scans)
        wl = RPIE_OF_BATCH
    else:
        s = make_inputs(args.workload, 0, scale=args.scale)
        scans, patterns = s, len(s["counts"])
    threads = os.cpu_count() or 1
    a = b = 0.0
    frames, secs = 0, 0.0
    fits = []
    for step in range(args.warmup + args.steps):
        if wl["algorithm"] in CYCLES:
            _, fit, _ = cycle_fit(s, wl, threads, cycles=1)
            if step >= args.warmup:
                fits.append(fit)
        else:
            _, d, t, _ = cpu_batches(s, wl, 0.0, threads)
            if step >= args.warmup:
                frames += d
                secs += t
    if wl["algorithm"] in CYCLES:
        a = statistics.mean(f["object_s_per_cycle"] for f in fits)
        b = statistics.mean(f["frame_s"] for f in fits)
        P = len(s["counts"])
        value = P / (a + b * P)
        ms_step = 1e3 * sum(f["samples"][0][1] + f["samples"][1][1] for f in fits) / len(fits)
        sample = (f"{args.steps} steps of one {wl['algorithm'].upper()} cycle over the first "
                  f"{fits[0]['samples'][0][0]} and {fits[0]['samples'][1][0]} frames with the "
                  f"full object; a cycle over all {P} frames = {a:.2f} s object-sized work + "
                  f"{1e3 * b:.1f} ms per frame, extrapolated")
    else:
        value = frames / secs
        ms_step = 1e3 * secs / max(args.steps, 1)
        sample = (f"{args.steps} steps of one {wl['algorithm']} batch update of {wl['batch']} "
                  f"frames ({frames} pattern-iterations in {secs:.1f} s)")
    line = {
        "impl": "reference", "metric": "diffraction patterns*iter/sec", "value": value,
        "unit": "patterns*iter/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": line_config(args, full_wl, scans, patterns, ws),
        "cpu_baseline": {"value": value, "unit": "patterns*iter/s", "cores": threads,
                         "kind": "port", "sample": sample + f", numpy float64 on {threads} "
                                                            "threads"},
        "e2e": {"value": value, "unit": "patterns*iter/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


BATCH_RPIE = dict(batch_size=100, obj_alpha=0.1, probe_alpha=0.1, seed=7)
BATCH_LSQML = dict(batch_size=256, cost="poisson", seed=7)
RPIE_OF_BATCH = dict(kind="batch32", algorithm="rpie", batch=100)


def batch_main(args, wl):
    """The batched workload: every scan a handle, all run at once by `ptyb_batch_run`; the
    step's device time is the batch's, from the first launch to the last of any scan."""
    from ptyrs_b200 import GpuPtycho, Scan, batch_run, build, sim
    from ptyrs_b200.replicas import Replicas, job_value
    group = Replicas("nccl")
    rank, ws, local = group.rank, group.world, group.local
    import torch
    build.build()
    scans = sim.make_batch(32, seed=rank, scale=args.scale)
    P = sum(len(s["counts"]) for s in scans)
    scan_of = lambda s, counts=None: Scan(s["counts"] if counts is None else counts, s["y"],
                                          s["x"], s["wavelength"], s["distance"],
                                          s["detector_pixel"])
    # launch shapes per frame side by measurement, outside the timed region (ptyrs_b200.tune)
    opts = [dict() for _ in scans]
    tuned = None
    if not args.no_tune:
        from ptyrs_b200.tune import autotune_batch
        opts, chosen = autotune_batch(
            scans, run=lambda h: batch_run([h], 1, 1, rpie=BATCH_RPIE, lsqml=BATCH_LSQML),
            device=local, make=lambda s: (scan_of(s), s["object"], s["probe"]))
        tuned = {str(n): {"chosen": best, "candidates_ms": [
            {"cluster": o["cluster"], "stack": o["stack_size"],
             "ms": None if ms is None else round(ms, 3)} for ms, o in table]}
            for n, (best, table) in sorted(chosen.items())}
    handles = [GpuPtycho(scan_of(s), s["object"], s["probe"], device=local, **o)
               for s, o in zip(scans, opts)]
    re_, le_ = wl["rpie_epochs"], wl["lsqml_epochs"]
    step = lambda hs: batch_run(hs, re_, le_, rpie=BATCH_RPIE, lsqml=BATCH_LSQML)
    for _ in range(args.warmup):
        step(handles)
    group.barrier()
    launches0 = sum(h.launches() for h in handles)
    clocks = Clocks(local)
    ms = sum(step(handles) for _ in range(args.steps))
    clk = clocks.stop()
    group.barrier()
    launches = sum(h.launches() for h in handles) - launches0
    # one step again with per-kernel events, for the kernel table
    for h in handles:
        h.set_timing(True)
    step(handles)
    times, frames, bytes_ = {}, {}, {}
    for h, s in zip(handles, scans):
        kf = h.kernel_frames()
        for k, (kms, kn) in h.kernel_times().items():
            t = times.setdefault(k, [0.0, 0])
            t[0] += kms
            t[1] += kn
            per = algorithmic_bytes(k, s, RPIE_OF_BATCH) or algorithmic_bytes(
                k, s, dict(algorithm="lsqml"))
            if per and kf.get(k):
                bytes_[k] = bytes_.get(k, 0.0) + per * kf[k]
                frames[k] = frames.get(k, 0) + kf[k]
        h.set_timing(False)
    ms = group.max(ms)
    value = job_value((re_ + le_) * P, ws, args.steps, ms)
    pk, pk_kind = peaks()
    kname = max(times.items(), key=lambda kv: kv[1][0])[0]
    # The scans' kernels overlap in time (one stream each), so a kernel's event times do not
    # add up to wall time: the step's bandwidth is every kernel's algorithmic bytes over the
    # batch's device time.
    total = sum(bytes_.values())  # one step's
    achieved = total * args.steps / (ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": "whole step (every kernel of every scan)",
                "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / pk["hbm_gbs"], "peak_source": pk_kind, "traffic": None,
                "traffic_source": None, "bytes_per_step": total,
                "largest_kernel_by_event_time": kname,
                "kernels_counted": sorted(bytes_)}
    e2e = None
    if args.e2e_steps > 0:
        pinned = []
        for s in scans:
            t = torch.empty(s["counts"].shape, dtype=torch.float32, pin_memory=True)
            t.numpy()[...] = s["counts"]
            pinned.append(t)
        group.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            hs = [GpuPtycho(scan_of(s, c.numpy()), s["object"], s["probe"], device=local, **o)
                  for s, c, o in zip(scans, pinned, opts)]
            step(hs)
            for h in hs:
                h.object()
                h.probe()
                h.close()
        dt = group.max(time.perf_counter() - t0)
        h2d = sum(s["counts"].nbytes + 8 * s["object"].size + 8 * s["probe"].size
                  + 16 * len(s["counts"]) for s in scans)
        d2h = sum(8 * s["object"].size + 8 * s["probe"].size for s in scans)
        e2e = {"value": (re_ + le_) * P * ws * args.e2e_steps / dt, "unit": "patterns*iter/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "what": "per step: create every scan's handle from pinned host counts, 30 rPIE "
                       "then 30 LSQML epochs on all at once, every object and probe read back"}
    cpu, acc = None, None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cpu, _ = cpu_baseline(scans[0], RPIE_OF_BATCH, threads)
        cpu["sample"] += f" (rPIE batch updates of the first scan, side {scans[0]['n']})"
        one, _ = cpu_baseline(scans[0], RPIE_OF_BATCH, 1, seconds=5.0)
        cpu["single_core"] = {"value": one["value"], "cores": 1, "sample": one["sample"]}
        # every scan: one rPIE epoch over its first batch, FP32 GPU vs float64 oracle
        per_scan = [accuracy_batches(x, RPIE_OF_BATCH, local, nbatch=1)["object_nrmse_vs_f64"]
                    for x in scans]
        acc = {"object_nrmse_vs_f64_per_scan": per_scan, "max": max(per_scan),
               "sample": "per scan: one rPIE epoch (batches of 100) over its first 100 frames, "
                         "GPU FP32 vs the float64 oracle from the same start"}
    for h in handles:
        h.close()
    if rank == 0:
        print(json.dumps({
            "metric": "diffraction patterns*iter/sec", "value": value,
            "unit": "patterns*iter/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": line_config(args, wl, scans, (re_ + le_) * P, ws),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "accuracy": acc,
            "gpu_launches": int(launches), "clocks": clk, "autotune": tuned,
            "kernels_ms": {k: round(v[0], 3) for k, v in sorted(times.items())},
        }), flush=True)
    group.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ml256", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cluster", type=int, default=0,
                    help="CTAs per frame of the frame kernel (0: the engine chooses)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the launch-shape autotuner (cluster and stack from the flags)")
    ap.add_argument("--stack", type=int, default=0,
                    help="frames per launch of the whole-scan passes (0: the engine's default)")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="keep this fraction of the scan's positions (small profiling cases)")
    ap.add_argument("--no-ttt", action="store_true", help="skip the time-to-target leg")
    ap.add_argument("--ttt-scan", default="rpie64",
                    help="scan of the time-to-target leg (rpie64: the rPIE configuration)")
    ap.add_argument("--ttt-iters", type=int, default=500,
                    help="iterations of the time-to-target leg's long runs")
    ap.add_argument("--ttt-scale", type=float, default=1.0,
                    help="fraction of the time-to-target scan's positions (a cut)")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return reference_arm(args, wl)
    if wl["algorithm"] == "batch":
        return batch_main(args, wl)

    from ptyrs_b200.replicas import Replicas, job_value
    group = Replicas("nccl")
    rank, ws, local = group.rank, group.world, group.local
    import torch

    from ptyrs_b200 import GpuPtycho, Scan, build, sim
    build.build()
    s = make_inputs(args.workload, seed=rank, scale=args.scale)
    P = len(s["counts"])
    scan = Scan(s["counts"], s["y"], s["x"], s["wavelength"], s["distance"], s["detector_pixel"])
    tuned = None
    if not args.no_tune and not args.cluster and not args.stack:
        # launch shapes by measurement, outside the timed region (ptyrs_b200.tune)
        from ptyrs_b200.tune import autotune
        best, table = autotune(scan, s["object"], s["probe"],
                               run=lambda h: run_algorithm(h, wl, 1),
                               prepare=lambda h: prepare(h, s, wl), device=local,
                               gaps=s.get("gaps"))
        args.cluster, args.stack = best["cluster"], best["stack_size"]
        tuned = {"chosen": best, "candidates_ms": [
            {"cluster": o["cluster"], "stack": o["stack_size"],
             "ms": None if ms is None else round(ms, 3)} for ms, o in table]}
    g = GpuPtycho(scan, s["object"], s["probe"], device=local, cluster=args.cluster,
                  stack_size=args.stack, gaps=s.get("gaps"))
    prepare(g, s, wl)
    run_algorithm(g, wl, args.warmup)
    g.synchronize()

    barrier = group.barrier

    # Timed region: K epochs, device time from events on the engine's stream around the call.
    barrier()
    g.synchronize()
    launches0 = g.launches()
    clocks = Clocks(local)
    run_algorithm(g, wl, args.steps)
    g.synchronize()
    clk = clocks.stop()
    barrier()
    ms = g.last_call_ms()
    launches = g.launches() - launches0
    # The same K steps again with every launch between events of its own, for the per-kernel
    # times (the events cost launch slots, so the value above is taken without them).
    g.set_timing(True)
    run_algorithm(g, wl, args.steps)
    g.synchronize()
    times = g.kernel_times()
    kframes = g.kernel_frames()
    instrumented_ms = g.last_call_ms()
    g.set_timing(False)
    ms = group.max(ms)
    value = job_value(P, ws, args.steps, ms)

    # Dominant kernel and its roofline (algorithmic bytes per launch / mean launch time).
    pk, pk_kind = peaks()
    # the top kernel kind with a per-frame byte count (the "misc" kind has none)
    typed = {k: v for k, v in times.items() if algorithmic_bytes(k, s, wl) and kframes.get(k)}
    top = max((typed or times).items(), key=lambda kv: kv[1][0])
    kname, (kms, kn) = top
    per_frame = algorithmic_bytes(kname, s, wl)
    roofline = None
    if per_frame and kframes.get(kname):
        frames_launch = kframes[kname] / kn
        bytes_launch = per_frame * frames_launch
        achieved = bytes_launch / (kms / kn / 1e3) / 1e9
        measured = NCU_DRAM_BYTES_PER_FRAME.get(args.workload, {}).get(kname)
        traffic = measured * frames_launch if measured and args.scale == 1.0 else None
        roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved,
                    "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                    "peak_source": pk_kind, "traffic": traffic,
                    "traffic_source": None if traffic is None else
                    "ncu DRAM bytes per frame on a cut of the same scan "
                    f"({NCU_PROFILE[args.workload]}) times this launch's frames",
                    "bytes_per_launch": bytes_launch, "mean_launch_ms": kms / kn,
                    "share": kms / sum(v[0] for v in times.values())}
        flops = fft_flops(kname, s)
        if flops:
            tf = flops * frames_launch / (kms / kn / 1e3) / 1e12
            roofline["secondary"] = {
                "bound": "fp32", "achieved": tf, "peak": FP32_NOMINAL_TFLOPS,
                "unit": "TFLOP/s", "frac": tf / FP32_NOMINAL_TFLOPS,
                "peak_source": "nominal (148 SMs x 128 FP32 lanes x 2 x 1.965 GHz)",
                "what": "the kernel's FFT flops, 5 N^2 log2(N^2) per plane and transform"}

    # End to end through the public API from pinned host buffers: per step, a fresh state
    # (counts, positions, object and probe uploaded), one epoch, the object and probe read back.
    e2e = None
    if args.e2e_steps > 0:
        pinned = torch.empty(s["counts"].shape, dtype=torch.float32, pin_memory=True)
        pinned.numpy()[...] = s["counts"]
        escan = Scan(pinned.numpy(), s["y"], s["x"], s["wavelength"], s["distance"],
                     s["detector_pixel"])
        ekw = dict(device=local, cluster=args.cluster, stack_size=args.stack, gaps=s.get("gaps"))
        with GpuPtycho(escan, s["object"], s["probe"], **ekw) as w:  # warm-up
            prepare(w, s, wl)
            run_algorithm(w, wl, 1)
            w.object()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            with GpuPtycho(escan, s["object"], s["probe"], **ekw) as w:
                prepare(w, s, wl)
                run_algorithm(w, wl, 1)
                w.objects()
                w.probe()
                if wl["algorithm"] == "ml":
                    w.positions()
        dt = time.perf_counter() - t0
        dt = group.max(dt)
        n = s["n"]
        # counts (f32), object and probe (complex64 on the device), positions (y, x and the
        # ML offsets in f64)
        pos_bytes = 16 * P + (16 * P if wl["algorithm"] == "ml" else 0)
        h2d = s["counts"].nbytes + 8 * s["object"].size + 8 * s["probe"].size + pos_bytes
        if wl.get("opr"):
            # the OPR start: eigenmodes (complex128), weights and main-mode weights (f64)
            h2d += 16 * wl["opr"] * n * n + 8 * P * wl["opr"] + 8 * P
        d2h = (8 * s["object"].size + 8 * s["probe"].size
               + (16 * P if wl["algorithm"] == "ml" else 0))
        e2e = {"value": P * ws * args.e2e_steps / dt, "unit": "patterns*iter/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "what": "per step: create from pinned host counts (and the start offsets), one "
                       "epoch or cycle, the object, probe (and offsets) read back"}

    cpu, acc = None, None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cpu, state = cpu_baseline(s, wl, threads)
        if wl["algorithm"] in CYCLES:
            acc = accuracy(s, wl, state, local)
        else:
            acc = accuracy_batches(s, wl, local)
        # the like-for-like figure of a single-threaded CPU engine
        if wl["algorithm"] in CYCLES:
            v1, fit1, _ = cycle_fit(s, wl, 1, cycles=1)
            one = {"value": v1, "cores": 1, "fit": fit1,
                   "sample": "as above, one cycle per sample, numpy float64 on 1 thread"}
        else:
            o, _ = cpu_baseline(s, wl, 1, seconds=8.0)
            one = {"value": o["value"], "cores": 1, "sample": o["sample"]}
        cpu["single_core"] = one
    g.close()
    ttt = None
    if rank == 0 and not args.no_ttt:
        ttt = time_to_target(local, kind=args.ttt_scan, long_iters=args.ttt_iters,
                             check=not args.no_cpu, scale=args.ttt_scale)
    if rank == 0:
        line = {
            "metric": "diffraction patterns*iter/sec", "value": value,
            "unit": "patterns*iter/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": line_config(args, wl, s, P, ws),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "accuracy": acc,
            "time_to_target": ttt,
            "gpu_launches": int(launches), "clocks": clk, "autotune": tuned,
            "ms_per_step_with_kernel_events": instrumented_ms / args.steps,
            "kernels_ms": {k: round(v[0], 3) for k, v in sorted(times.items())},
        }
        print(json.dumps(line), flush=True)
    group.close()


if __name__ == "__main__":
    main()
