"""Parity at the benchmark configurations' full size: the FP32 CUDA path against the float64
oracle over whole scans, at checkpoints of one run (test infrastructure, not the product).

    python tests/at_size.py oracle CONFIG DIR   # host only: the oracle's run and checkpoints
    python tests/at_size.py meta CONFIG DIR     # host only: the inputs' digest and the mask alone
    python tests/at_size.py gpu CONFIG DIR OUT  # the CUDA path from the same inputs, compared
    python tests/at_size.py sensitivity CONFIG DIR OUT [EPS]  # the oracle from a start
                                                # perturbed by EPS (1e-7), compared the same way

CONFIG is one of CONFIGS: rpie64 (400 frames of 64², rPIE with α = β = 0.1 in batches of 100),
lsqml128 (4096 frames of 128² × 3 modes, Poisson LSQML in batches of 256) and ml256 (the first
2500 of the 10000 frames of 256² × 2 modes with the whole 2048² object, Poisson ML conjugate
gradient refining the positions: the float64 oracle holds every view's exit wave at once, about
21 GB per array for all 10000 frames, more host memory than a run here has) and msml128 (6000
frames of 128² × 2 modes through three 1536² slices, Poisson ML through the slices; the oracle
runs one call of k cycles per checkpoint, since the opening rescale and the conjugate
directions belong to a call). The inputs
are the benchmark's seeded scans (`sim.make_scan`; ml256's counts made with torch on the host,
so both phases read the same counts, checked by a digest). The oracle phase runs one call of
the longest run and keeps a snapshot after each checkpoint's iteration; the GPU phase runs
each checkpoint as one call of that many iterations on a fresh state (the calls are the
reference's: a k-iteration call is the first k iterations of a longer one) and writes, for
each checkpoint the oracle's run has reached, the object's and probe's relative L2 error against the oracle's, the object NRMSE
with the global phase and a phase ramp removed (scale kept) over the illuminated pixels, and
for ml256 the largest difference of the refined offsets. The sensitivity phase measures how far
the float64 run itself moves when its start object is multiplied by (1 + EPS·ξ), ξ seeded
complex normal: the scale of difference that rounding alone leaves after k iterations.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

CONFIGS = {
    "rpie64": dict(kind="rpie64", algorithm="rpie", batch=100, checkpoints=[1, 2, 5, 10, 20, 50]),
    "lsqml128": dict(kind="lsqml128", algorithm="lsqml", batch=256,
                     checkpoints=[1, 2, 5, 10, 20, 50, 100]),
    "ml256": dict(kind="ml256", algorithm="ml", checkpoints=[1, 2], scale=0.25),
    "msml128": dict(kind="ms128", algorithm="ml_slices", checkpoints=[1, 2]),
}


def inputs(cfg):
    from ptyrs_b200 import sim
    s = sim.make_scan(cfg["kind"], seed=0, scale=cfg.get("scale", 1.0), device="cpu")
    digest = hashlib.sha256(np.ascontiguousarray(s["counts"]).tobytes()).hexdigest()
    return s, digest


def optics_of(s):
    """The far field of the scan's geometry, through its slices when it has gaps."""
    from oracle import ops
    optics = ops.Optics.far_field(s["wavelength"], s["distance"], s["detector_pixel"],
                                  [s["n"], s["n"]])
    if s.get("gaps"):
        optics = optics.with_slices([ops.Wavefield([s["n"], s["n"]], s["wavelength"],
                                                   optics.pixel, z) for z in s["gaps"]])
    return optics


def write_meta(name, out, s, digest, mask, times):
    os.makedirs(out, exist_ok=True)
    np.savez(os.path.join(out, f"{name}_mask.npz"), mask=np.packbits(mask), shape=mask.shape)
    with open(os.path.join(out, f"{name}_meta.json"), "w") as f:
        json.dump({"config": name, "digest": digest, "seconds": times,
                   "threads": os.cpu_count()}, f)


def run_meta(name, out):
    """The digest and the illuminated-pixel mask of a configuration's inputs, without the run."""
    from oracle import ops
    from oracle.ptycho import Ptycho
    s, digest = inputs(CONFIGS[name])
    p = Ptycho(s["counts"], s["y"], s["x"], optics_of(s), s["object"][:1], s["probe"])
    illum = ops.illumination(p.addr.views, p.object.shape, p.probe)
    write_meta(name, out, s, digest, illum >= 1e-3 * illum.max(), {})


def run_oracle(name, out, eps=0.0, save_as=None):
    """The oracle's run of the longest checkpoint, a snapshot at each checkpoint (`save_as(k,
    obj, probe, offsets)` instead of the files when given); the start object perturbed by
    `eps` when it is not 0."""
    from oracle import ops
    from oracle.lsqml import Lsqml
    from oracle.ptycho import Ptycho
    cfg = CONFIGS[name]
    os.makedirs(out, exist_ok=True)
    ops.FFT_WORKERS = os.cpu_count()  # the oracle's transforms on every host core
    t0 = time.perf_counter()
    s, digest = inputs(cfg)
    optics = optics_of(s)
    start = s["object"]
    if eps:
        rng = np.random.default_rng(11)
        xi = (rng.standard_normal(start.shape) + 1j * rng.standard_normal(start.shape)) / np.sqrt(2)
        start = start * (1.0 + eps * xi)
    p = Ptycho(s["counts"], s["y"], s["x"], optics, start[:1], s["probe"])
    illum = ops.illumination(p.addr.views, p.object.shape, p.probe)
    mask = illum >= 1e-3 * illum.max()
    last = max(cfg["checkpoints"])
    times = {}
    if save_as is None:
        write_meta(name, out, s, digest, mask, times)

    def save(k, obj, probe, offsets=None):
        times[k] = time.perf_counter() - t0
        if save_as is not None:
            save_as(k, obj, probe, offsets)
            return
        np.savez(os.path.join(out, f"{name}_{k}.npz"), object=obj.astype(np.complex64),
                 probe=probe, offsets=np.zeros(0) if offsets is None else offsets)
        write_meta(name, out, s, digest, mask, times)
        print(f"{name}: checkpoint {k} at {times[k]:.0f} s", flush=True)

    if cfg["algorithm"] == "rpie":
        for k in range(1, last + 1):
            p.rpie(1, batch_size=cfg["batch"], obj_alpha=0.1, probe_alpha=0.1, seed=7)
            if k in cfg["checkpoints"]:
                save(k, p.object, p.probe)
    elif cfg["algorithm"] == "ml_slices":
        # ML through the slices (one call of k cycles per checkpoint: the opening rescale and
        # the conjugate directions are a call's)
        from oracle.lsqml import multislice_ml
        slices = [start[k:k + 1] for k in range(start.shape[0])]
        for k in cfg["checkpoints"]:
            objs, probe, _ = multislice_ml(p.addr, p.obs, optics, slices, p.probe, k)
            save(k, np.concatenate(objs), probe)
    elif cfg["algorithm"] == "lsqml":
        run = Lsqml(cfg["batch"], "poisson", 7)
        obj, probe = p.object, p.probe
        for k in range(1, last + 1):
            obj, probe, _ = run.epoch(p.addr, p.obs, optics, obj, probe)
            if k in cfg["checkpoints"]:
                save(k, obj, probe)
    else:
        p.set_positions(np.zeros((p.addr.nframe, 2)), refine=True)

        def after(ic):
            if ic + 1 in cfg["checkpoints"]:
                save(ic + 1, p.object, p.probe, p.offsets.copy())

        p.ml(last, update_object=True, update_probe=True, calc_llk=0, zero_phase_ramp=False,
             after_cycle=after)


def compare(name, ref, k, obj, probe, offsets):
    """One checkpoint's row against the oracle's snapshot in `ref`."""
    from ptyrs_b200.metrics import object_nrmse
    m = np.load(os.path.join(ref, f"{name}_mask.npz"))
    mask = np.unpackbits(m["mask"])[:int(np.prod(m["shape"]))].reshape(m["shape"])
    mask = mask.reshape(mask.shape[-2:]).astype(bool)  # one object mode (or every slice)
    r = np.load(os.path.join(ref, f"{name}_{k}.npz"))
    ro, rp = r["object"].astype(np.complex128), r["probe"]
    full = np.broadcast_to(mask, obj.shape)
    row = {"iterations": k,
           "object_rel_l2": float(np.linalg.norm(obj - ro) / np.linalg.norm(ro)),
           "object_rel_l2_illuminated": float(np.linalg.norm((obj - ro)[full])
                                              / np.linalg.norm(ro[full])),
           "probe_rel_l2": float(np.linalg.norm(probe - rp) / np.linalg.norm(rp)),
           "object_nrmse": object_nrmse(obj, ro, full.astype(float))}
    if offsets is not None and len(r["offsets"]):
        row["offsets_max_abs_diff_px"] = float(np.abs(offsets - r["offsets"]).max())
    print(json.dumps(row), flush=True)
    return row


def report(name, ref, out, rows, **extra):
    cfg = CONFIGS[name]
    meta = json.load(open(os.path.join(ref, f"{name}_meta.json")))
    with open(out, "w") as f:
        json.dump({"config": name, "kind": cfg["kind"], "oracle_seconds": meta["seconds"],
                   "oracle_threads": meta["threads"], "rows": rows, **extra}, f, indent=1)


def run_gpu(name, ref, out):
    """Each checkpoint on the CUDA path, compared with the oracle's snapshot."""
    from ptyrs_b200 import GpuPtycho, Scan
    cfg = CONFIGS[name]
    meta = json.load(open(os.path.join(ref, f"{name}_meta.json")))
    s, digest = inputs(cfg)
    if digest != meta["digest"]:
        raise RuntimeError("the inputs differ from the oracle run's")
    scan = Scan(s["counts"], s["y"], s["x"], s["wavelength"], s["distance"], s["detector_pixel"])
    rows = []
    reached = [k for k in cfg["checkpoints"] if os.path.exists(os.path.join(ref, f"{name}_{k}.npz"))]
    for k in reached:
        with GpuPtycho(scan, s["object"], s["probe"], gaps=s.get("gaps")) as g:
            if cfg["algorithm"] == "rpie":
                g.rpie(k, batch_size=cfg["batch"], obj_alpha=0.1, probe_alpha=0.1, seed=7)
            elif cfg["algorithm"] == "lsqml":
                g.lsqml(k, batch_size=cfg["batch"], cost="poisson", seed=7)
            elif cfg["algorithm"] == "ml_slices":
                g.ml(k, update_object=True, update_probe=True, calc_llk=0,
                     zero_phase_ramp=False)
            else:
                g.set_positions(np.zeros((len(s["counts"]), 2)), refine=True)
                g.ml(k, update_object=True, update_probe=True, calc_llk=0,
                     zero_phase_ramp=False)
            obj = g.objects() if s.get("gaps") else g.object()
            probe = g.probe()
            d = g.positions() if cfg["algorithm"] == "ml" else None
        rows.append(compare(name, ref, k, obj, probe, d))
    report(name, ref, out, rows, path="CUDA FP32")


def run_sensitivity(name, ref, out, eps):
    """The float64 oracle from the perturbed start, compared with its own unperturbed run."""
    rows = []
    path = f"float64 oracle, start perturbed by {eps:g}"

    def save_as(k, o, p, d):
        rows.append(compare(name, ref, k, o, p, d))
        report(name, ref, out, rows, path=path)  # kept current, so a run cut short still reports

    run_oracle(name, ref, eps=eps, save_as=save_as)


if __name__ == "__main__":
    if (len(sys.argv) < 4 or sys.argv[1] not in ("oracle", "meta", "gpu", "sensitivity")
            or sys.argv[2] not in CONFIGS):
        raise SystemExit(__doc__)
    if sys.argv[1] == "oracle":
        run_oracle(sys.argv[2], sys.argv[3])
    elif sys.argv[1] == "meta":
        run_meta(sys.argv[2], sys.argv[3])
    elif sys.argv[1] == "gpu":
        run_gpu(sys.argv[2], sys.argv[3], sys.argv[4])
    else:
        run_sensitivity(sys.argv[2], sys.argv[3], sys.argv[4],
                        float(sys.argv[5]) if len(sys.argv) > 5 else 1e-7)
