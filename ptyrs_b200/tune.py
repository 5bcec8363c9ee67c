"""The engine's launch shapes picked by measurement: for a scan, each candidate of the cluster
size (the CTAs that share one frame's FFT tiles, so the rows each CTA transforms) and the stack
(frames per launch of the whole-scan passes) runs one warm-up and one timed call of the
algorithm on its own handle, timed on the device; the fastest wins. Candidates the device cannot
launch (a cluster too large for its shared memory) are skipped.
"""
import itertools

from .engine import GpuPtycho, PtybError


def clusters_for(n):
    """The cluster sizes the engine has kernels for at frame side `n` (0 lets it choose)."""
    return {64: [1], 96: [2], 128: [2, 4], 192: [8], 256: [16, 8]}.get(n, [0])


def autotune(scan, obj, probe, run, prepare=None, stacks=None, clusters=None, device=0, **kw):
    """`(best, table)`: `best` the `dict(cluster=..., stack_size=...)` of the fastest timed call
    of `run(handle)` (its device time: the float `run` returns, else the handle's last call's)
    and `table` every candidate's `(ms, options)` (None if it failed);
    `prepare(handle)` sets each fresh handle up (positions and the like) before the warm-up.
    The default stacks run 512, 1024 and 4096 frames per launch and the whole scan in one."""
    n = probe.shape[-1]
    clusters = clusters_for(n) if clusters is None else clusters
    if stacks is None:
        nframe = scan.counts.shape[0]
        stacks = sorted({min(st, nframe) for st in (512, 1024, 4096, nframe)})
    table = []
    for c, st in itertools.product(clusters, stacks):
        opts = dict(cluster=c, stack_size=st)
        try:
            with GpuPtycho(scan, obj, probe, device=device, **opts, **kw) as g:
                if prepare is not None:
                    prepare(g)
                run(g)
                g.synchronize()
                ms = run(g)
                g.synchronize()
                table.append((ms if isinstance(ms, float) else g.last_call_ms(), opts))
        except PtybError:
            table.append((None, opts))
    timed = [t for t in table if t[0] is not None]
    if not timed:
        raise RuntimeError("no candidate launch shape ran")
    return min(timed, key=lambda t: t[0])[1], table


def autotune_batch(scans, run, device=0, stacks=(256, 512, 1024), make=None):
    """Launch shapes for many uneven scans: per frame side, `autotune` on the side's first scan
    (the shapes depend on the side and the frame count per launch, not on the object), applied
    to every scan of that side. `scans` are dicts with `n` (the side) and what `make(scan)`
    turns into `(Scan, object, probe)`; returns `(options per scan, {side: (best, table)})`."""
    chosen = {}
    for s in scans:
        if s["n"] in chosen:
            continue
        scan, obj, probe = make(s)
        chosen[s["n"]] = autotune(scan, obj, probe, run=run, stacks=stacks, device=device)
    return [chosen[s["n"]][0] for s in scans], chosen
