"""The opr128 workload's seeded OPR start (`sim.opr_start`, bench.py's `prepare` and
`oracle_variation`): the shapes, the same start on every call, the eigenmodes at the main
mode's scale, and the same variation for the GPU arm and the oracle arm."""
import numpy as np

from ptyrs_b200 import sim


def probe(n=32, k=3, seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(k, n, n)) + 1j * rng.normal(size=(k, n, n))


def test_opr_start_shapes_and_determinism():
    p = probe()
    u, w, c = sim.opr_start(p, 50, 2)
    assert u.shape == (2, 32, 32) and w.shape == (50, 2) and c.shape == (50,)
    assert np.all(c == 1.0) and np.abs(w).max() <= 0.1
    u2, w2, c2 = sim.opr_start(p, 50, 2)
    assert np.array_equal(u, u2) and np.array_equal(w, w2) and np.array_equal(c, c2)
    scale = np.sqrt((np.abs(p[0]) ** 2).mean())
    for ui in u:
        assert abs(np.sqrt((np.abs(ui) ** 2).mean()) - scale) <= 1e-12 * scale


def test_bench_arms_get_the_same_variation():
    import bench
    wl = bench.WORKLOADS["opr128"]
    assert wl["kind"] == "lsqml128" and wl["opr"] == 2
    s = dict(probe=probe(), counts=np.zeros((40, 32, 32), np.float32))
    var = bench.oracle_variation(s, wl)
    u, w, c = bench.opr_start(s, wl)
    assert np.array_equal(var.eigenmodes, u)
    assert np.array_equal(var.weights, w.ravel())
    assert np.array_equal(var.intensity, c)
    assert bench.oracle_variation(s, bench.WORKLOADS["lsqml128"]) is None
    n2, K = 32 * 32, 3
    assert bench.algorithmic_bytes("opr_step", s | {"n": 32}, wl) == 16 * n2 + 8 * K * n2
