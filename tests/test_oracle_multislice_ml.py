"""The multislice ML oracle (oracle.lsqml.slice_jet, multislice_ml): its line search's
first-order and second-order coefficients against central differences of the Poisson LLK
along the direction through three slices, its one-slice case against PyNX's `cg_gamma`, and
its cycles lowering the LLK."""
import numpy as np

from oracle import ops
from oracle.lsqml import SliceWaves, multislice_grads, multislice_ml, slice_jet
from oracle.ptycho import Ptycho
from ptyrs_b200 import sim
from scenarios import far_field, oracle_state
from test_gpu_multislice import multislice_scan, oracle_of


def poisson_sum(cpu, objs, probe):
    views = cpu.addr.views
    w = SliceWaves(cpu.optics, views, objs, probe[views["probe"].astype(np.int64)])
    psi = cpu.optics.exit_forward(w.psi)
    return ops.llk(cpu.obs, slice(0, cpu.addr.nframe), cpu.addr.nmode, psi).poisson


def test_line_search_terms_match_central_differences():
    s = multislice_scan(64, 2, 12, 160, (2e-6, 3e-6), seed=4)
    cpu = oracle_of(s)
    rng = np.random.default_rng(6)
    objs = [o * (1 + 0.05 * rng.normal(size=o.shape)) * np.exp(0.05j) for o in s["objects"]]
    probe = cpu.probe
    _, go, gp = multislice_grads(cpu.addr, cpu.obs, cpu.optics, objs, probe)
    d_objs, d_probe = [-g for g in go], -gp
    po, a, b = slice_jet(cpu.optics, cpu.addr.views, objs, probe, d_objs, d_probe)
    num, den = ops.cg_poisson_gamma(cpu.obs, slice(0, cpu.addr.nframe), cpu.addr.nmode, po, a,
                                    b)
    scale = max(np.abs(o).max() for o in objs) / max(np.abs(d).max() for d in d_objs)
    h = 1e-4 * scale
    at = lambda t: poisson_sum(cpu, [o + t * d for o, d in zip(objs, d_objs)],
                               probe + t * d_probe)
    f0, fp, fm = at(0.0), at(h), at(-h)
    assert abs((fp - fm) / (2 * h) + num) <= 1e-5 * abs(num)
    assert abs((fp - 2 * f0 + fm) / h ** 2 - den) <= 1e-3 * abs(den)


def test_one_slice_is_pynx_cg_gamma():
    s = far_field(64, 2, 20, 192, seed=5)
    cpu = oracle_state(s)
    rng = np.random.default_rng(8)
    d_obj = 0.01 * (rng.normal(size=cpu.object.shape) + 1j * rng.normal(size=cpu.object.shape))
    d_probe = 0.01 * np.abs(cpu.probe).max() * rng.normal(size=cpu.probe.shape)
    want = cpu.cg_gamma(d_obj, d_probe)
    po, a, b = slice_jet(cpu.optics, cpu.addr.views, [cpu.object], cpu.probe, [d_obj], d_probe)
    got = ops.cg_poisson_gamma(cpu.obs, slice(0, cpu.addr.nframe), cpu.addr.nmode, po, a, b)
    assert np.allclose(got, want, rtol=1e-12, atol=0)


def test_cycles_lower_the_llk():
    s = multislice_scan(64, 2, 16, 160, (2e-6, 3e-6), seed=2)
    cpu = oracle_of(s)
    _, _, recs = multislice_ml(cpu.addr, cpu.obs, cpu.optics, s["objects"], cpu.probe, 6,
                               calc_llk=1)
    p = [r.poisson for r in recs]
    assert all(b < a for a, b in zip(p, p[1:]))
