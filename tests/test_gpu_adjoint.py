"""The hand-written adjoint through the C ABI (`ptyb_gradients`) and the torch autograd function
on it, against the float64 oracle, whose object and probe gradients match central differences
(test_oracle_positions.py) and whose position gradient matches the reference's golden one
(test_oracle_farfield.py); and, as the ML configuration's gradient check does, against
central differences at h = 1e-3 along 64 random entries of each array, taken of the float64
Poisson sum (the engine's FP32 sum rounds at ~1e-7 of the loss, a few per cent of such a
difference)."""
import numpy as np
import pytest
import torch

from oracle import ops
from ptyrs_b200 import GpuPtycho, PtybError, Scan, sim
from ptyrs_b200.autograd import poisson_loss
from scenarios import far_field, oracle_state, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4
# The FP32 gradient against float64 central differences: their truncation at h = 1e-3 and the
# gradient's own 1e-4.
FD_TOL = 1e-3

SHAPES = [(64, 2, 40, 192), (128, 3, 24, 320), (256, 2, 10, 448)]


@pytest.fixture(scope="module", params=SHAPES, ids=lambda p: f"n{p[0]}k{p[1]}")
def case(request):
    n, k, nframe, side = request.param
    s = far_field(n, k, nframe, side, masked=True, seed=n + k)
    s["object"] = s["truth"] * 0.9 * np.exp(0.1j)
    s["offsets"] = np.random.default_rng(9).uniform(-0.6, 0.6, (nframe, 2))
    return s


def gpu_of(s):
    scan = Scan(s["counts"], s["y"], s["x"], sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL)
    return GpuPtycho(scan, s["object"], s["probe"])


def oracle_loss(cpu):
    psi = cpu.optics.exit_forward(cpu.calc_psi())
    return ops.llk(cpu.obs, slice(0, cpu.addr.nframe), cpu.addr.nmode, psi).poisson


@pytest.mark.parametrize("moved", [False, True])
def test_gradients_match_oracle(case, moved):
    cpu = oracle_state(case)
    if moved:
        cpu.set_positions(case["offsets"])
    go, gp = cpu.grads()
    with gpu_of(case) as g:
        if moved:
            g.set_positions(case["offsets"], refine=False)
        got = g.gradients(positions=moved)
        assert abs(got["loss"] - oracle_loss(cpu)) <= TOL * abs(oracle_loss(cpu))
        assert rel_l2(got["object"], go) < TOL
        assert rel_l2(got["probe"], gp) < TOL
        if moved:
            want = cpu.position_grad("poisson")
            assert rel_l2(got["positions"], want) < 10 * TOL
        # the state is not changed
        assert np.array_equal(g.object(), case["object"].astype(np.complex64).astype(complex))


def test_gradients_match_directional_differences(case):
    rng = np.random.default_rng(11)
    h = 1e-3
    with gpu_of(case) as g:
        g.set_positions(case["offsets"], refine=False)
        got = g.gradients()
    cpu = oracle_state(case)

    def loss(obj, probe, d):
        cpu.object, cpu.probe = obj, probe
        cpu.set_positions(d)
        return oracle_loss(cpu)

    base = (case["object"].copy(), case["probe"].copy(), case["offsets"].copy())
    for which, grad in ((0, got["object"]), (1, got["probe"]), (2, got["positions"])):
        x = base[which]
        v = np.zeros_like(x)
        flat = v.reshape(-1)
        k = min(64, flat.size)  # every offset of a scan of fewer than 32 frames
        idx = rng.choice(flat.size, k, replace=False)
        scale = np.abs(x).max()
        if np.iscomplexobj(x):
            flat[idx] = scale * (rng.normal(size=k) + 1j * rng.normal(size=k))
            an = float(np.sum(grad.real * v.real + grad.imag * v.imag))
        else:
            flat[idx] = rng.normal(size=k)
            an = float(np.sum(grad * v))
        args_p = list(base)
        args_m = list(base)
        args_p[which] = x + h * v
        args_m[which] = x - h * v
        fd = (loss(*args_p) - loss(*args_m)) / (2 * h)
        assert abs(fd - an) <= FD_TOL * abs(an), (which, fd, an)


def test_autograd_function(case):
    with gpu_of(case) as g:
        g.set_positions(case["offsets"], refine=False)
        want = g.gradients()
        obj = torch.tensor(case["object"], requires_grad=True)
        probe = torch.tensor(case["probe"], requires_grad=True)
        d = torch.tensor(case["offsets"], requires_grad=True)
        loss = poisson_loss(obj, probe, d, g)
        assert abs(loss.item() - want["loss"]) <= 1e-12 * abs(want["loss"])
        loss.backward()
        assert np.allclose(obj.grad.numpy(), want["object"], rtol=0, atol=0)
        assert np.allclose(probe.grad.numpy(), want["probe"], rtol=0, atol=0)
        assert np.allclose(d.grad.numpy(), want["positions"], rtol=0, atol=0)
        # a small step against the gradient lowers the loss
        with torch.no_grad():
            t = 1e-3 * obj.abs().max() / obj.grad.abs().max()
            obj2 = obj - t * obj.grad
        assert poisson_loss(obj2, probe, d, g).item() < loss.item()


def test_autograd_function_on_cuda_tensors(case):
    """CUDA tensors stay on the device (`ptyb_set_object_device`, `ptyb_set_probe_device`,
    `ptyb_gradients_device`): the same loss and, in complex64, the same gradients as the host
    path's, on CUDA tensors; a host pointer is refused and changes nothing."""
    dev = torch.device("cuda:0")
    with gpu_of(case) as g:
        g.set_positions(case["offsets"], refine=False)
        want = g.gradients()
        obj = torch.tensor(case["object"], dtype=torch.complex64, device=dev, requires_grad=True)
        probe = torch.tensor(case["probe"], dtype=torch.complex64, device=dev, requires_grad=True)
        d = torch.tensor(case["offsets"], device=dev, requires_grad=True)
        loss = poisson_loss(obj, probe, d, g)
        assert loss.device.type == "cuda"
        # the state went in as complex64 either way, so the loss and gradients are the same
        assert abs(loss.item() - want["loss"]) <= 1e-12 * abs(want["loss"])
        loss.backward()
        assert obj.grad.is_cuda and probe.grad.is_cuda
        go, gp = obj.grad.cpu().numpy(), probe.grad.cpu().numpy()
        assert np.abs(go - want["object"]).max() <= 1e-6 * np.abs(want["object"]).max()
        assert np.abs(gp - want["probe"]).max() <= 1e-6 * np.abs(want["probe"]).max()
        assert np.allclose(d.grad.cpu().numpy(), want["positions"], rtol=0, atol=0)
        before = g.object()
        host = np.ascontiguousarray(case["object"], np.complex64)
        with pytest.raises(PtybError):
            g.set_object_device(host.ctypes.data, *host.shape)
        with pytest.raises(PtybError):
            g.set_object_device(obj.detach().data_ptr(), 1, 1, 1)  # wrong dims
        assert np.array_equal(g.object(), before)
