"""The far-field Poisson model as a torch autograd function, its backward the engine's
hand-written adjoint (`ptyb_gradients`).

    loss = PoissonLoss.apply(obj, probe, offsets, engine)
    loss.backward()       # obj.grad, probe.grad, offsets.grad

`obj` is complex `[1, nyo, nxo]` (every slice, `[nslice, nyo, nxo]`, on a multislice engine),
`probe` complex `[nprobe, ny, nx]`, `offsets` real `[nframe, 2]` (sub-pixel (dy, dx) per frame in
object pixels under Patch sampling, physwkim/ptyrs engine/features.rs:558-1025) or None (required
None on a multislice engine), `engine` a `GpuPtycho` of the scan. The loss is the Poisson LLK
sum over the unmasked pixels (engine/ops.rs:119-154); the complex gradients follow torch's
convention, ∂L/∂Re z + i·∂L/∂Im z, which is the reference's `obj_grad` / `probe_grad`
(engine/ptycho.rs:492-515), and the offsets' gradient is its `position_grad`
(engine/features.rs:1055-1100). Forward writes the arrays into the engine's state. CUDA tensors
stay on the device: they enter the engine by device pointer and their gradients are written
into CUDA tensors (complex64, the engine's precision); CPU tensors go through host arrays.
"""
import numpy as np
import torch


class PoissonLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, obj, probe, offsets, engine):
        if obj.is_cuda and probe.is_cuda:
            g = _device_pass(ctx, obj, probe, offsets, engine)
        else:
            g = _host_pass(ctx, obj, probe, offsets, engine)
        grads = []
        for x, key in ((obj, "object"), (probe, "probe"), (offsets, "positions")):
            if x is None:
                grads.append(None)
                continue
            v = g[key]
            grads.append(None if v is None else
                         torch.as_tensor(v, device=x.device).to(x.dtype).reshape(x.shape))
        ctx.grads = grads
        return torch.tensor(g["loss"], dtype=torch.float64, device=obj.device)

    @staticmethod
    def backward(ctx, grad_loss):
        out = [None if g is None else grad_loss.to(g.real.dtype) * g for g in ctx.grads]
        return out[0], out[1], out[2], None


def _host_pass(ctx, obj, probe, offsets, engine):
    """CPU tensors: through host arrays (complex128 at the C ABI)."""
    o = obj.detach().cpu().numpy().astype(np.complex128)
    if engine.nslice() > 1:
        engine.set_objects(o)
    else:
        engine.set_object(o)
    engine.set_probe(probe.detach().cpu().numpy().astype(np.complex128))
    if offsets is not None:
        engine.set_positions(offsets.detach().cpu().numpy().astype(np.float64), refine=False)
    return engine.gradients(obj=ctx.needs_input_grad[0], probe=ctx.needs_input_grad[1],
                            positions=offsets is not None)


def _device_pass(ctx, obj, probe, offsets, engine):
    """CUDA tensors: the object and probe go to the engine and the gradients come back as
    complex64 device memory (`data_ptr()` of contiguous tensors, reference
    `GpuPtycho::set_object_device`), with no host copy of either."""
    o = obj.detach().to(torch.complex64).contiguous()
    p = probe.detach().to(torch.complex64).contiguous()
    # the engine's stream reads them: the producers' work must have finished
    torch.cuda.current_stream(o.device).synchronize()
    if engine.nslice() > 1:
        engine.set_objects_device(o.data_ptr(), *o.shape)
    else:
        engine.set_object_device(o.data_ptr(), *o.shape)
    engine.set_probe_device(p.data_ptr(), *p.shape)
    if offsets is not None:
        engine.set_positions(offsets.detach().cpu().numpy().astype(np.float64), refine=False)
    go = torch.empty_like(o) if ctx.needs_input_grad[0] else None
    gp = torch.empty_like(p) if ctx.needs_input_grad[1] else None
    loss, gd = engine.gradients_device(None if go is None else go.data_ptr(),
                                       None if gp is None else gp.data_ptr(),
                                       positions=offsets is not None)
    return dict(loss=loss, object=go, probe=gp, positions=gd)


def poisson_loss(obj, probe, offsets, engine):
    """`PoissonLoss.apply(obj, probe, offsets, engine)`."""
    return PoissonLoss.apply(obj, probe, offsets, engine)
