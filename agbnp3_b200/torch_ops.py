"""PyTorch operators over the engine for callers whose coordinates already
live on the GPU (an MD engine or a training loop written in PyTorch).

    import agbnp3_b200 as A
    from agbnp3_b200 import torch_ops
    inst = A.Instance(system)                       # agbnp3_new
    xyz = torch.tensor(coords, device="cuda", dtype=torch.float64)
    e, sp, br, sa, grads = torch.ops.agbnp3.ener(inst.tag, False, 1, xyz)
    E = torch_ops.total_energy(inst, xyz.requires_grad_())
    E.backward()                                    # xyz.grad = dE/dx

Both call `agbnp3_ener_device` / `agbnp3_batch_ener_device` of the C-ABI on
torch's current stream: the evaluation is ordered after the work already
queued there and the outputs are ready for the work queued after it, with
no host copies.  Outputs:

    energies  [7 * members]   egb, evdw, ecorr_vdw, ecav, ecorr_cav, ehb,
                              mol_volume per member
    sp, br, surf_area  [N]
    grads     [4, N, 3]       d/dx of egb, evdw + ecorr_vdw, ecav +
                              ecorr_cav, ehb (the engine's gradient arrays)

The backward pass differentiates the energies only.  Because the second and
third gradient arrays belong to the sums evdw + ecorr_vdw and ecav +
ecorr_cav, it is exact for losses that weight each of these pairs equally
(the total energy does) and raises otherwise; mol_volume has no gradient.
"""
import ctypes

import torch

from . import AGBNP_OK, AGBNPError, last_error, lib

__all__ = ["ener", "total_energy"]


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


@torch.library.custom_op("agbnp3::ener", mutates_args=(), device_types="cuda")
def ener(tag: int, batch: bool, members: int, xyz: torch.Tensor) -> tuple[
        torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    if xyz.dim() != 2 or xyz.shape[1] != 3:
        raise ValueError("xyz must have shape [natoms, 3]")
    x = xyz.detach().to(torch.float64)
    cols = [x[:, k].contiguous() for k in range(3)]
    n = x.shape[0]
    opts = dict(dtype=torch.float64, device=x.device)
    energies = torch.empty(7 * members, **opts)
    sp, br, sa = (torch.empty(n, **opts) for _ in range(3))
    grads = torch.empty(4, n, 3, **opts)
    stream = torch.cuda.current_stream(x.device).cuda_stream
    fn = lib().agbnp3_batch_ener_device if batch else lib().agbnp3_ener_device
    rc = fn(tag, *(_vp(c) for c in cols), _vp(energies), _vp(sp), _vp(br), _vp(sa),
            *(_vp(grads[k]) for k in range(4)), ctypes.c_void_p(stream))
    if rc != AGBNP_OK:
        raise AGBNPError(f"agbnp3 device evaluation failed: {last_error()}")
    return energies, sp, br, sa, grads


@ener.register_fake
def _(tag, batch, members, xyz):
    n = xyz.shape[0]
    opts = dict(dtype=torch.float64, device=xyz.device)
    return (xyz.new_empty(7 * members, **opts), xyz.new_empty(n, **opts), xyz.new_empty(n, **opts),
            xyz.new_empty(n, **opts), xyz.new_empty(4, n, 3, **opts))


def _setup(ctx, inputs, output):
    ctx.save_for_backward(output[4])
    ctx.members = inputs[2]
    ctx.natoms = inputs[3].shape[0]
    ctx.dtype = inputs[3].dtype


def _backward(ctx, g_e, g_sp, g_br, g_sa, g_grads):
    (grads,) = ctx.saved_tensors
    if g_e is None:
        return None, None, None, None
    g = g_e.view(ctx.members, 7)
    if not (torch.equal(g[:, 1], g[:, 2]) and torch.equal(g[:, 3], g[:, 4])):
        raise RuntimeError("agbnp3::ener backward needs equal weights on evdw/ecorr_vdw and ecav/ecorr_cav")
    if torch.any(g[:, 6] != 0):
        raise RuntimeError("agbnp3::ener has no gradient for mol_volume")
    if ctx.members == 1:
        w = g[0, [0, 1, 3, 5]]
        gx = torch.einsum("k,knc->nc", w, grads)
    else:
        raise RuntimeError("agbnp3::ener backward of a batch: use one instance per operator call")
    return None, None, None, gx.to(ctx.dtype)


torch.library.register_autograd("agbnp3::ener", _backward, setup_context=_setup)


def total_energy(obj, xyz: torch.Tensor) -> torch.Tensor:
    """Sum of the six energy terms of one instance (kcal/mol), differentiable
    with respect to xyz [natoms, 3] on the instance's GPU."""
    e = torch.ops.agbnp3.ener(obj.tag, False, 1, xyz)[0]
    return e[:6].sum()
