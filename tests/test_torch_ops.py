"""PyTorch operators over the device-array entry points (agbnp3_ener_device,
agbnp3_batch_ener_device): same results as the host-array API, gradients
through autograd, ordering on torch's current stream."""
import numpy as np
import pytest
import torch

import agbnp3_b200 as A
from conftest import ENERGY_KEYS, load_golden, rms_rel


def test_operator_registered():
    from agbnp3_b200 import torch_ops  # noqa: F401
    assert hasattr(torch.ops.agbnp3, "ener")


def _host(inst, s):
    r = inst.ener(s.coords())
    return np.array([r[k] for k in ENERGY_KEYS]), r


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_ener_device_matches_host(prec):
    from agbnp3_b200 import torch_ops
    s, _ = load_golden("globule2000_hbmix")
    inst = A.Instance(s, precision=prec)
    try:
        e_host, r = _host(inst, s)
        xyz = torch.tensor(s.coords(), dtype=torch.float64, device="cuda")
        side = torch.cuda.Stream()
        with torch.cuda.stream(side):  # a non-default current stream
            xyz2 = xyz * 1.0           # queued on the side stream before the operator
            e, sp, br, sa, g = torch.ops.agbnp3.ener(inst.tag, False, 1, xyz2)
            e2 = e.clone()
        torch.cuda.synchronize()
        tol = 1e-12 if prec == A.PREC_FP64 else 1e-9
        assert np.allclose(e2.cpu().numpy(), e_host, rtol=tol, atol=tol)
        for k, name in enumerate(("dgbdr", "dvwdr", "decav", "dehb")):
            assert rms_rel(g[k].cpu().numpy(), r[name]) <= tol, name
        for t, name in ((sp, "sp"), (br, "br"), (sa, "surf_area")):
            assert rms_rel(t.cpu().numpy(), r[name]) <= tol, name
        # autograd of the total energy
        x = xyz.clone().requires_grad_()
        E = torch_ops.total_energy(inst, x)
        E.backward()
        want = r["dgbdr"] + r["dvwdr"] + r["decav"] + r["dehb"]
        assert abs(E.item() - e_host[:6].sum()) <= tol * abs(e_host[:6].sum())
        assert rms_rel(x.grad.cpu().numpy(), want) <= tol
    finally:
        inst.close()


@pytest.mark.gpu
def test_batch_ener_device_matches_members():
    from agbnp3_b200 import torch_ops  # noqa: F401
    systems = [load_golden(n)[0] for n in ("globule50", "globule300_shuffled", "globule2000_hbmix")]
    insts = [A.Instance(x, precision=A.PREC_FP64) for x in systems]
    B = A.Batch(insts)
    B.set_mode(A.PREC_FP64, True)
    try:
        xyz = torch.tensor(np.concatenate([x.coords() for x in systems]), dtype=torch.float64, device="cuda")
        e, sp, br, sa, g = torch.ops.agbnp3.ener(B.btag, True, len(systems), xyz)
        torch.cuda.synchronize()
        e = e.view(len(systems), 7).cpu().numpy()
        for k, x in enumerate(systems):
            r = insts[k].ener(x.coords())
            o0, o1 = B.offsets[k], B.offsets[k + 1]
            assert np.allclose(e[k], [r[q] for q in ENERGY_KEYS], rtol=1e-10, atol=1e-10)
            assert rms_rel(g[0, o0:o1].cpu().numpy(), r["dgbdr"]) <= 1e-10
    finally:
        B.close()
        for i in insts:
            i.close()
