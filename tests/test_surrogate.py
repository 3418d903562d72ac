"""Tensor-core (tcgen05) kernels of the learned surrogate against torch."""
import ctypes

import pytest
import torch

import agbnp3_b200 as A


def _lib():
    L = A.lib()
    L.agbnp3_tc_gemm.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                 ctypes.c_void_p] + [ctypes.c_int] * 4 + [ctypes.c_void_p]
    return L


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K,lda", [(128, 16, 16, 16), (300, 128, 160, 160), (257, 128, 128, 136), (64, 2, 128, 128),
                                       (1000, 256, 256, 256), (128, 160, 4096, 4096), (5, 7, 48, 48)])
def test_tc_gemm_matches_torch(M, N, K, lda):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    Abuf = torch.randn(M, lda, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(N, device="cuda", generator=g)
    C = torch.full((M, N), float("nan"), device="cuda")
    torch.cuda.synchronize()
    assert _lib().agbnp3_tc_gemm(_p(Abuf), lda, _p(B), K, _p(b), _p(C), N, M, N, K, None) == 0
    ref = Abuf[:, :K].float() @ B.float().T + b
    assert torch.allclose(C, ref, rtol=1e-4, atol=1e-3 * (K / 128) ** 0.5), (C - ref).abs().max().item()


CLASS_RADII = (1.7, 1.55, 1.52, 1.8, 1.15)  # C, N, O, S, H of the globule generator


def _features(inst, natoms):
    L = A.lib()
    L.agbnp3_surrogate_classes.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    L.agbnp3_surrogate_features.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    cr = (ctypes.c_double * 5)(*CLASS_RADII)
    un = ctypes.c_int(-1)
    assert L.agbnp3_surrogate_classes(inst.tag, cr, 5, ctypes.byref(un)) == A.AGBNP_OK
    out = torch.empty(natoms, 160, dtype=torch.bfloat16, device="cuda")
    assert L.agbnp3_surrogate_features(inst.tag, None, None, _p(out)) == A.AGBNP_OK
    torch.cuda.synchronize()  # the features are queued on the instance's stream
    return un.value, out.float().cpu().numpy()


@pytest.mark.gpu
def test_features_match_cpu_reference():
    import numpy as np
    import surrogate_ref as S
    from conftest import load_golden
    s, _ = load_golden("globule300_shuffled")
    inst = A.Instance(s, precision=A.PREC_MIXED)
    try:
        inst.ener()
        unmatched, F = _features(inst, s.natoms)
        assert unmatched == 0
        int2ext, _ = s.internal_order()
        radii = np.asarray(s.r)[int2ext]
        cls = np.array([int(np.argmin(np.abs(np.array(CLASS_RADII) - r))) for r in radii])
        xyz = s.coords()[int2ext].astype(np.float32).astype(np.float64)
        ref = S.features(xyz, cls)
        err = np.abs(F - ref)
        assert (err <= 1e-2 * np.abs(ref) + 2e-3).all(), err.max()
    finally:
        inst.close()


@pytest.mark.gpu
def test_mlp_gradients_match_cpu_reference():
    """One backward pass of the training kernels (tcgen05 GEMMs, SiLU and
    loss-gradient kernels) against the float64 NumPy reference on the same
    bf16-rounded inputs and weights."""
    import numpy as np
    import surrogate_ref as S
    from agbnp3_b200.surrogate import Mlp
    B = 256
    net = Mlp(seed=3, batch=B)
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn(B, 160, device="cuda", generator=g).to(torch.bfloat16)
    T = torch.randn(B, 2, device="cuda", generator=g)
    idx = torch.arange(B, device="cuda")
    loss = net.gradients(X, T, idx).item()
    torch.cuda.synchronize()
    p = {k: (v.to(torch.bfloat16).double() if k.startswith("W") else v.double()).cpu().numpy()
         for k, v in net.p.items()}
    ref_loss, ref = S.mlp_grads(p, X.double().cpu().numpy(), T.double().cpu().numpy())
    assert abs(loss - ref_loss) <= 2e-2 * abs(ref_loss)
    for k, r in ref.items():
        got = net.g[k].double().cpu().numpy()
        rel = np.linalg.norm(got - r) / np.linalg.norm(r)
        assert rel <= 3e-2, (k, rel)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 300, 1000, 20000])
def test_fused_forward_matches_layers(n):
    """The one-launch network (agbnp3_mlp_forward: three tcgen05 layers, the
    activations kept on chip) gives the layer-by-layer GEMM path's outputs:
    the same bf16 products accumulated in fp32 and the same bf16 rounding of
    the hidden activations, so they agree to fp32 rounding; row counts that
    are not a multiple of the 128-row tile and several tiles per block."""
    from agbnp3_b200 import surrogate as SG
    net = SG.Mlp(seed=3, batch=4096)
    for k in ("b1", "b2", "b3"):  # nonzero biases
        net.p[k].copy_(torch.linspace(-0.5, 0.5, len(net.p[k]), device="cuda"))
    g = torch.Generator(device="cuda").manual_seed(n)
    X = torch.randn(n, 160, device="cuda", generator=g).to(torch.bfloat16)
    ref = net.predict(X)
    out = net.predict_fused(X)
    torch.cuda.synchronize()
    assert net.L.agbnp3_tc_error(1, None) == 0
    assert torch.allclose(out, ref, rtol=1e-4, atol=1e-4), (out - ref).abs().max().item()


@pytest.mark.gpu
def test_surrogate_training_reduces_loss():
    """A short training run on FP64 labels of perturbed globule conformations
    lowers the loss and predicts held-out descreening sums better than their
    mean."""
    import numpy as np
    from agbnp3_b200 import surrogate as SG
    X, T = SG.make_dataset(conformations=12, natoms=1500, bases=3, log=lambda *a: None)
    ntr = 10 * 1500
    model = SG.train(X[:ntr], T[:ntr], epochs=6, batch=1024, lr=2e-3, log=lambda *a: None)
    assert model["loss"][-1] < 0.5 * model["loss"][0]
    net = SG.load_model(model, batch=1024)
    Xn = ((X[ntr:].float() - torch.as_tensor(model["fmean"], device="cuda"))
          * torch.as_tensor(model["finvstd"], device="cuda")).to(torch.bfloat16)
    Y = net.predict(Xn) * torch.as_tensor(model["tstd"], device="cuda") + torch.as_tensor(model["tmean"],
                                                                                          device="cuda")
    t = T[ntr:, 0].cpu().numpy()
    e = Y[:, 0].cpu().numpy() - t
    assert np.sqrt((e ** 2).mean()) < 0.5 * t.std()


@pytest.mark.gpu
def test_surrogate_gain_and_fallback():
    """What the trained ensemble gains, as gain() measures it: with
    tolerance 0 every atom falls back to the plain descreening and the GB
    energy is the exact one; with an infinite tolerance none does; in
    between the fallback fraction falls as the tolerance grows.  The
    networks' relative error of the descreening sums is above the accuracy
    the 1e-4 energy target needs (sum_accuracy_bound), so without fallback
    the GB energy misses 1e-4, and meeting it takes most atoms back to the
    exact sums; the measured times and the gain are printed."""
    import json
    from agbnp3_b200 import surrogate as SG
    X, T = SG.make_dataset(conformations=12, natoms=1500, bases=3, log=lambda *a: None)
    models = [SG.train(X, T, epochs=4, batch=1024, lr=2e-3, seed=sd, log=lambda *a: None) for sd in (0, 1)]
    r = SG.gain(models, 3000, seed=11)
    print(json.dumps(r))
    rows = r["rows"]
    assert rows[0]["fallback_fraction"] == 1.0 and rows[0]["egb_rel_err"] <= 1e-12
    assert rows[0]["linearised_total_rel_err"] == 0.0
    assert rows[-1]["fallback_fraction"] == 0.0
    fr = [q["fallback_fraction"] for q in rows]
    assert all(a >= b for a, b in zip(fr, fr[1:]))
    assert r["surrogate_ms"] > 0 and r["exact_stage_ms"] > 0 and r["features_ms"] > 0 and r["networks_ms"] > 0
    b = r["accuracy_bound"]
    assert 0.0 < b["sigma_common"] < b["sigma_random"] < r["network_rel_rms_err"]
    assert rows[-1]["egb_rel_err"] > 1e-4
    assert r["min_fallback_meeting_1e-4"] >= 0.5
