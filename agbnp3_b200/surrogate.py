"""Learned surrogate of the per-atom descreening sums and self volumes.

A per-atom MLP (160 radial-feature inputs, two hidden layers of 128 SiLU
units, 2 outputs) maps an atom's neighbourhood within 8 A to its
descreening sum S_i = sum_j sp_j Q4_ij (the sum in 1/B_i = 1/R_i - S_i/4pi)
and its self volume sp_i V_i.  Weights are used in bf16 with fp32
accumulation; every matrix product of the forward and backward passes is
the library's tcgen05 GEMM (agbnp3_tc_gemm) and every other step (SiLU and
its derivative, the loss gradient, Adam, weight packing, batch gathering)
one of its kernels (agbnp3_mlp_*).  torch only holds the device buffers.

    python -m agbnp3_b200.surrogate train --out model.npz [--conformations 2000 --natoms 5000]
    python -m agbnp3_b200.surrogate evaluate --model model.npz --natoms 25000
    python -m agbnp3_b200.surrogate bound [--natoms N]   (accuracy the sums need)
    python -m agbnp3_b200.surrogate kernels --natoms N --epochs REPS   (inference kernels alone)

Training data: perturbed conformations (N(0, 0.3 A) coordinate noise) of
seeded globules, labelled by the plain FP64 path of the engine.
"""
import argparse
import ctypes
import time

import numpy as np
import torch

from . import AGBNP_OK, AGBNPError, Instance, PREC_FP64, PREC_MIXED, last_error, lib, make_globule

NIN, NH, NOUT = 160, 128, 2
CLASS_RADII = (1.7, 1.55, 1.52, 1.8, 1.15)  # C, N, O, S, H (A, without the 0.5 A increment)
ATOM_DESC_SUM, ATOM_SP = 19, 3  # per-atom debug arrays: descreening sum, sp
ATOM_Q2AB, ATOM_ABRW = 12, 13  # the chain-rule factors through the Born radii


def _bind():
    L = lib()
    vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.agbnp3_tc_gemm_async.argtypes = [vp, i, vp, i, vp, vp, i, i, i, i, vp]
    L.agbnp3_tc_error.argtypes = [i, vp]
    L.agbnp3_mlp_act.argtypes = [vp, i, i, i, vp, i, vp, i, vp]
    L.agbnp3_mlp_act_grad.argtypes = [vp, vp, i, i, vp, vp, i, vp, vp]
    L.agbnp3_mlp_mse_grad.argtypes = [vp, vp, i, i, f, vp, vp, i, vp, vp, vp]
    L.agbnp3_mlp_adam.argtypes = [vp, vp, vp, vp, ctypes.c_longlong, f, f, f, f, i, vp]
    L.agbnp3_mlp_pack.argtypes = [vp, i, i, vp, vp, i, vp]
    L.agbnp3_mlp_gather.argtypes = [vp, vp, vp, i, i, i, vp, vp, i, vp, vp]
    L.agbnp3_surrogate_classes.argtypes = [i, vp, i, vp]
    L.agbnp3_surrogate_features.argtypes = [i, vp, vp, vp]
    L.agbnp3_mlp_forward.argtypes = [vp, i, vp, vp, vp, vp, vp, vp, vp, vp]
    return L


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _ok(rc, what):
    if rc != 0:
        raise AGBNPError(f"{what} failed ({rc})")


class Mlp:
    """Parameters (fp32 masters, bf16 copies for the GEMMs), Adam state and
    work buffers of one network; forward / backward by the library's
    kernels on torch's current stream."""

    def __init__(self, seed=0, batch=4096, lr=1e-3, device="cuda"):
        self.L = _bind()
        g = torch.Generator().manual_seed(seed)
        dev = torch.device(device)

        def init(n, k):
            return (torch.randn(n, k, generator=g) * (2.0 / k) ** 0.5).to(dev)

        self.p = {"W1": init(NH, NIN), "b1": torch.zeros(NH, device=dev), "W2": init(NH, NH),
                  "b2": torch.zeros(NH, device=dev), "W3": init(NOUT, NH) * 0.1, "b3": torch.zeros(NOUT, device=dev)}
        self.m = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.g = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.t, self.lr, self.batch, self.dev = 0, lr, batch, dev
        bf = dict(dtype=torch.bfloat16, device=dev)
        self.W1b, self.W2b, self.W3b = torch.empty(NH, NIN, **bf), torch.empty(NH, NH, **bf), torch.empty(NOUT, NH, **bf)
        self.W2t, self.W3t = torch.empty(NH, NH, **bf), torch.empty(NH, 16, **bf)
        self.pack()
        self._alloc(batch)

    def _alloc(self, B):
        f32, bf = dict(dtype=torch.float32, device=self.dev), dict(dtype=torch.bfloat16, device=self.dev)
        self.B = B
        self.Xb, self.Xt, self.Tb = torch.empty(B, NIN, **bf), torch.empty(NIN, B, **bf), torch.empty(B, NOUT, **f32)
        self.Z1, self.Z2, self.Y = torch.empty(B, NH, **f32), torch.empty(B, NH, **f32), torch.empty(B, NOUT, **f32)
        self.H1, self.H1t = torch.empty(B, NH, **bf), torch.empty(NH, B, **bf)
        self.H2, self.H2t = torch.empty(B, NH, **bf), torch.empty(NH, B, **bf)
        self.dY16, self.dYt = torch.empty(B, 16, **bf), torch.empty(NOUT, B, **bf)
        self.dH = torch.empty(B, NH, **f32)
        self.dZ, self.dZt = torch.empty(B, NH, **bf), torch.empty(NH, B, **bf)
        self.loss = torch.zeros(1, **f32)

    def _s(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def pack(self):
        L, s, p = self.L, self._s(), self.p
        _ok(L.agbnp3_mlp_pack(_p(p["W1"]), NH, NIN, _p(self.W1b), None, NH, s), "pack W1")
        _ok(L.agbnp3_mlp_pack(_p(p["W2"]), NH, NH, _p(self.W2b), _p(self.W2t), NH, s), "pack W2")
        _ok(L.agbnp3_mlp_pack(_p(p["W3"]), NOUT, NH, _p(self.W3b), _p(self.W3t), 16, s), "pack W3")

    def _gemm(self, A, lda, B, ldb, bias, C, ldc, M, N, K):
        _ok(self.L.agbnp3_tc_gemm_async(_p(A), lda, _p(B), ldb, _p(bias), _p(C), ldc, M, N, K, self._s()), "tc_gemm")

    def forward_batch(self, Xb, n, train=False):
        """Y[:n] for bf16 inputs Xb [n, 160] (n <= B); keeps the activations
        (and, for training, their transposes)"""
        L, s, p = self.L, self._s(), self.p
        h1t, h2t = (self.H1t, self.H2t) if train else (None, None)
        self._gemm(Xb, NIN, self.W1b, NIN, p["b1"], self.Z1, NH, n, NH, NIN)
        _ok(L.agbnp3_mlp_act(_p(self.Z1), n, NH, NH, _p(self.H1), NH, _p(h1t), self.B, s), "act1")
        self._gemm(self.H1, NH, self.W2b, NH, p["b2"], self.Z2, NH, n, NH, NH)
        _ok(L.agbnp3_mlp_act(_p(self.Z2), n, NH, NH, _p(self.H2), NH, _p(h2t), self.B, s), "act2")
        self._gemm(self.H2, NH, self.W3b, NH, p["b3"], self.Y, NOUT, n, NOUT, NH)
        return self.Y[:n]

    def gradients(self, X, T, idx):
        """loss and parameter gradients (self.g) of the batch X[idx], T[idx]"""
        L, s, B = self.L, self._s(), len(idx)
        if B != self.B:
            self._alloc(B)
        _ok(L.agbnp3_mlp_gather(_p(X), _p(T), _p(idx), B, NIN, NOUT, _p(self.Xb), _p(self.Xt), B, _p(self.Tb), s),
            "gather")
        self.forward_batch(self.Xb, B, train=True)
        for v in self.g.values():
            v.zero_()
        self.loss.zero_()
        g = self.g
        _ok(L.agbnp3_mlp_mse_grad(_p(self.Y), _p(self.Tb), B, NOUT, 1.0 / B, _p(self.dY16), _p(self.dYt), B,
                                  _p(g["b3"]), _p(self.loss), s), "mse")
        self._gemm(self.dYt, B, self.H2t, B, None, g["W3"], NH, NOUT, NH, B)
        self._gemm(self.dY16, 16, self.W3t, 16, None, self.dH, NH, B, NH, 16)
        _ok(L.agbnp3_mlp_act_grad(_p(self.dH), _p(self.Z2), B, NH, _p(self.dZ), _p(self.dZt), B, _p(g["b2"]), s),
            "act_grad2")
        self._gemm(self.dZt, B, self.H1t, B, None, g["W2"], NH, NH, NH, B)
        self._gemm(self.dZ, NH, self.W2t, NH, None, self.dH, NH, B, NH, NH)
        _ok(L.agbnp3_mlp_act_grad(_p(self.dH), _p(self.Z1), B, NH, None, _p(self.dZt), B, _p(g["b1"]), s),
            "act_grad1")
        self._gemm(self.dZt, B, self.Xt, B, None, g["W1"], NIN, NH, NIN, B)
        return self.loss

    def step(self, X, T, idx):
        loss = self.gradients(X, T, idx)
        self.t += 1
        for k in self.p:
            _ok(self.L.agbnp3_mlp_adam(_p(self.p[k]), _p(self.g[k]), _p(self.m[k]), _p(self.v[k]), self.p[k].numel(),
                                       self.lr, 0.9, 0.999, 1e-8, self.t, self._s()), "adam")
        self.pack()
        return loss

    def predict(self, X):
        """fp32 outputs for bf16 inputs X [n, 160]"""
        n = len(X)
        out = torch.empty(n, NOUT, device=self.dev)
        for r0 in range(0, n, self.B):
            r1 = min(n, r0 + self.B)
            out[r0:r1] = self.forward_batch(X[r0:r1], r1 - r0)
        return out

    def predict_fused(self, X):
        """fp32 outputs [n, 2] for bf16 inputs X [n, 160], all three layers in
        one launch (agbnp3_mlp_forward: weights in shared memory, activations
        in TMEM and shared memory)"""
        X = X.contiguous()
        n = len(X)
        out = torch.empty(n, NOUT, device=self.dev)
        p = self.p
        _ok(self.L.agbnp3_mlp_forward(_p(X), n, _p(self.W1b), _p(p["b1"]), _p(self.W2b), _p(p["b2"]), _p(self.W3b),
                                      _p(p["b3"]), _p(out), self._s()), "mlp_forward")
        return out

    def state(self):
        return {k: v.detach().cpu().numpy() for k, v in self.p.items()}

    def load(self, st):
        for k in self.p:
            self.p[k].copy_(torch.as_tensor(st[k], device=self.dev))
        self.pack()


def set_classes(inst):
    """assigns the atom classes from the radii; returns the unmatched count"""
    L = _bind()
    cr = (ctypes.c_double * len(CLASS_RADII))(*CLASS_RADII)
    un = ctypes.c_int(0)
    if L.agbnp3_surrogate_classes(inst.tag, cr, len(CLASS_RADII), ctypes.byref(un)) != AGBNP_OK:
        raise AGBNPError("agbnp3_surrogate_classes failed")
    return un.value


def features(inst, natoms, mean=None, invstd=None, out=None):
    """radial features (bf16 [natoms, 160], internal order) of the coordinates
    of inst's last evaluation, ordered before the work that torch's current
    stream queues next"""
    if out is None:
        out = torch.empty(natoms, NIN, dtype=torch.bfloat16, device="cuda")
    ist = torch.cuda.ExternalStream(inst.stream)
    ist.wait_stream(torch.cuda.current_stream())
    if _bind().agbnp3_surrogate_features(inst.tag, _p(mean), _p(invstd), _p(out)) != AGBNP_OK:
        raise AGBNPError("agbnp3_surrogate_features failed")
    torch.cuda.current_stream().wait_stream(ist)
    return out


def classes_and_features(inst, natoms, mean=None, invstd=None):
    un = set_classes(inst)
    return un, features(inst, natoms, mean, invstd)


def labels(inst, natoms, system):
    """FP64 labels of the last evaluation, internal order: descreening sum,
    self volume sp V (hydrogens: 0)"""
    S = inst.atom_array(ATOM_DESC_SUM)
    sp = inst.atom_array(ATOM_SP)
    int2ext, _ = system.internal_order()
    r = np.asarray(system.r)[int2ext] + 0.5
    vol = 4.0 / 3.0 * np.pi * r ** 3
    heavy = np.zeros(natoms, bool)
    heavy[:system.nheavy] = True
    return np.stack([S, np.where(heavy, sp * vol, 0.0)], 1)


def make_dataset(conformations, natoms, bases=20, noise=0.3, seed=7, log=print):
    """features (raw, bf16) and FP64 labels of perturbed conformations"""
    per = max(1, conformations // bases)
    X, T = [], []
    rng = np.random.default_rng(seed)
    t0 = time.time()
    for b in range(bases):
        s = make_globule(natoms, seed * 1000 + b)
        inst = Instance(s, precision=PREC_FP64)
        for k in range(per if b < bases - 1 else conformations - per * (bases - 1)):
            xyz = s.coords() + rng.normal(0.0, noise, size=(s.natoms, 3))
            inst.ener(xyz)
            sv = s.with_coords(xyz)
            un, F = classes_and_features(inst, s.natoms)
            X.append(F)
            T.append(torch.as_tensor(labels(inst, s.natoms, sv), dtype=torch.float32, device="cuda"))
        inst.close()
        log(f"base {b + 1}/{bases}: {len(X)} conformations, {time.time() - t0:.1f} s")
    return torch.cat(X), torch.cat(T)


def train(X, T, epochs=2, batch=4096, lr=1e-3, seed=0, log=print):
    """normalises inputs and targets and trains one network; returns the model
    dictionary (parameters + normalisation)"""
    Xf = X.float()
    mean = Xf.mean(0)
    invstd = 1.0 / Xf.std(0).clamp_min(1e-3)
    Xn = ((Xf - mean) * invstd).to(torch.bfloat16)
    del Xf
    tmean, tstd = T.mean(0), T.std(0).clamp_min(1e-6)
    Tn = (T - tmean) / tstd
    net = Mlp(seed=seed, batch=batch, lr=lr)
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = len(Xn)
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g, device="cuda")
        tot, cnt = torch.zeros(1, device="cuda"), 0
        for r0 in range(0, n - batch + 1, batch):
            tot += net.step(Xn, Tn, perm[r0:r0 + batch])
            cnt += 1
        hist.append(tot.item() / cnt)
        log(f"epoch {ep + 1}: loss {hist[-1]:.5f} (normalised targets)")
    if net.L.agbnp3_tc_error(1, None) != 0:
        raise AGBNPError("a tensor-core MMA did not complete")
    model = {k: v for k, v in net.state().items()}
    model.update(fmean=mean.cpu().numpy(), finvstd=invstd.cpu().numpy(), tmean=tmean.cpu().numpy(),
                 tstd=tstd.cpu().numpy(), loss=np.array(hist))
    return model


def load_model(model, seed=0, batch=4096):
    net = Mlp(seed=seed, batch=batch)
    net.load(model)
    return net


def predict_system(net, model, inst, natoms):
    """predicted (descreening sum, self volume) per atom, internal order, for
    the coordinates of inst's last evaluation; and the unmatched-atom count"""
    mean = torch.as_tensor(model["fmean"], device="cuda")
    invstd = torch.as_tensor(model["finvstd"], device="cuda")
    un, F = classes_and_features(inst, natoms, mean, invstd)
    Y = net.predict_fused(F)
    Y = Y * torch.as_tensor(model["tstd"], device="cuda") + torch.as_tensor(model["tmean"], device="cuda")
    return un, Y


def born_radii(S, radius):
    """Born radii from descreening sums as the engine computes them
    (agbnp3.c:1174-1188): beta = 1/R - S/4pi, filtered to sqrt(0.02^2 + beta^2)"""
    beta = 1.0 / radius - S / (4.0 * np.pi)
    bf = np.where(beta < 0.0, 0.02, np.sqrt(0.02 ** 2 + beta ** 2))
    return 1.0 / bf


def energy_gradient_in_sums(q2ab, abrw, eps_in, eps_out):
    """dE/dS_i = -(332 df q2ab_i + abrw_i) / 4pi for every atom (see
    sum_accuracy_bound)"""
    df = -0.5 * (1.0 / eps_in - 1.0 / eps_out)
    return -(332.0 * df * np.asarray(q2ab, dtype=np.float64) + np.asarray(abrw, dtype=np.float64)) / (4.0 * np.pi)


def sum_accuracy_bound(S, radius, q2ab, abrw, e_total, eps_in, eps_out, target=1e-4):
    """How accurately a surrogate must reproduce the descreening sums S_i
    (the sum in 1/B_i = 1/R_i - S_i/4pi) for the total energy to stay within
    `target` (relative), to first order.

    dE/dS_i = -(332 df q2ab_i + abrw_i) / 4pi with df = -(1/eps_in -
    1/eps_out)/2: the GB energy and the vdW term depend on S_i only through
    B_i (agbnp3_utils.c:615-670, agbnp3.c:1466-1487; q2ab_i and abrw_i are
    the chain-rule factors the engine forms after the GB pair pass,
    agbnp3_cpu_simd_kernels.c:440-457).  With w_i = S_i dE/dS_i, relative
    errors e_i of the sums move the energy by sum_i w_i e_i: independent
    errors of RMS sigma by sigma |w|_2 (RMS), a common relative error sigma
    by sigma |sum_i w_i|.  Returns the largest sigma of each kind, and the
    distribution of kappa_i = (S_i/4pi) / beta_i, the factor by which the
    subtraction 1/R_i - S_i/4pi amplifies a relative error of S_i."""
    S, radius = (np.asarray(a, dtype=np.float64) for a in (S, radius))
    w = energy_gradient_in_sums(q2ab, abrw, eps_in, eps_out) * S
    beta = 1.0 / radius - S / (4.0 * np.pi)
    kappa = (S / (4.0 * np.pi)) / np.maximum(beta, 1e-12)
    return {"target": target,
            "sigma_random": float(target * abs(e_total) / np.sqrt((w ** 2).sum())),
            "sigma_common": float(target * abs(e_total) / abs(w.sum())),
            "kappa_median": float(np.median(kappa)), "kappa_p90": float(np.percentile(kappa, 90)),
            "kappa_max": float(kappa.max())}


# largest system agbnp3_gb_energy_static accepts (the size of its static
# device scratch array)
STATIC_MAX_ATOMS = 32768


def gb_energy(system, int2ext, radii_b):
    """GB energy (kcal/mol) of the system (internal order) at the given Born
    radii, by the library's allocation-free GB pair kernel
    (agbnp3_gb_energy_static), which takes at most STATIC_MAX_ATOMS atoms."""
    if not 0 < system.natoms <= STATIC_MAX_ATOMS:
        raise AGBNPError(f"gb_energy: {system.natoms} atoms; agbnp3_gb_energy_static takes 1..{STATIC_MAX_ATOMS}")
    L = lib()
    vp = ctypes.c_void_p
    L.agbnp3_gb_energy_static.argtypes = [ctypes.c_int] + [vp] * 5 + [ctypes.c_double] * 2 + [vp] * 3 + [vp]
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    xyz = system.coords()[int2ext]
    n = system.natoms
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    dera = torch.zeros(n, dtype=torch.float64, device="cuda")
    grad = torch.zeros(n, 3, dtype=torch.float64, device="cuda")
    args = [d(xyz[:, 0]), d(xyz[:, 1]), d(xyz[:, 2]), d(np.asarray(system.charge)[int2ext]), d(radii_b)]
    torch.cuda.synchronize()
    rc = L.agbnp3_gb_energy_static(n, *(_p(a) for a in args), system.eps_in, system.eps_out, _p(e), _p(dera),
                                   _p(grad), None)
    if rc != AGBNP_OK:
        raise AGBNPError(f"agbnp3_gb_energy_static failed: {last_error()}")
    torch.cuda.synchronize()
    return e.item()


def gain(models, natoms, seed=1, tolerances=(0.0, 0.01, 0.03, 0.1, 0.3, float("inf"))):
    """What the ensemble surrogate gains on one globule, all measured:
    - the device time of the surrogate inference (features + networks) and of
      the exact descreening stage it would replace (chosen mode);
    - for each tolerance of the residual check (atoms whose two networks
      disagree by more than tol on the descreening sum fall back to the
      exact sum) the fraction that falls back and the relative error of the
      GB energy at the resulting Born radii;
    - the networks' relative RMS error of the sums against the accuracy the
      1e-4 energy target needs (sum_accuracy_bound, from the FP64 path's
      chain-rule factors)."""
    s = make_globule(natoms, seed)
    int2ext, _ = s.internal_order()
    radius = np.asarray(s.r)[int2ext]
    inst = Instance(s, precision=PREC_FP64)
    R64 = inst.ener()
    exact = labels(inst, natoms, s)[:, 0]
    q2ab, abrw = inst.atom_array(ATOM_Q2AB), inst.atom_array(ATOM_ABRW)
    e_total = sum(R64[k] for k in ("egb", "evdw", "ecav", "ehb"))
    bound = sum_accuracy_bound(exact, radius, q2ab, abrw, e_total, s.eps_in, s.eps_out)
    dEdS = energy_gradient_in_sums(q2ab, abrw, s.eps_in, s.eps_out)
    # the exact stage's time, from the chosen (mixed) path
    mixed = Instance(s, precision=PREC_MIXED)
    mixed.ener()
    mixed.stage_timing(True)
    ts = []
    for _ in range(5):
        mixed.ener()
        ts.append(mixed.stage_times()["invb"])
    t_exact = float(np.median(ts))
    mixed.close()
    nets = [load_model(m, batch=max(4096, (natoms + 15) // 16 * 16)) for m in models]
    means = [torch.as_tensor(m["fmean"], device="cuda") for m in models]
    invs = [torch.as_tensor(m["finvstd"], device="cuda") for m in models]
    set_classes(inst)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    preds = []
    times = []
    F = torch.empty(natoms, NIN, dtype=torch.bfloat16, device="cuda")
    for rep in range(4):
        e0.record()
        preds = []
        last = None
        for net, m, mu, iv in zip(nets, models, means, invs):
            if last is None or not (torch.equal(mu, last[0]) and torch.equal(iv, last[1])):
                features(inst, natoms, mu, iv, out=F)  # shared by networks with one normalisation
                last = (mu, iv)
            Y = net.predict_fused(F)[:, 0] * float(m["tstd"][0]) + float(m["tmean"][0])
            preds.append(Y)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    t_sur = float(np.median(times[1:]))

    def timed(fn, reps=5):
        ts = []
        for _ in range(reps):
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts[1:]))

    t_feat = timed(lambda: features(inst, natoms, means[0], invs[0], out=F))
    t_nets = timed(lambda: [n.predict_fused(F) for n in nets])
    P = torch.stack(preds).cpu().numpy()
    mean, spread = P.mean(0), np.abs(P[0] - P[1]) if len(P) > 1 else np.zeros(natoms)
    # the GB energy at the surrogate's Born radii needs the allocation-free GB
    # kernel, which takes at most STATIC_MAX_ATOMS atoms; beyond that only the
    # first-order total-energy errors are reported, and the smallest fallback
    # that meets 1e-4 is judged by their RMS over sign draws (one signed sum
    # can cancel by chance)
    exact_gb = natoms <= STATIC_MAX_ATOMS
    e_exact = gb_energy(s, int2ext, born_radii(exact, radius)) if exact_gb else None
    rows = []
    for tol in tolerances:
        fall = spread > tol if np.isfinite(tol) else np.zeros(natoms, bool)
        if tol == 0.0:
            fall[:] = True
        S = np.where(fall, exact, mean)
        frac = float(fall.mean())
        de = dEdS * (S - exact)  # first-order energy change of each atom's error
        row = {"tolerance": tol, "fallback_fraction": frac,
               "linearised_total_rel_err": float(abs(de.sum()) / abs(e_total)),
               # the same errors with independent signs: the RMS over sign draws
               "linearised_rms_rel_err": float(np.sqrt((de ** 2).sum()) / abs(e_total)),
               "rms_sum_err": float(np.sqrt(((S - exact) ** 2).mean()))}
        if exact_gb:
            e = gb_energy(s, int2ext, born_radii(S, radius))
            row["egb_rel_err"] = abs(e - e_exact) / abs(e_exact)
        rows.append(row)
    inst.close()
    key = "egb_rel_err" if exact_gb else "linearised_rms_rel_err"
    ok = [q["fallback_fraction"] for q in rows if q[key] <= 1e-4]
    return {"natoms": natoms, "surrogate_ms": t_sur, "features_ms": t_feat, "networks_ms": t_nets,
            "exact_stage_ms": t_exact,
            "stage_speedup_without_fallback": t_exact / t_sur, "egb": e_exact, "rows": rows,
            "network_rel_rms_err": float(np.sqrt((((mean - exact) / np.abs(exact)) ** 2).mean())),
            "accuracy_bound": bound, "min_fallback_meeting_1e-4": min(ok) if ok else None,
            "error_measure": key}


def bench_report(sizes=(25000, 50000), conformations=60, train_atoms=5000, epochs=4, log=lambda *a: None):
    """The surrogate's measured figures for the benchmark line: two networks
    trained on the GPU (perturbed conformations of train_atoms-atom globules
    labelled by the FP64 path, a reduced set so that it fits a benchmark run),
    then gain() on a globule of each size."""
    import time as _t
    t0 = _t.time()
    X, T = make_dataset(conformations, train_atoms, bases=max(1, conformations // 10), log=log)
    models = [train(X, T, epochs=epochs, batch=4096, lr=2e-3, seed=sd, log=log) for sd in (0, 1)]
    del X, T
    t_train = _t.time() - t0
    out = {"training": {"conformations": conformations, "atoms": train_atoms, "epochs": epochs, "networks": 2,
                        "seconds": t_train, "final_loss": [float(m["loss"][-1]) for m in models]}}
    for n in sizes:
        out[str(n)] = gain(models, n)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "evaluate", "gain", "bound", "kernels"])
    ap.add_argument("--models", nargs="*", default=[])
    ap.add_argument("--seeds", type=int, nargs="*", default=[0])
    ap.add_argument("--out", default="surrogate_model.npz")
    ap.add_argument("--model", default="surrogate_model.npz")
    ap.add_argument("--conformations", type=int, default=2000)
    ap.add_argument("--natoms", type=int, default=5000)
    ap.add_argument("--epochs", type=int, default=2)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    from . import initialize
    initialize()
    if a.cmd == "train":
        X, T = make_dataset(a.conformations, a.natoms)
        for sd in a.seeds:
            model = train(X, T, epochs=a.epochs, seed=sd)
            out = a.out.replace("{seed}", str(sd))
            np.savez(out, **model)
            print(f"saved {out}")
    elif a.cmd == "kernels":
        # the inference kernels alone (untrained network), for timing and
        # profiling: features of a globule, then the fused network on them
        s = make_globule(a.natoms, 1)
        inst = Instance(s, precision=PREC_MIXED)
        inst.ener()
        set_classes(inst)
        net = Mlp(seed=a.seed)
        F = torch.empty(s.natoms, NIN, dtype=torch.bfloat16, device="cuda")
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        for _ in range(a.epochs):
            e0.record()
            features(inst, s.natoms, out=F)
            e1.record()
            net.predict_fused(F)
            e2.record()
            e2.synchronize()
            print(f"{s.natoms} atoms: features {e0.elapsed_time(e1):.3f} ms, network {e1.elapsed_time(e2):.3f} ms")
        inst.close()
    elif a.cmd == "bound":
        import json
        for n in (a.natoms,) if a.natoms != 5000 else (5000, 25000, 50000):
            s = make_globule(n, 1)
            inst = Instance(s, precision=PREC_FP64)
            R = inst.ener()
            int2ext, _ = s.internal_order()
            b = sum_accuracy_bound(inst.atom_array(ATOM_DESC_SUM), np.asarray(s.r)[int2ext],
                                   inst.atom_array(ATOM_Q2AB), inst.atom_array(ATOM_ABRW),
                                   sum(R[k] for k in ("egb", "evdw", "ecav", "ehb")), s.eps_in, s.eps_out)
            print(json.dumps({"natoms": n, **b}))
            inst.close()
    elif a.cmd == "gain":
        import json
        r = gain([dict(np.load(m)) for m in a.models], a.natoms)
        print(json.dumps(r))
    else:
        model = dict(np.load(a.model))
        net = load_model(model)
        s = make_globule(a.natoms, 1)
        inst = Instance(s, precision=PREC_FP64)
        inst.ener()
        un, Y = predict_system(net, model, inst, s.natoms)
        ref = labels(inst, s.natoms, s)
        Y = Y.cpu().numpy()
        for k, name in enumerate(("descreening sum", "self volume")):
            e = Y[:, k] - ref[:, k]
            print(f"{name}: rms error {np.sqrt((e ** 2).mean()):.4g}, rms value {np.sqrt((ref[:, k] ** 2).mean()):.4g}, "
                  f"mean error {e.mean():.4g}, unmatched atoms {un}")


if __name__ == "__main__":
    main()
