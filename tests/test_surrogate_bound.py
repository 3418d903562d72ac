"""The accuracy a descreening-sum surrogate needs (surrogate.sum_accuracy_bound),
checked on the CPU against the FP64 oracle: the energy as a function of the
descreening sums, its derivative by finite differences, and the energy
error of random per-atom sum errors at the bound."""
import numpy as np

import oracle as O
from agbnp3_b200.surrogate import sum_accuracy_bound
from agbnp3_b200.system import make_globule

TOKCAL, RW = 332.0, 1.4


def _energy(beta, x, q, alpha, df):
    """GB + vdW energy of the oracle's formulas (agbnp3_utils.c:615-670,
    agbnp3_cpu_simd_kernels.c:66-151, agbnp3.c:1466-1487) at inverse Born
    radii beta"""
    b = 1.0 / np.where(beta < 0.0, 0.02, np.sqrt(0.02 ** 2 + beta ** 2))
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    bb = b[:, None] * b[None, :]
    f = 1.0 / np.sqrt(d2 + bb * np.exp(-0.25 * d2 / bb))
    iu = np.triu_indices(len(q), 1)
    epair = 2.0 * (q[:, None] * q[None, :] * f)[iu].sum()
    egb = TOKCAL * df * ((q * q / b).sum() + epair)
    return egb + (alpha / (b + RW) ** 3).sum()


def test_descreening_sum_sensitivity():
    s = make_globule(300, 5)
    Q = O.oracle_eval(s, compat=True, internals=True)
    I, a = Q["int"], O.internal_arrays(s)
    x = np.stack([a["x"], a["y"], a["z"]], 1)
    q, alpha, r = a["charge"], a["ialpha"], a["r"]
    df = -0.5 * (1.0 / s.eps_in - 1.0 / s.eps_out)
    bfil = I["br1"]  # the filtered inverse Born radius sqrt(0.02^2 + beta^2)
    assert (bfil > 0.02).all()
    beta = np.sqrt(bfil ** 2 - 0.02 ** 2)
    e0 = _energy(beta, x, q, alpha, df)
    assert abs(e0 - (Q["egb"] + Q["evdw"])) <= 1e-9 * abs(e0)
    # dE/d(S_i/4pi) = -(332 df q2ab_i + abrw_i), against central differences
    g = -(TOKCAL * df * I["q2ab"] + I["abrw"])
    h = 1e-6
    for i in (0, 7, 50, 123, 299):
        e1, e2 = beta.copy(), beta.copy()
        e1[i] -= h  # S_i/4pi up by h
        e2[i] += h
        fd = (_energy(e1, x, q, alpha, df) - _energy(e2, x, q, alpha, df)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(g[i]), 1e-3), (i, fd, g[i])
    # random per-atom relative errors of RMS sigma_random move the energy by
    # about target |E| (RMS over draws); a common one of sigma_common by target |E|
    S = 4.0 * np.pi * (1.0 / (r - 0.5) - beta)
    etot = Q["egb"] + Q["evdw"] + Q["ecav"] + Q["ehb"]
    bd = sum_accuracy_bound(S, r - 0.5, I["q2ab"], I["abrw"], etot, s.eps_in, s.eps_out)
    assert 0.0 < bd["sigma_common"] and 0.0 < bd["sigma_random"] and bd["kappa_median"] > 0.0
    rng = np.random.default_rng(3)
    dev = []
    for _ in range(40):
        eps = rng.normal(0.0, bd["sigma_random"], len(S))
        dev.append(_energy(1.0 / (r - 0.5) - S * (1.0 + eps) / (4.0 * np.pi), x, q, alpha, df) - e0)
    rms = np.sqrt(np.mean(np.square(dev))) / abs(etot)
    assert 0.6e-4 < rms < 1.6e-4, rms
    ec = _energy(1.0 / (r - 0.5) - S * (1.0 + bd["sigma_common"]) / (4.0 * np.pi), x, q, alpha, df) - e0
    assert 0.8e-4 < abs(ec) / abs(etot) < 1.25e-4, abs(ec) / abs(etot)
