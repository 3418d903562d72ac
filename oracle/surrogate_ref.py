"""CPU reference of the learned surrogate's pieces, for the tests only: the
radial neighbour features and the MLP's forward and backward passes in
NumPy (float64).  It restates the definitions the device kernels implement
(agbnp3_b200/csrc/agbnp3_dev.cu k_sfeat, agbnp3_b200/surrogate.py) so that
their outputs and gradients can be checked; it is never on the product path.
"""
import numpy as np

NC, NB, RC, W = 5, 32, 8.0, 4
DELTA = RC / (NB - 1)


def features(xyz, cls):
    """xyz [n, 3] and class [n] (-1: none) in the engine's internal order ->
    raw features [n, NC * NB]: per neighbour class the Gaussians of width
    DELTA centred at k * DELTA (only the 2W+1 nearest to each distance)
    times 0.5 (cos(pi d / RC) + 1), summed over neighbours within RC, plus
    the atom's own class at d = 0."""
    n = len(xyz)
    out = np.zeros((n, NC * NB))

    def add(i, c, d):
        fc = 0.5 * (np.cos(np.pi * d / RC) + 1.0)
        kc = int(np.rint(d / DELTA))
        for k in range(max(0, kc - W), min(NB - 1, kc + W) + 1):
            u = d - k * DELTA
            out[i, c * NB + k] += fc * np.exp(-u * u / (2 * DELTA * DELTA))

    for i in range(n):
        if cls[i] >= 0:
            add(i, cls[i], 0.0)
        d = np.sqrt(((xyz - xyz[i]) ** 2).sum(1))
        for j in np.nonzero((d < RC) & (cls >= 0))[0]:
            if j != i:
                add(i, cls[j], d[j])
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def mlp_forward(p, x):
    z1 = x @ p["W1"].T + p["b1"]
    h1 = silu(z1)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = silu(z2)
    y = h2 @ p["W3"].T + p["b3"]
    return y, (x, z1, h1, z2, h2)


def mlp_grads(p, x, t):
    """gradients of mean over rows of sum over outputs of (y - t)^2"""
    y, (x, z1, h1, z2, h2) = mlp_forward(p, x)
    dy = 2.0 * (y - t) / len(x)
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ p["W3"]) * dsilu(z2)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ p["W2"]) * dsilu(z1)
    g["W1"], g["b1"] = dz1.T @ x, dz1.sum(0)
    return ((y - t) ** 2).sum(1).mean(), g
