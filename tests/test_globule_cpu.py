"""The seeded synthetic globules that stand in for the benchmark's inputs
(CPU): the geometry and parameter distributions of the benchmark
configurations, and reproducibility from the seed."""
import numpy as np
import pytest

from agbnp3_b200.system import make_globule

RADIUS = {0: 1.7, 1: 1.55, 2: 1.52, 3: 1.8, 4: 1.15}  # C, N, O, S, H


@pytest.fixture(scope="module")
def glob():
    return make_globule(4000, 21)


def test_reproducible_from_seed(glob):
    again = make_globule(4000, 21)
    assert np.array_equal(glob.coords(), again.coords()) and np.array_equal(glob.charge, again.charge)
    other = make_globule(4000, 22)
    assert not np.array_equal(glob.coords(), other.coords())


def test_composition_and_parameters(glob):
    el = glob.element
    heavy = el != 4
    assert heavy.sum() == glob.nheavy and np.array_equal(np.nonzero(~heavy)[0], glob.ihydrogen)
    frac = np.bincount(el[heavy], minlength=4)[:4] / heavy.sum()
    assert np.allclose(frac, [0.62, 0.17, 0.19, 0.02], atol=0.04)
    for e, r in RADIUS.items():
        assert np.all(glob.r[el == e] == r)
    assert abs(glob.charge.sum()) < 1e-9
    assert np.all(glob.igamma[heavy] == 0.117) and np.all(glob.igamma[~heavy] == 0.0)
    assert np.all((glob.ialpha >= -0.09) & (glob.ialpha <= -0.02))
    assert (glob.eps_in, glob.eps_out) == (1.0, 80.0)
    assert glob.stats["density"] == pytest.approx(0.05, rel=1e-6)


def test_bond_geometry(glob):
    xyz, el = glob.coords(), glob.element
    d = np.linalg.norm(xyz[glob.bonds[:, 0]] - xyz[glob.bonds[:, 1]], axis=1)
    hb = (el[glob.bonds[:, 0]] == 4) | (el[glob.bonds[:, 1]] == 4)
    assert np.allclose(d[~hb], 1.53, atol=1e-5) and np.allclose(d[hb], 1.0, atol=1e-5)
    # every hydrogen has exactly one bond, to a heavy atom; at most two per heavy atom
    hcount = np.bincount(glob.bonds[hb].ravel(), minlength=glob.natoms)
    assert np.all(hcount[glob.ihydrogen] == 1)
    assert np.all(np.bincount(np.where(el[glob.bonds[hb, 0]] == 4, glob.bonds[hb, 1], glob.bonds[hb, 0]),
                              minlength=glob.natoms) <= 2)


def test_non_bonded_heavy_distances(glob):
    """heavy atoms that are neither 1-2 nor 1-3 partners stay >= 3.0 A apart"""
    xyz = glob.coords()
    h = np.nonzero(glob.element != 4)[0]
    pos = {int(a): i for i, a in enumerate(h)}
    n = len(h)
    adj = np.zeros((n, n), dtype=bool)
    for a, b in glob.bonds:
        if a in pos and b in pos:
            adj[pos[a], pos[b]] = adj[pos[b], pos[a]] = True
    near = adj | ((adj.astype(np.int32) @ adj.astype(np.int32)) > 0)
    np.fill_diagonal(near, True)
    p = xyz[h]
    d = np.sqrt(((p[:, None, :] - p[None, :, :]) ** 2).sum(-1))
    assert d[~near].min() >= 3.0 - 1e-5
