"""Verlet-skin reuse of the heavy-atom near list (agbnp3_set_nblist_skin).

The skin changes when the candidate pairs are searched, never the list an
evaluation uses: at every step the near list must equal the one the engine
builds without a skin (itself checked pair for pair against the reference's
golden lists in test_gpu_parity.py), and the outputs must equal those of an
instance without a skin up to the order of the double atomic sums (1e-12
relative); candidate searches happen exactly when a heavy atom has moved
half the skin since the last one.
"""
import numpy as np
import pytest

import oracle as O
from conftest import ENERGY_KEYS, load_golden, rms_rel

pytestmark = pytest.mark.gpu

A = pytest.importorskip("agbnp3_b200")


@pytest.fixture(scope="module")
def engine():
    A.initialize()
    yield A
    A.terminate()


def same_results(r, q, tol=1e-12):
    for k in ENERGY_KEYS:
        assert abs(r[k] - q[k]) <= tol * max(abs(q[k]), 1.0), (k, r[k], q[k])
    for k in ("sp", "br", "surf_area", "dgbdr", "dvwdr", "decav", "dehb"):
        assert rms_rel(r[k], q[k]) <= 1e3 * tol, (k, rms_rel(r[k], q[k]))


def same_near_list(a, b):
    ca, la = a.near_list()
    cb, lb = b.near_list()
    assert np.array_equal(ca, cb)
    assert np.array_equal(la, lb)


def ball_steps(rng, n, radius):
    """displacements of length < radius for n atoms"""
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v * (radius * rng.uniform(0.0, 1.0, (n, 1)) ** (1.0 / 3.0))


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_skin_trajectory(engine, prec):
    """A short random walk of the atoms: small steps reuse the candidates,
    a step that takes some atom past half the skin searches them again, and
    every step matches an instance without a skin exactly."""
    s, _ = load_golden("globule2000_hbmix")
    n, nh = s.natoms, s.nheavy
    heavy_ext = s.internal_order()[0][:nh]
    skin = 1.0
    ref = A.Instance(s, precision=prec)
    inst = A.Instance(s, precision=prec)
    rng = np.random.default_rng(3)
    try:
        inst.set_nblist_skin(skin)
        xyz0 = s.coords()
        same_results(inst.ener(xyz0), ref.ener(xyz0))
        same_near_list(inst, ref)
        assert inst.stats()["near_builds"] == 1
        xyz = xyz0.copy()
        builds = 1
        for step in range(6):
            # four steps of at most 0.12 A keep every atom within skin/2 of
            # the first positions; the fifth moves one heavy atom 1.2 A
            if step == 4:
                xyz = xyz.copy()
                xyz[int(heavy_ext[nh // 2])] += np.array([1.2, 0.0, 0.0])
            else:
                xyz = xyz + ball_steps(rng, n, 0.12)
            xyz = s.with_coords(xyz).coords()  # float-rounded, as the oracle takes them
            moved = np.linalg.norm((xyz - xyz0)[heavy_ext], axis=1).max()
            r = inst.ener(xyz)
            q = ref.ener(xyz)
            same_results(r, q)
            same_near_list(inst, ref)
            if moved >= 0.5 * skin:
                builds += 1
                xyz0 = xyz.copy()
            assert inst.stats()["near_builds"] == builds, (step, moved)
        assert builds >= 2
        # against the oracle at the last positions
        Q = O.oracle_eval(s.with_coords(xyz))
        tol = 1e-9 if prec == A.PREC_FP64 else 1e-5
        for k in ENERGY_KEYS:
            assert abs(r[k] - Q[k]) <= tol * max(abs(Q[k]), 10.0), (k, r[k], Q[k])
        # switching the skin off gives the grid search again
        inst.set_nblist_skin(0.0)
        same_results(inst.ener(xyz), q)
        same_near_list(inst, ref)
    finally:
        inst.close()
        ref.close()


def test_skin_capacity_regrowth(engine, monkeypatch):
    """Candidate and near-list buffers that start far too small overflow,
    are regrown, and the evaluation repeated gives the same results."""
    s, _ = load_golden("globule300_shuffled")
    ref = A.Instance(s, precision=A.PREC_FP64)
    monkeypatch.setenv("AGBNP3_CAPACITY_SCALE", "0.001")
    inst = A.Instance(s, precision=A.PREC_FP64)
    try:
        inst.set_nblist_skin(2.0)
        same_results(inst.ener(), ref.ener())
        same_near_list(inst, ref)
        assert inst.stats()["error"] == 0
    finally:
        inst.close()
        ref.close()


def test_skin_batch(engine):
    """A batch with a skin: results as without, over steps that do and do
    not search the candidates again."""
    systems = [load_golden(n)[0] for n in ("globule50", "globule300_shuffled", "globule2000_hbmix")]
    insts = [A.Instance(x, precision=A.PREC_MIXED) for x in systems]
    b0 = A.Batch(insts)
    b1 = A.Batch(insts)
    try:
        b1.set_nblist_skin(0.8)
        xyz = np.concatenate([x.coords() for x in systems])
        rng = np.random.default_rng(7)
        for step in range(4):
            b0.set_coords(xyz)
            b0.ener_resident()
            b1.set_coords(xyz)
            b1.ener_resident()
            r0, r1 = b0.results(), b1.results()
            for k in ENERGY_KEYS:
                assert np.allclose(r1[k], r0[k], rtol=1e-12, atol=1e-9), k
            for k in ("br", "dgbdr", "dvwdr", "decav", "dehb"):
                assert rms_rel(r1[k], r0[k]) <= 1e-9, k
            xyz = xyz + ball_steps(rng, len(xyz), 0.15)
    finally:
        b1.close()
        b0.close()
        for i in insts:
            i.close()
