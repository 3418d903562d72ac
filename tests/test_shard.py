"""Row sharding of one instance (agbnp3_shard).

A run here has one GPU, so the ranks of a sharded evaluation are emulated
by several instances of the same system on that GPU, each holding one
rank's share of the pair-pass work items and evaluated segment by segment;
between segments the host adds the ranks' partial sums (what the NCCL
all-reduce does on a multi-GPU run) and hands them back.  No kernel waits
for another instance.  Every rank must then hold the unsharded outputs, up
to the order of the double sums (1e-11 relative).  The NCCL path itself
(the all-reduces captured in the evaluation graph) runs with a one-rank
communicator.
"""
import os

import numpy as np
import pytest

from conftest import ENERGY_KEYS, load_golden, rms_rel

pytestmark = pytest.mark.gpu

A = pytest.importorskip("agbnp3_b200")


@pytest.fixture(scope="module")
def engine():
    A.initialize()
    yield A
    A.terminate()


def same_results(r, q, tol=1e-11):
    for k in ENERGY_KEYS:
        assert abs(r[k] - q[k]) <= tol * max(abs(q[k]), 1.0), (k, r[k], q[k])
    for k in ("sp", "br", "surf_area", "dgbdr", "dvwdr", "decav", "dehb"):
        assert rms_rel(r[k], q[k]) <= 100 * tol, (k, rms_rel(r[k], q[k]))


def emulated_evaluation(ranks, xyz):
    for inst in ranks:
        inst.set_coords(xyz)
    for seg in range(4):
        for inst in ranks:
            inst.shard_segment(seg)
        if seg < 3:
            total = sum(inst.shard_sums(seg) for inst in ranks)
            for inst in ranks:
                inst.set_shard_sums(seg, total)
    return [inst.results() for inst in ranks]


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("nranks", [2, 3])
def test_emulated_ranks(engine, prec, nranks):
    s, _ = load_golden("globule2000_hbmix")
    ref = A.Instance(s, precision=prec)
    ranks = [A.Instance(s, precision=prec) for _ in range(nranks)]
    try:
        xyz = s.coords()
        q = ref.ener(xyz)
        for r, inst in enumerate(ranks):
            inst.ener(xyz)  # sizes the buffers (an unsharded evaluation)
            inst.shard(r, nranks)
        # a rank's own share alone is not the whole: its partial sums differ
        ranks[0].set_coords(xyz)
        ranks[0].shard_segment(0)
        part = ranks[0].shard_sums(0)
        full = ref.atom_array(19)  # descreening sums of the unsharded run
        assert not np.allclose(part, full)
        for step in range(2):
            for res in emulated_evaluation(ranks, xyz):
                same_results(res, q)
            xyz = s.with_coords(xyz + np.random.default_rng(step).normal(0.0, 0.05, xyz.shape)).coords()
            q = ref.ener(xyz)
        # undoing the sharding gives whole evaluations again
        ranks[1].shard(0, 1)
        same_results(ranks[1].ener(xyz), q)
    finally:
        for inst in ranks:
            inst.close()
        ref.close()


def test_nccl_single_rank(engine):
    """A one-rank NCCL communicator: the all-reduces sit in the captured
    evaluation graph and leave the sums as they are."""
    os.environ.setdefault("NCCL_SOCKET_IFNAME", "lo")
    s, _ = load_golden("globule2000_hbmix")
    ref = A.Instance(s, precision=A.PREC_MIXED)
    inst = A.Instance(s, precision=A.PREC_MIXED)
    try:
        uid = A.shard_unique_id()
        assert len(uid) == 128
        inst.shard(0, 1, uid)
        xyz = s.coords()
        for step in range(3):
            same_results(inst.ener(xyz), ref.ener(xyz))
            inst.set_coords(xyz)
            inst.ener_resident()
            same_results(inst.results(), ref.results())
            xyz = s.with_coords(xyz + 0.05).coords()
        inst.shard(0, 1)
        same_results(inst.ener(xyz), ref.ener(xyz))
    finally:
        inst.close()
        ref.close()


def test_shard_with_skin_and_errors(engine):
    """Sharding composes with the near-list skin; bad ranks and tuning a
    sharded instance are refused."""
    s, _ = load_golden("globule300_shuffled")
    ref = A.Instance(s, precision=A.PREC_FP64)
    ranks = [A.Instance(s, precision=A.PREC_FP64) for _ in range(2)]
    try:
        xyz = s.coords()
        q = ref.ener(xyz)
        for r, inst in enumerate(ranks):
            inst.set_nblist_skin(1.0)
            inst.ener(xyz)
            inst.shard(r, 2)
        for step in range(3):
            for res in emulated_evaluation(ranks, xyz):
                same_results(res, q)
            xyz = s.with_coords(xyz + np.random.default_rng(10 + step).normal(0.0, 0.1, xyz.shape)).coords()
            q = ref.ener(xyz)
        with pytest.raises(A.AGBNPError):
            ranks[0].shard(2, 2)
        with pytest.raises(A.AGBNPError):
            ranks[0].autotune()
        with pytest.raises(A.AGBNPError):
            ranks[0].shard_segment(4)
    finally:
        for inst in ranks:
            inst.close()
        ref.close()
