"""The multi-rank host logic of the benchmark, run as two gloo ranks on CPU:
each rank builds its own workload (different seeds, no shared data), the
ranks agree on the maximum device time, and the whole-job throughput is
world * units / max time."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from agbnp3_b200 import make_globule
from agbnp3_b200.shard import max_over_ranks, rank_seed, throughput


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = make_globule(400, rank_seed(7, rank))
        fake_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        m = max_over_ranks(fake_ms, world)
        out[rank] = (float(s.x.sum()), m, throughput(3, m / 1e3, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        r0, r1 = out[0], out[1]
    assert r0[0] != r1[0]                     # independent conformations per rank
    assert r0[1] == r1[1] == 15.0             # both ranks see the slowest rank's time
    assert r0[2] == pytest.approx(2 * 3 / 0.015)


def test_rank_zero_matches_single_gpu_run():
    assert rank_seed(11, 0) == 11
    a, b = make_globule(300, rank_seed(11, 0)), make_globule(300, 11)
    assert np.array_equal(a.x, b.x)


class _FakeInstance:
    """Records the agbnp3_shard call a rank would make."""

    def __init__(self):
        self.calls = []

    def shard(self, rank, nranks, uid):
        self.calls.append((rank, nranks, uid))


def _shard_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from agbnp3_b200.shard import shard_instance
        made = []

        def make_id():  # only rank 0 may make the communicator's id
            made.append(rank)
            return os.urandom(128)

        inst = _FakeInstance()
        r, w = shard_instance(inst, make_id=make_id)
        out[rank] = (r, w, inst.calls, made)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_shard_instance_id_exchange():
    """Row sharding of one instance: rank 0 alone makes the NCCL unique id,
    every rank joins with that same id, its own rank and the world size."""
    world = 2
    port = 30500 + os.getpid() % 1000
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_shard_worker, args=(world, port, out), nprocs=world, join=True)
        res = [out[0], out[1]]
    for rank, (r, w, calls, made) in enumerate(res):
        assert (r, w) == (rank, world)
        assert len(calls) == 1 and calls[0][:2] == (rank, world)
        assert made == ([0] if rank == 0 else [])
    assert res[0][2][0][2] == res[1][2][0][2] and len(res[0][2][0][2]) == 128
