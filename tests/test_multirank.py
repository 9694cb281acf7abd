"""Multi-rank replicas on CPU with the gloo backend (world size 2): each
rank evaluates its own seeded replica with the oracle, the ranks agree on
the max step time, and rank 0 reports the aggregate."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from protomoladdon_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        from oracle import oracle as O
        from protomoladdon_b200 import water
        s = water.water_box(5, rc=7.0, ron=6.0, seed=replicas.replica_seed(1234, rank))
        f, e, _, _ = O.restate_eval(s, s["pos"], 0)
        fake_ms = 0.2 + 0.1 * rank  # this rank's step time
        dist.barrier()
        (mx,) = replicas.max_over_ranks([fake_ms], dist)
        agg = replicas.aggregate_ns_per_day(mx, world)
        out[rank] = (float(e[0]), float(np.abs(f.sum(0)).max()), mx, agg)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_replicas():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    r0, r1 = out[0], out[1]
    assert r0[0] != r1[0]                       # distinct replicas
    assert r0[1] < 1e-9 and r1[1] < 1e-9        # each replica's forces sum to zero
    assert r0[2] == r1[2] and abs(r0[2] - 0.3) < 1e-12  # every rank sees the slowest step
    assert abs(r0[3] - 2 * 0.0864 / 0.3e-3) < 1e-9


def test_single_process_helpers():
    assert replicas.max_over_ranks([1.0, 2.0]) == [1.0, 2.0]
    assert abs(replicas.aggregate_ns_per_day(0.2, 1) - 432.0) < 1e-9


class _ToyShardForce:
    """Stands in for a libpmb200 context on CPU: shard s of S takes the pairs
    (i < j) with i % S == s of a toy 1/r^2 pair force and writes them as
    int64 fixed-point sums, the contract of pmb200_shard_eval_device; the
    finalize adds the summed accumulator, converted, to the forces."""
    SCALE = 2.0 ** 32

    def __init__(self, pos):
        self.pos = pos

    def contributions(self, shard, nshards):
        n = len(self.pos)
        acc = np.zeros((3, n), dtype=np.int64)
        for i in range(shard, n, nshards):
            for j in range(i + 1, n):
                d = self.pos[j] - self.pos[i]
                f = np.rint(d / np.dot(d, d) ** 1.5 * self.SCALE).astype(np.int64)
                acc[:, j] += f
                acc[:, i] -= f
        return acc

    def shard_eval_device(self, topo, pos_ptr, shard, nshards, facc_ptr, out_ptr, flags,
                          stream):
        import ctypes
        n = len(self.pos)
        dst = np.ctypeslib.as_array((ctypes.c_int64 * (3 * n)).from_address(facc_ptr))
        dst[:] = self.contributions(shard, nshards).reshape(-1)
        if out_ptr:
            o = np.ctypeslib.as_array((ctypes.c_double * 20).from_address(out_ptr))
            o[:] = 0.0
            o[0] = float(shard + 1)

    def shard_finalize(self, facc_ptr, force_ptr, stream):
        import ctypes
        n = len(self.pos)
        acc = np.ctypeslib.as_array((ctypes.c_int64 * (3 * n)).from_address(facc_ptr))
        frc = np.ctypeslib.as_array((ctypes.c_double * (3 * n)).from_address(force_ptr))
        frc.reshape(n, 3)[:] += acc.reshape(3, n).T / self.SCALE


def _shard_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import torch
        from protomoladdon_b200.shard import sharded_evaluate
        rng = np.random.default_rng(7)
        pos = rng.uniform(0.0, 10.0, (40, 3))  # the same positions on every rank
        toy = _ToyShardForce(pos)
        forces = torch.zeros((40, 3), dtype=torch.float64)
        res = torch.zeros(20, dtype=torch.float64)
        sharded_evaluate(toy, None, torch.tensor(pos), forces, res, flags=1)
        full = toy.contributions(0, 1).T / _ToyShardForce.SCALE
        out[rank] = (forces.numpy().copy(), full, float(res[0]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_sharded_evaluation():
    """sharded_evaluate: each rank's shard accumulator, one integer all-reduce,
    then the finalize: every rank holds the one-shard forces bit for bit and
    the summed energies."""
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_shard_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    (f0, full, e0), (f1, _, e1) = out[0], out[1]
    assert np.array_equal(f0, f1) and np.array_equal(f0, full)
    assert e0 == e1 == 3.0
