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
