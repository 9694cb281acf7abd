"""Multi-GPU replicas: one independent periodic system per rank.

A 41k-atom box takes ~0.16 ms per step on one B200, so splitting one box over
GPUs (replicated-data force decomposition with an all-reduce of the force
array, the reference's MPI scheme in protomol/src/protomol/parallel/
Parallel.cpp:122-135; protomoladdon_b200.shard for large systems) would spend
about as long in the collective as in the force.  The headline workload
therefore scales by replicas: each rank integrates its own system and the only
collectives are the timing barrier and a max over ranks.
"""
from __future__ import annotations

DT_FS_DEFAULT = 1.0


def replica_seed(base: int, rank: int) -> int:
    """Seed of rank's replica (distinct systems per rank)."""
    return base + rank


def max_over_ranks(values, dist=None, device=None):
    """Element-wise max of a list of floats over all ranks (identity when
    dist is None).  Every rank must call it, in the same order."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def ns_per_day(sec_per_step: float, dt_fs: float = DT_FS_DEFAULT) -> float:
    return 0.0864 * dt_fs / sec_per_step


def aggregate_ns_per_day(max_ms_per_step: float, world: int, dt_fs: float = DT_FS_DEFAULT) -> float:
    """Whole-job throughput: world replicas, each at the slowest rank's pace."""
    return world * ns_per_day(max_ms_per_step * 1e-3, dt_fs)
