"""One system's force evaluation split over the ranks of a process group,
one GPU per rank: the replicated-data decomposition of the reference's
parallel evaluation (NonbondedCutoffSystemForce::parallelEvaluate,
protomol/src/protomol/force/nonbonded/NonbondedCutoffSystemForce.h:57-77,
which deals contiguous runs of cell pairs to the MPI ranks and sums the
forces).  Every rank holds the whole topology and the same positions; rank r
evaluates its run of i-cells into an int64 fixed-point accumulator
(pmb200_shard_eval_device), the accumulators are summed with one integer
all-reduce (exact, so the forces are bit-identical to a one-GPU evaluation
whatever the reduction order), and every rank converts the sum
(pmb200_shard_finalize).  Energies and virials are summed with a second,
20-double all-reduce.
"""
from __future__ import annotations


def _stream_handle(t):
    """The current stream of t's device as a raw handle for libpmb200 (the
    legacy default stream is passed as 0x1, since NULL would select the
    context's own stream); None for CPU tensors."""
    if not t.is_cuda:
        return None
    import torch
    h = torch.cuda.current_stream(t.device).cuda_stream
    return h if h else 1


def sharded_evaluate(force, topo, pos, forces, out=None, flags=0, group=None, dist=None):
    """Adds this evaluation's forces to ``forces`` ((n, 3) float64, on every
    rank) from identical ``pos`` on every rank of ``group``; when ``flags``
    ask for energies / virials, ``out`` (20 float64) receives their totals
    (overwritten).  Collective: every rank of the group must call it."""
    import torch
    if dist is None:
        import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    n = int(pos.shape[0])
    facc = torch.empty(3 * n, dtype=torch.int64, device=pos.device)
    part = torch.zeros(20, dtype=torch.float64, device=pos.device) if flags else None
    stream = _stream_handle(pos)
    force.shard_eval_device(topo, pos.data_ptr(), rank, world, facc.data_ptr(),
                            part.data_ptr() if part is not None else None, flags, stream)
    dist.all_reduce(facc, group=group)  # integer sum: exact in any order
    if part is not None:
        dist.all_reduce(part, group=group)
        out.copy_(part)
    force.shard_finalize(facc.data_ptr(), forces.data_ptr(), stream)
