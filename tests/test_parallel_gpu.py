"""The reference's parallel decomposition through the C ABI
(pmb200_eval_cells): SystemForce::parallelEvaluate on each of N ranks in the
reference's static mode (block i of numberOfBlocks to rank i mod N, block i
covering the cells [n i / count, n (i + 1) / count)), summed as
Parallel::reduce sums the ranks, gives evaluate()'s forces, energies and
virials.

Tolerance (written here, checked below): 1e-12 relative -- every pair is
evaluated by exactly one rank with the same arithmetic; only the host's FP64
additions of the ranks' shares differ from one evaluation's.
"""
import numpy as np
import pytest

from protomoladdon_b200 import water
from protomoladdon_b200.force import (EwaldRealB200SystemForce, NonbondedCutoffB200SystemForce,
                                      PeriodicTopology, ScalarStructure)

pytestmark = pytest.mark.gpu


def _make(kind, s, precision):
    if kind == "cutoff":
        return NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"],
                                              precision=precision)
    return EwaldRealB200SystemForce(0.35, float(np.exp(-(0.35 * 8.0) ** 2)),
                                    precision=precision)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("kind", ["cutoff", "ewald"])
def test_ranks_sum_to_one_evaluation(kind, precision):
    s = water.water_box(9, rc=8.0, ron=7.0, seed=33)
    topo = PeriodicTopology.from_dict(s)
    import torch
    f = _make(kind, s, precision)
    F1 = np.zeros_like(s["pos"])
    E1 = ScalarStructure(virial=True, molecular_virial=True)
    f.evaluate(topo, s["pos"], F1, E1)
    # the forces of one evaluation in FP64 (the host-buffer call of a mixed
    # context returns them in FP32)
    # (an energy launch, as the shares are: the same task split)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda:0")
    frc = torch.zeros_like(pos)
    out = torch.zeros(20, dtype=torch.float64, device="cuda:0")
    f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), out.data_ptr(), 1)
    f.sync()
    F1 = frc.cpu().numpy()
    blocks = f.number_of_blocks(topo)
    assert blocks == int(np.prod(f.grid()[0]))
    for nranks in (1, 2, 3, 7, blocks + 3):  # the last: some ranks get no block
        F = np.zeros_like(s["pos"])
        E = ScalarStructure(virial=True, molecular_virial=True)
        for r in range(nranks):
            f.parallel_evaluate(topo, s["pos"], F, E, r, nranks)
        scale = np.abs(F1).max()
        assert np.abs(F - F1).max() <= 1e-12 * scale, nranks
        t1 = E1.table
        assert np.allclose(E.table, t1, rtol=1e-12, atol=1e-12 * np.abs(t1).max()), nranks
    f.close()


def test_cell_range_arguments_are_checked():
    from protomoladdon_b200._lib import PmbError
    s = water.small_648()
    topo = PeriodicTopology.from_dict(s)
    f = _make("cutoff", s, "mixed")
    n = f.number_of_blocks(topo)
    F = np.zeros_like(s["pos"])
    E = ScalarStructure()
    for lo, hi in ((-1, 2), (3, 2), (0, n + 1)):
        with pytest.raises(PmbError):
            f.evaluate_cells(topo, s["pos"], F, E, lo, hi)
    f.evaluate_cells(topo, s["pos"], F, E, 2, 2)  # an empty share adds nothing
    assert not F.any() and E[0] == 0.0 and E[1] == 0.0
    f.close()
