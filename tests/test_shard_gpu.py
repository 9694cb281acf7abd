"""Force decomposition (pmb200_shard_eval_device / pmb200_shard_finalize) on
one GPU: the shards of one evaluation, run one after another and summed as an
integer all-reduce would sum them, give the forces of a single evaluation.

Tolerances (written here, checked below):
* forces: bit-identical to pmb200_eval_device (the same cells, stencil split
  and staging per shard; integer sums);
* energies and virials (sums of the shards' FP64 partials): within 1e-12
  relative of the single evaluation.
"""
import numpy as np
import pytest
import torch

from protomoladdon_b200 import _lib, water
from protomoladdon_b200.force import (EwaldRealB200SystemForce, NonbondedCutoffB200SystemForce,
                                      PeriodicTopology)

pytestmark = pytest.mark.gpu


def _force(kind, s):
    if kind == "cutoff":
        return NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"])
    return EwaldRealB200SystemForce(0.35, float(np.exp(-(0.35 * 8.0) ** 2)))


def _single(f, topo, pos, flags):
    frc = torch.zeros_like(pos)
    out = torch.zeros(20, dtype=torch.float64, device="cuda")
    f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), out.data_ptr(), flags, 1)
    torch.cuda.synchronize()
    f.sync()
    return frc.cpu().numpy(), out.cpu().numpy()


def _sharded(f, topo, pos, flags, nshards):
    n = pos.shape[0]
    total = torch.zeros(3 * n, dtype=torch.int64, device="cuda")
    out = torch.zeros(20, dtype=torch.float64, device="cuda")
    for s in range(nshards):
        facc = torch.full((3 * n,), 12345, dtype=torch.int64, device="cuda")  # overwritten
        part = torch.full((20,), 7.0, dtype=torch.float64, device="cuda")
        f.shard_eval_device(topo, pos.data_ptr(), s, nshards, facc.data_ptr(),
                            part.data_ptr() if flags else None, flags, 1)
        total += facc
        if flags:
            out += part
    frc = torch.zeros_like(pos)
    f.shard_finalize(total.data_ptr(), frc.data_ptr(), 1)
    torch.cuda.synchronize()
    f.sync()
    return frc.cpu().numpy(), out.cpu().numpy()


@pytest.mark.parametrize("kind", ["cutoff", "ewald"])
@pytest.mark.parametrize("flags", [0, _lib.PMB200_ENERGY | _lib.PMB200_VIRIAL])
def test_shards_sum_to_one_evaluation(kind, flags):
    s = water.water_box(9, rc=8.0, ron=7.0, seed=21)
    topo = PeriodicTopology.from_dict(s)
    f = _force(kind, s)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    F1, o1 = _single(f, topo, pos, flags)
    ncell = int(np.prod(f.grid()[0]))
    for nshards in (2, 3, 7, ncell + 2):  # the last: some shards hold no cell
        F2, o2 = _sharded(f, topo, pos, flags, nshards)
        assert np.array_equal(F1, F2), nshards
        if flags:
            assert np.allclose(o2[:11], o1[:11], rtol=1e-12, atol=1e-12 * np.abs(o1[:11]).max())
    f.close()


def test_shard_arguments_are_checked():
    s = water.small_648()
    topo = PeriodicTopology.from_dict(s)
    f = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"])
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    facc = torch.zeros(3 * s["n"], dtype=torch.int64, device="cuda")
    for shard, nshards in ((2, 2), (-1, 2), (0, 0)):
        with pytest.raises(_lib.PmbError) as ei:
            f.shard_eval_device(topo, pos.data_ptr(), shard, nshards, facc.data_ptr())
        assert ei.value.code == _lib.PMB200_EINVAL
    f.close()
    g = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"],
                                       precision="fp64")
    with pytest.raises(_lib.PmbError) as ei:
        g.shard_eval_device(topo, pos.data_ptr(), 0, 2, facc.data_ptr())
    assert ei.value.code == _lib.PMB200_EUNSUPPORTED
    g.close()
