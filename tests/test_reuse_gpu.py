"""One context reused across systems and boxes of different sizes.

Between evaluations the context keeps state on the device: the cell counts
are cleared by the scan kernel after it reads them (no memset per
evaluation), the force accumulator by the cell-index kernel, and the
host-buffer path replays a captured graph.  Growing and shrinking the cell
grid on one context (within and beyond its allocation) must give, every
time, exactly the forces and energies of a fresh context.

Tolerance: bit-identical forces and energies (same kernels, same inputs,
integer force sums).
"""
import numpy as np
import pytest
import torch

from protomoladdon_b200 import _lib, water
from protomoladdon_b200.force import (NonbondedCutoffB200SystemForce, PeriodicTopology,
                                      ScalarStructure)

pytestmark = pytest.mark.gpu


def _force(s):
    return NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"],
                                          precision="mixed")


def _host_eval(f, s):
    topo = PeriodicTopology.from_dict(s)
    F = np.zeros_like(s["pos"])
    E = ScalarStructure()
    f.evaluate(topo, s["pos"], F, E)
    return F, np.array([E[0], E[1]])


def _device_eval(f, s):
    topo = PeriodicTopology.from_dict(s)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    frc = torch.zeros_like(pos)
    f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), None, 0, 1)
    torch.cuda.synchronize()
    f.sync()
    return frc.cpu().numpy()


def _scaled(s, factor):
    """The same atoms in a box stretched by `factor` (a different grid)."""
    t = dict(s)
    c = s["origin"]
    t["pos"] = c + (s["pos"] - c) * factor
    t["box"] = s["box"] * factor
    return t


def test_one_context_across_grids():
    small, big = water.water_box(6, rc=8.0, ron=7.0, seed=5), water.water_box(9, rc=8.0,
                                                                             ron=7.0, seed=6)
    sequence = [small, big, small, _scaled(big, 1.15), big, _scaled(small, 1.4), big]
    reused = _force(small)
    for k, s in enumerate(sequence):
        Fh, Eh = _host_eval(reused, s)
        Fd = _device_eval(reused, s)
        fresh = _force(s)
        Fh0, Eh0 = _host_eval(fresh, s)
        Fd0 = _device_eval(fresh, s)
        fresh.close()
        assert np.array_equal(Fh, Fh0), k
        assert np.array_equal(Eh, Eh0), k
        assert np.array_equal(Fd, Fd0), k
        # the two paths (energy and forces-only launches) agree to rounding
        assert np.sqrt(((Fh - Fd) ** 2).sum() / (Fd ** 2).sum()) <= 1e-6, k
    reused.close()
