"""pmb200_autotune: the single-context autotuner (cell size, and for mixed
precision the warps per i-cell of the pair kernel) on the 648-atom fixture
boxes, then the tuned context against the reference's own outputs.

Tolerances (written here, checked below): as the untuned kernels -- mixed
forces RMS relative <= 1e-5 and energies within 1e-6 relative of the
reference's (the cutoff-form Coulomb energy is summed from FP64 distances);
FP64 forces RMS relative <= 1e-12, energies relative <= 1e-11.  A second
context with the same workload takes the cached choice (no configuration
timed) and gives bit-identical results."""
import numpy as np
import pytest

from protomoladdon_b200.force import (NonbondedCutoffB200SystemForce, PeriodicTopology,
                                      ScalarStructure)

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def tuned(d, precision):
    import torch
    topo = PeriodicTopology.from_dict(d)
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"],
                                       precision=precision)
    pos = torch.tensor(d["pos"], dtype=torch.float64, device="cuda:0")
    choice = f.autotune(topo, pos.data_ptr(), reps=3)
    F = np.zeros_like(d["pos"])
    E = ScalarStructure(virial=True, molecular_virial=True)
    f.evaluate(topo, d["pos"], F, E)
    grid = f.grid()
    f.close()
    return choice, F, E, grid


@pytest.mark.parametrize("fx", ["water648", "modified648"])
def test_tuned_mixed_context_matches_reference(fx, request):
    d = request.getfixturevalue(fx)
    choice, F, E, grid = tuned(d, "mixed")
    assert choice["warps_per_cell_energy"] in (2, 4, 8)
    assert choice["warps_per_cell_forces"] in (2, 4, 8)
    assert choice["ms_energy"] > 0 and choice["ms_forces"] > 0
    rc = d["rc_alg"]
    # the grid the hint gives: the largest cells of at most the hint, at
    # least a third of the cutoff
    hint = max(choice["cellsize_hint"], rc / 3.0)
    L = np.diag(np.asarray(d["box"])) if np.ndim(d["box"]) == 2 else np.asarray(d["box"])
    assert grid[0] == tuple(int(np.floor(x / hint)) for x in L)
    assert rms_rel(F, d["ref_forces"]) <= 1e-5
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 1e-6 * abs(e[0]) and abs(E[1] - e[1]) <= 1e-6 * abs(e[1])
    v = d["ref_virial"]
    assert np.abs(E.virial_matrix().ravel() - v).max() <= 1e-5 * np.abs(v).max()


def test_cached_choice_is_reused_bit_for_bit(water648):
    c1, F1, E1, g1 = tuned(water648, "mixed")
    c2, F2, E2, g2 = tuned(water648, "mixed")
    assert c2["configurations_timed"] == 0
    for k in ("cellsize_hint", "warps_per_cell_energy", "warps_per_cell_forces"):
        assert c1[k] == c2[k]
    assert g1 == g2
    assert np.array_equal(F1, F2) and np.array_equal(E1.table, E2.table)


def test_tuned_fp64_context_matches_reference(water648):
    d = water648
    choice, F, E, _ = tuned(d, "fp64")
    assert choice["warps_per_cell_forces"] == 0 and choice["warps_per_cell_energy"] == 0
    assert rms_rel(F, d["ref_forces"]) <= 1e-12
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 1e-11 * abs(e[0]) and abs(E[1] - e[1]) <= 1e-11 * abs(e[1])


def test_tuning_on_the_legacy_default_stream():
    """The tuner times graph replays of an evaluation; on a stream that
    cannot be captured (the legacy default stream, handle 0x1) it times
    direct launches instead, with the same result structure.  (A fresh box
    size, so that no cached choice is taken.)"""
    import torch
    from protomoladdon_b200 import water
    d = water.water_box(7, rc=8.0, ron=7.0, seed=21)
    topo = PeriodicTopology.from_dict(d)
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"])
    pos = torch.tensor(d["pos"], dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    choice = f.autotune(topo, pos.data_ptr(), reps=2, stream=0x1)
    assert choice["configurations_timed"] > 0 and choice["ms_energy"] > 0.0
    F = np.zeros_like(d["pos"])
    E = ScalarStructure()
    f.evaluate(topo, d["pos"], F, E)
    f.close()
    from oracle import oracle as O
    fo, eo, _, _ = O.restate_eval(d, d["pos"], virial_mode=0)
    assert rms_rel(F, fo) <= 1e-5
