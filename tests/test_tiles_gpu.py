"""The cluster-pair (tile) mixed kernel (pmb200_set_pair_kernel
PMB200_KERNEL_TILES) against the reference's own outputs (committed
fixtures), the CPU oracle, and the search kernel on the same inputs.

Tolerances (written here, checked below): as the search kernel's -- forces
RMS relative <= 1e-5; cutoff-form Coulomb and LJ energies within 1e-6
relative (the Coulomb energy is summed in FP64 from FP64 distances); Ewald
energies within 1e-6 of the summed pair magnitudes.  Against the search
kernel: the same pair count (the same FP32 pair test) and forces within
1e-6 RMS relative (only the order and grouping of the fixed-point sums
differ).  Two evaluations give bit-identical results (integer sums)."""
import numpy as np
import pytest

from oracle import oracle as O
from protomoladdon_b200 import water
from protomoladdon_b200.force import (EwaldRealB200SystemForce, NonbondedCutoffB200SystemForce,
                                      PeriodicTopology, ScalarStructure)

from .conftest import load_fixture
from .test_ewald_gpu import abs_pair_energy

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def cutoff_eval(d, kernel, energy=True, pos=None, reps=1):
    topo = PeriodicTopology.from_dict(d)
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"])
    f.set_pair_kernel(kernel)
    out = []
    for _ in range(reps):
        F = np.zeros_like(d["pos"])
        E = ScalarStructure()
        if energy:
            f.evaluate(topo, d["pos"] if pos is None else pos, F, E)
        else:  # a forces-only launch (device buffers, flags 0)
            import torch
            p = torch.tensor(d["pos"] if pos is None else pos, dtype=torch.float64,
                             device="cuda:0")
            fr = torch.zeros_like(p)
            f.evaluate_device(topo, p.data_ptr(), fr.data_ptr(), None, 0)
            f.sync()
            F = fr.cpu().numpy()
        out.append((F, E, f.last_pair_count()))
    f.close()
    return out if reps > 1 else out[0]


@pytest.mark.parametrize("fx", ["water423", "water648", "modified648"])
def test_tiles_match_reference_and_search(fx, request):
    d = request.getfixturevalue(fx)
    (F, E, pairs), (F2, E2, _) = cutoff_eval(d, "tiles", reps=2)
    assert np.array_equal(F, F2) and np.array_equal(E.table, E2.table)
    assert rms_rel(F, d["ref_forces"]) <= 1e-5
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 1e-6 * abs(e[0]) and abs(E[1] - e[1]) <= 1e-6 * abs(e[1])
    Fs, Es, ps = cutoff_eval(d, "search")
    assert pairs == ps
    assert rms_rel(F, Fs) <= 1e-6


def test_tiles_forces_only_launch(water648):
    d = water648
    F, _, _ = cutoff_eval(d, "tiles", energy=False)
    Fs, _, _ = cutoff_eval(d, "search", energy=False)
    assert rms_rel(F, d["ref_forces"]) <= 1e-5
    assert rms_rel(F, Fs) <= 1e-6


def test_tiles_41k_box_against_oracle():
    s = water.medium_41k()
    fo, eo, _, _ = O.restate_eval(s, s["pos"], virial_mode=0)
    F, E, pairs = cutoff_eval(s, "tiles")
    assert rms_rel(F, fo) <= 1e-5
    assert abs(E[0] - eo[0]) <= 1e-6 * abs(eo[0]) and abs(E[1] - eo[1]) <= 1e-6 * abs(eo[1])
    po = O.restate_count_pairs(s, s["pos"])
    assert abs(pairs - po) <= 1e-6 * po


@pytest.mark.parametrize("name", ["ewald_water_ref.npz", "ewald_ions_ref.npz"])
@pytest.mark.parametrize("form", ["poly5", "exact"])
def test_tiles_ewald_matches_reference(name, form):
    d = load_fixture(name)
    topo = PeriodicTopology.from_dict(d)
    f = EwaldRealB200SystemForce(float(d["alpha"]), float(d["accuracy"]), erfc=form)
    f.set_pair_kernel("tiles")
    F = np.zeros_like(d["pos"])
    E = ScalarStructure()
    f.evaluate(topo, d["pos"], F, E)
    alpha, rc = f.ewald_info()
    f.close()
    assert rms_rel(F, d[f"{form}_forces"]) <= 1e-5
    e = float(d[f"{form}_energy"])
    assert abs(E[0] - e) <= 1e-6 * abs_pair_energy(d, alpha, rc)
