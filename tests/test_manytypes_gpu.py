"""More Lennard-Jones types than the mixed kernel stages in shared memory
(16): the 648-atom water box spread over a 30-type table (24 types used, the
rest only in the table, as in a force-field parameter file), with the H-H
pair of each water modified (A14/B14, Coulomb scaling 0.5).  The reference's
own forces (tests/golden/manytypes_ref.npz, from the reference compiled from
its sources) and the oracle on the same inputs are the checks.

Tolerances (written here, checked below): FP64 kernel forces RMS relative
<= 1e-12, energies relative <= 1e-11; mixed kernel forces RMS relative
<= 1e-5, energies within 1e-6 of the summed pair magnitudes (2e-3 kcal/mol
on this box), virial relative <= 1e-5.
"""
import numpy as np
import pytest

from oracle import oracle as O
from protomoladdon_b200 import water
from protomoladdon_b200.force import (NonbondedCutoffB200SystemForce, PeriodicTopology,
                                      ScalarStructure)

from .conftest import load_fixture

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def run(d, precision, pos=None):
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"],
                                       precision=precision)
    F = np.zeros_like(d["pos"])
    E = ScalarStructure(virial=True, molecular_virial=True)
    f.evaluate(PeriodicTopology.from_dict(d), d["pos"] if pos is None else pos, F, E)
    f.close()
    return F, E


@pytest.fixture(scope="module")
def manytypes():
    return load_fixture("manytypes_ref.npz")


def test_fixture_has_more_types_than_shared_memory_holds(manytypes):
    assert manytypes["lj"].shape[0] == 30 and np.unique(manytypes["type"]).size >= 20


def test_fp64_matches_reference(manytypes):
    d = manytypes
    F, E = run(d, "fp64")
    assert rms_rel(F, d["ref_forces"]) <= 1e-12
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 1e-11 * abs(e[0]) and abs(E[1] - e[1]) <= 1e-11 * abs(e[1])
    assert np.allclose(E.virial_matrix().ravel(), d["ref_virial"], rtol=1e-11, atol=1e-9)


def test_mixed_matches_reference(manytypes):
    d = manytypes
    F, E = run(d, "mixed")
    assert rms_rel(F, d["ref_forces"]) <= 1e-5
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 2e-3 and abs(E[1] - e[1]) <= 2e-3
    v = d["ref_virial"]
    assert np.abs(E.virial_matrix().ravel() - v).max() <= 1e-5 * np.abs(v).max()
    mv = d["ref_molvirial"]
    assert np.abs(E.molvirial_matrix().ravel() - mv).max() <= 1e-5 * np.abs(v).max()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_larger_box_many_types_vs_oracle(precision):
    """A 5,184-atom box over 40 types against the oracle (unwrapped, shifted
    positions)."""
    s = water.many_types(water.water_box(12, rc=9.0, ron=8.0, seed=11), n_o_types=20,
                         n_h_types=14, n_unused=6, seed=3)
    pos = s["pos"] + np.array([11.5, -30.25, 7.0])
    fo, eo, vo, _ = O.restate_eval(s, pos, virial_mode=1)
    F, E = run(s, precision, pos=pos)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rms_rel(F, fo) <= tol
    assert np.abs(E.virial_matrix().ravel() - vo).max() <= max(tol, 1e-11) * np.abs(vo).max()
