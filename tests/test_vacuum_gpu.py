"""Vacuum boundaries (pmb200_set_vacuum_domain) against the reference's own
vacuum cutoff force on a water droplet (tests/golden/vacuum_ref.npz), and
against itself when atoms sit outside the cell domain or the domain changes.

Tolerances (written here, checked below): FP64 forces RMS relative
<= 1e-12, energies relative <= 1e-11; mixed forces RMS relative <= 1e-5,
energies within 2e-3 kcal/mol, virial within 1e-5 of its largest
component."""
import numpy as np
import pytest

from protomoladdon_b200 import _lib
from protomoladdon_b200._lib import PmbError
from protomoladdon_b200.force import (EwaldRealB200SystemForce, NonbondedCutoffB200SystemForce,
                                      PeriodicTopology, ScalarStructure)

from .conftest import load_fixture

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def drop():
    return load_fixture("vacuum_ref.npz")


def run(d, precision, domain, pos=None):
    topo = PeriodicTopology.from_dict(d)
    topo.domain = domain
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"],
                                       precision=precision)
    F = np.zeros_like(d["pos"])
    E = ScalarStructure(virial=True, molecular_virial=True)
    f.evaluate(topo, d["pos"] if pos is None else pos, F, E)
    f.close()
    return F, E


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_vacuum_matches_reference(drop, precision):
    lo, hi = drop["pos"].min(0) - 1.0, drop["pos"].max(0) + 1.0
    F, E = run(drop, precision, (lo, hi))
    fr, er, vr = drop["ref_forces"], drop["ref_energies"], drop["ref_virial"]
    if precision == "fp64":
        assert rms_rel(F, fr) <= 1e-12
        for k in (0, 1):
            assert abs(E[k] - er[k]) <= 1e-11 * abs(er[k])
        assert np.allclose(E.virial_matrix().ravel(), vr, rtol=1e-11, atol=1e-11 * np.abs(vr).max())
    else:
        assert rms_rel(F, fr) <= 1e-5
        for k in (0, 1):
            assert abs(E[k] - er[k]) <= 2e-3
        assert np.abs(E.virial_matrix().ravel() - vr).max() <= 1e-5 * np.abs(vr).max()
    mvr = drop["ref_molvirial"]
    assert np.abs(E.molvirial_matrix().ravel() - mvr).max() <= 1e-5 * np.abs(mvr).max()


def test_atoms_outside_the_domain_and_small_domains(drop):
    """A domain that covers only the middle of the droplet (atoms outside
    are clamped into boundary cells) and one smaller than the cutoff give the
    same forces as a covering domain."""
    lo, hi = drop["pos"].min(0) - 1.0, drop["pos"].max(0) + 1.0
    F0, E0 = run(drop, "fp64", (lo, hi))
    for dom in ((lo + 6.0, hi - 6.0), (np.full(3, -2.0), np.full(3, 3.0)),
                (lo - 30.0, hi + 30.0)):
        F, E = run(drop, "fp64", dom)
        assert rms_rel(F, F0) <= 1e-12
        assert abs(E[0] - E0[0]) <= 1e-11 * abs(E0[0])


def test_vacuum_refuses_the_ewald_term(drop):
    topo = PeriodicTopology.from_dict(drop)
    topo.domain = (np.full(3, -10.0), np.full(3, 10.0))
    f = EwaldRealB200SystemForce(0.3, 1e-5)
    with pytest.raises(PmbError) as ei:
        f.evaluate(topo, drop["pos"], np.zeros_like(drop["pos"]), ScalarStructure())
    assert ei.value.code == _lib.PMB200_EUNSUPPORTED
    f.close()
