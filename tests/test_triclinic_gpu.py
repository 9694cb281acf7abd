"""General (non-orthogonal) periodic cells: PeriodicBoundaryConditions with
any basis, whose minimal image is the general branch of
PeriodicBoundaryConditions::minimalDifference
(protomol/src/protomol/topology/PeriodicBoundaryConditions.h:62-67, 95-100:
diff -= e1 rint(e1r.diff) + e2 rint(e2r.diff) + e3 rint(e3r.diff)).

The check is the reference's own pair function over every pair at that image
(NonbondedSimpleFullSystemForce, compiled from the reference sources;
tests/golden/triclinic_ref.npz).  The reference's cell-list force is not:
on general cells it bins atoms into Cartesian cells over the cell's bounding
box and wraps cell indices by that box, so it misses pairs across the sheared
faces (measured: forces off by up to 26 kcal/mol/A), and on some boxes it
stops on an array-bounds assertion.

Tolerances (written here, checked below): FP64 kernel forces RMS relative
<= 1e-12, energies relative <= 1e-11, virials <= 1e-11 relative; mixed
kernel forces RMS relative <= 1e-5, LJ + C1 energies within 2e-3 kcal/mol
(1e-6 of the summed pair magnitudes on this 2,187-atom box), the Ewald
term's energy within 1e-6 of its summed pair magnitudes, virials <= 1e-5.
"""
import numpy as np
import pytest
from scipy.special import erfc

from protomoladdon_b200 import _lib, water
from protomoladdon_b200._lib import PmbError
from protomoladdon_b200.force import (EwaldRealB200SystemForce, NonbondedCutoffB200SystemForce,
                                      PeriodicTopology, ScalarStructure)

from .conftest import load_fixture

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def run(d, precision, pos=None, molvir=True):
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"],
                                       precision=precision)
    F = np.zeros_like(d["pos"])
    E = ScalarStructure(virial=True, molecular_virial=molvir)
    f.evaluate(PeriodicTopology.from_dict(d), d["pos"] if pos is None else pos, F, E)
    f.close()
    return F, E


@pytest.fixture(scope="module")
def tric():
    d = load_fixture("triclinic_ref.npz")
    assert np.count_nonzero(d["box"] - np.diag(np.diag(d["box"]))) > 0  # a general cell
    return d


def test_fp64_matches_reference_all_pairs(tric):
    d = tric
    F, E = run(d, "fp64")
    assert rms_rel(F, d["ref_forces"]) <= 1e-12
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 1e-11 * abs(e[0]) and abs(E[1] - e[1]) <= 1e-11 * abs(e[1])
    v = d["ref_virial"]
    assert np.abs(E.virial_matrix().ravel() - v).max() <= 1e-11 * np.abs(v).max()
    mv = d["ref_molvirial"]
    assert np.abs(E.molvirial_matrix().ravel() - mv).max() <= 1e-11 * np.abs(v).max()


def test_mixed_matches_reference_all_pairs(tric):
    d = tric
    F, E = run(d, "mixed")
    assert rms_rel(F, d["ref_forces"]) <= 1e-5
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 2e-3 and abs(E[1] - e[1]) <= 2e-3
    v = d["ref_virial"]
    assert np.abs(E.virial_matrix().ravel() - v).max() <= 1e-5 * np.abs(v).max()
    mv = d["ref_molvirial"]
    assert np.abs(E.molvirial_matrix().ravel() - mv).max() <= 1e-5 * np.abs(v).max()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_lattice_translations_and_unwrapped_positions(tric, precision):
    """Atoms moved by lattice vectors: the same forces (the cell build wraps
    by fractional coordinates)."""
    d = tric
    e = np.asarray(d["box"])
    rng = np.random.default_rng(5)
    k = rng.integers(-2, 3, size=(len(d["pos"]), 3))
    moved = d["pos"] + k @ e
    F0, _ = run(d, precision, molvir=False)
    F1, _ = run(d, precision, pos=moved, molvir=False)
    tol = 1e-11 if precision == "fp64" else 1e-5
    assert rms_rel(F1, F0) <= tol


def _ewald_brute(d, alpha, rc):
    """Real-space Ewald over all pairs at the reference's minimal image."""
    pos, q = d["pos"], d["qscaled"]
    e = np.asarray(d["box"])
    er = np.linalg.inv(e)  # fractional coordinates: x @ er
    full = {(min(a, b), max(a, b)) for a, b, k in d["excl"] if k == 2}
    n = len(q)
    F = np.zeros_like(pos)
    E = 0.0
    A = 0.0  # sum of the pair energies' magnitudes
    for i in range(n - 1):
        dv = pos[i + 1:] - pos[i]
        dv -= np.rint(dv @ er) @ e
        r2 = (dv ** 2).sum(1)
        js = np.arange(i + 1, n)
        m = r2 <= rc * rc
        m &= np.array([(i, j) not in full for j in js])
        r = np.sqrt(r2[m])
        qq = q[i] * q[js[m]]
        g = erfc(alpha * r) / r
        E += (qq * g).sum()
        A += np.abs(qq * g).sum()
        fr = qq * (g + 2 * alpha / np.sqrt(np.pi) * np.exp(-(alpha * r) ** 2)) / r2[m]
        fv = dv[m] * fr[:, None]
        F[i] -= fv.sum(0)
        np.add.at(F, js[m], fv)
    return F, E, A


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_ewald_real_term_on_a_general_cell(tric, precision):
    d = tric
    alpha = 0.45
    acc = float(np.exp(-(alpha * 6.0) ** 2))  # rc = 6 A
    # erfc itself (the reference's -DUSE_EWALD_EXACT_ERF build), as in the
    # brute force below
    f = EwaldRealB200SystemForce(alpha, acc, precision=precision, erfc="exact")
    F = np.zeros_like(d["pos"])
    E = ScalarStructure()
    f.evaluate(PeriodicTopology.from_dict(d), d["pos"], F, E)
    f.close()
    Fb, Eb, Ab = _ewald_brute(d, alpha, 6.0)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rms_rel(F, Fb) <= tol
    # the mixed Ewald energy is judged on the summed pair magnitudes, as on
    # the orthogonal boxes (tests/test_ewald_gpu.py)
    assert abs(E[0] - Eb) <= (1e-10 * abs(Eb) + 1e-9 if precision == "fp64" else 1e-6 * Ab)


def test_large_sheared_box_mixed_against_fp64():
    """The 41,472-atom benchmark box, sheared: the mixed kernel against the
    FP64 kernel, and Newton's third law."""
    s = water.sheared(water.medium_41k(), 0.25, -0.1, 0.15)
    Fm, Em = run(s, "mixed", molvir=False)
    Fd, Ed = run(s, "fp64", molvir=False)
    assert rms_rel(Fm, Fd) <= 1e-5
    assert abs(Em[1] - Ed[1]) <= 1e-6 * abs(Ed[1])
    rms = np.sqrt((Fd ** 2).sum(1).mean())
    assert np.abs(Fm.sum(0)).max() <= 1e-5 * rms * np.sqrt(len(Fm))


def test_too_narrow_a_general_cell_is_refused(tric):
    """Widths of 12.6-13.4 A for a 6 A cutoff: wider than twice the cutoff,
    but 6 cells of ~2.1 A per axis cannot hold 3 cells on each side of a
    cell plus the cell itself, so the set-up refuses the box (before any
    evaluation: the positions are not rescaled)."""
    d = dict(tric)
    d["box"] = np.asarray(d["box"]) * 0.48
    w = 1.0 / np.linalg.norm(np.linalg.inv(d["box"]).T, axis=1)
    assert (w > 2 * d["rc_lj"]).all() and (w < 2.5 * d["rc_lj"]).all()
    with pytest.raises(PmbError) as ei:
        run(d, "mixed")
    assert ei.value.code == _lib.PMB200_EUNSUPPORTED
