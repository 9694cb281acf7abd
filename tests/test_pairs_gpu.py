"""The other periodic cutoff registrations (OneAtomPair / OneAtomPairTwo with
C1, C2, Cn, ComplimentCnCn switches; pmb200_create_pair) against the reference's own
outputs (tests/golden/pairs_ref.npz, written by make_golden.py from the
reference compiled from its sources).

Tolerances (written here, checked below): FP64 kernel forces RMS relative
<= 1e-12, energies relative <= 1e-11 -- <= 1e-10 for both when a Cn or
ComplimentCnCn switch is involved: the reference sums their polynomial in power form, whose terms
cancel to ~1e-4 of their size at orders 4-6, so its own rounding is
~1e-12..1e-11 while the kernel uses the positive Bernstein form; mixed kernel forces RMS relative
<= 1e-5; energies within 1e-6 of the sum over pairs of |E_pair| (bounded
here by the unswitched |q_i q_j / r| and |A r^-12| + |B r^-6| within the
cutoff: the Coulomb terms cancel to ~2% of their magnitudes on this box, and
the per-pair FP32 switch values of this form carry no compensated energy
sums); virial within 1e-5 of its largest component."""
import numpy as np
import pytest

from protomoladdon_b200.force import NonbondedCutoffB200PairForce, PeriodicTopology, ScalarStructure

from .conftest import load_fixture

pytestmark = pytest.mark.gpu

CASES = ["c2_c2", "c2_cn", "cn_cn", "lj_c1", "lj_cn", "coul_c2", "coul_cn",
         "cm_cm", "lj_cm", "coul_cm", "cm5_c1"]
NAMES = {1: "C1", 2: "C2", 3: "Cn", 4: "ComplimentCnCn"}


@pytest.fixture(scope="module")
def fx():
    return load_fixture("pairs_ref.npz")


def magnitudes(d, rc):
    """(sum |q_i q_j / r|, sum |A r^-12| + |B r^-6|) over non-excluded pairs
    within rc (numpy, minimum image)."""
    pos, q, box = d["pos"], d["qscaled"], np.asarray(d["box"], float)
    typ, lj = d["type"], np.asarray(d["lj"]).reshape(-1, 4)
    nt = int(round(np.sqrt(lj.shape[0])))
    n = len(q)
    full = np.zeros((n, n), bool)
    for a, b, k in np.asarray(d["excl"]).reshape(-1, 3):
        if k == 2:
            full[a, b] = full[b, a] = True
    mc = ml = 0.0
    for i in range(n - 1):
        dv = pos[i + 1:] - pos[i]
        dv -= box * np.rint(dv / box)
        r = np.sqrt((dv ** 2).sum(1))
        m = (r <= rc) & ~full[i, i + 1:]
        rm = r[m]
        mc += np.abs(q[i] * q[i + 1:][m] / rm).sum()
        p = lj[typ[i] * nt + typ[i + 1:][m]]
        ml += (np.abs(p[:, 0]) * rm ** -12 + np.abs(p[:, 1]) * rm ** -6).sum()
    return mc, ml


def spec(a):
    return None if a[0] == 0 else (NAMES[int(a[0])], *[float(x) for x in a[1:]])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", CASES)
def test_switch_policies_match_reference(fx, case, precision):
    f = NonbondedCutoffB200PairForce(spec(fx[f"{case}_lj"]), spec(fx[f"{case}_coul"]), 8.0,
                                     precision=precision)
    topo = PeriodicTopology.from_dict(fx)
    F = np.zeros_like(fx["pos"])
    E = ScalarStructure(virial=True, molecular_virial=True)
    f.evaluate(topo, fx["pos"], F, E)
    f.close()
    fr, er = fx[f"{case}_forces"], fx[f"{case}_energies"]
    err = float(np.sqrt(((F - fr) ** 2).sum() / (fr ** 2).sum()))
    vr, mvr = fx[f"{case}_virial"], fx[f"{case}_molvirial"]
    if precision == "fp64":
        cn = "cn" in case or "cm" in case  # power-form polynomials in the reference
        assert err <= (1e-10 if cn else 1e-12), err
        for k in (0, 1):
            assert abs(E[k] - er[k]) <= (1e-10 if cn else 1e-11) * max(1.0, abs(er[k]))
        assert np.allclose(E.virial_matrix().ravel(), vr, rtol=1e-11, atol=1e-11 * np.abs(vr).max())
    else:
        assert err <= 1e-5, err
        mags = magnitudes(fx, 8.0)
        for k in (0, 1):
            assert abs(E[k] - er[k]) <= 1e-6 * mags[k] + 1e-9, (k, E[k], er[k], mags[k])
        assert np.abs(E.virial_matrix().ravel() - vr).max() <= 1e-5 * np.abs(vr).max()
    assert np.abs(E.molvirial_matrix().ravel() - mvr).max() <= 1e-5 * max(np.abs(mvr).max(), 1.0)
