"""The tabulated Lennard-Jones registrations, OneAtomPair<BC,
UniversalSwitchingFunction, LennardJonesTableForce<S, 7, Real>> with S = C2,
Cn, ComplimentCnCn (NonbondedCutoffForceModule.cpp:67-72 periodic, 121-126
vacuum), against the reference's own outputs (tests/golden/ljtable_*_ref.npz,
written by make_golden.py --ljtable-only from the reference compiled from its
sources).

CPU: the numpy restatement of the table (oracle/ljtable.py) against those
fixtures, the table's grid and hash, the force ids.  GPU: the FP64 kernel,
which reads the same table, and the mixed kernel, which evaluates the switched
LJ the table approximates.

Tolerances (written here, checked below):
* oracle vs reference: forces RMS relative <= 1e-13 with a C2 switch, <= 1e-10
  with Cn / ComplimentCnCn (the switch polynomial in power form cancels to
  ~1e-4 of its terms, and a switch that starts at 0 leaves net forces ~1e-3
  of the pair forces); energies relative <= 1e-13 / 1e-10.
* FP64 kernel vs reference: forces RMS relative <= 1e-12 (C2) / 1e-10 (Cn,
  ComplimentCnCn, whose switch values the table holds from the kernel's
  Bernstein form); energies relative <= 1e-11 / 1e-10; virial within 1e-11
  / 1e-10 of its largest component.
* mixed kernel vs reference: forces RMS relative <= 1e-5 (the FP32 pair
  arithmetic plus the table's own interpolation error, measured at 2.9e-6
  RMS on these boxes); energies within 1e-6 of the sum over pairs of
  |A r^-12| + |B r^-6| plus 1e-7 of |E| for the interpolation; virial within
  1e-5 of its largest component.
"""
import ctypes

import numpy as np
import pytest

from oracle import ljtable as LT
from protomoladdon_b200 import _lib
from protomoladdon_b200.force import NonbondedCutoffB200PairForce, PeriodicTopology, ScalarStructure

from .conftest import load_fixture

NAMES = {2: "C2", 3: "Cn", 4: "ComplimentCnCn"}
FILES = {"water": ["t_c2", "t_cn", "t_cm"], "modified": ["t_c2"],
         "vacuum": ["t_c2", "t_cn", "t_cm"]}
CASES = [(f, c) for f, cs in FILES.items() for c in cs]


@pytest.fixture(scope="module")
def fx():
    return {f: load_fixture(f"ljtable_{f}_ref.npz") for f in FILES}


def spec(a):
    return (NAMES[int(a[0])], *[float(x) for x in a[1:]])


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


# ---- CPU: the restatement and the grid ------------------------------------
@pytest.mark.parametrize("fname,case", CASES)
def test_oracle_table_matches_reference(fx, fname, case):
    d = fx[fname]
    sw = spec(d[f"{case}_lj"])
    T = LT.LJTable(sw[0], sw[1:])
    F, E = LT.all_pairs(d, d["pos"], T, periodic=fname != "vacuum")
    tol = 1e-13 if sw[0] == "C2" else 1e-10
    assert rms_rel(F, d[f"{case}_forces"]) <= tol
    er = d[f"{case}_energies"]
    assert er[0] == 0.0
    assert abs(E - er[1]) <= tol * abs(er[1])


def test_table_grid_and_hash():
    """rc 8: 11 octaves of r^2 from 1/16 to 128, 128 intervals each; the
    hash of a grid point's r^2 is its index; r^2 below 1/16 and beyond the
    grid clamp to the ends with dt = 0; within an interval dt is r^2 minus
    the interval's start."""
    T = LT.LJTable("C2", (6.5, 8.0, 0, 0))
    assert T.t.shape == (11 * 128 + 1, 8)
    assert T.last == 11 * 128
    pts = np.array([0.0625 * 2.0 ** (i // 128) * (1 + (i % 128) / 128) for i in range(T.last + 1)])
    i, dt = T.index(pts)
    assert np.array_equal(i, np.arange(T.last + 1)) and np.all(dt == 0)
    i, dt = T.index(np.array([0.01, 0.0625 * (1 + 0.5 / 128), 200.0]))
    assert list(i) == [0, 0, T.last]
    assert dt[0] == 0 and dt[2] == 0 and dt[1] == pytest.approx(0.0625 * 0.5 / 128, rel=1e-15)
    # beyond the cutoff the switched entries are zero
    assert np.all(T.t[T.index(np.array([64.5]))[0][0] + 1:, [0, 1, 4, 5]] == 0)
    # the interpolant meets the next grid point (the refined c, d)
    x = 0.0625 / 128
    t0, t1 = T.t[0], T.t[1]
    for j in (0, 4):
        v = ((t0[j + 3] * x + t0[j + 2]) * x + t0[j + 1]) * x + t0[j]
        assert v == pytest.approx(t1[j], rel=1e-12)


def test_pair_force_id_round_trip():
    fid = ("LennardJonesTable -algorithm NonbondedCutoffB200 -switchingFunction Cn "
           "-n 3 -switchon 6 -switchoff 8 -cutoff 8 -cutoff 8")
    f = NonbondedCutoffB200PairForce.from_id(fid)
    assert f.lj_table and f.coulomb is None and f.lj == ("Cn", 6.0, 8.0, 3.0, 8.0)
    assert f.get_id() == fid
    with pytest.raises(ValueError):
        NonbondedCutoffB200PairForce(("C1", 0, 8.0), None, lj_table=True)
    with pytest.raises(ValueError):
        NonbondedCutoffB200PairForce(("C2", 6.5, 8.0), ("C1", 0, 8.0), lj_table=True)


def test_create_refuses_other_table_combinations():
    """C1 under the table and a Coulomb term beside it are not registered by
    the reference: PMB200_EUNSUPPORTED before any device work."""
    L = _lib.lib()
    arr = (ctypes.c_double * 4)
    for ljk, cok in ((_lib.PMB200_SW_TABLE | _lib.PMB200_SW_C1, _lib.PMB200_SW_NONE),
                     (_lib.PMB200_SW_TABLE | _lib.PMB200_SW_C2, _lib.PMB200_SW_C1),
                     (_lib.PMB200_SW_TABLE, _lib.PMB200_SW_NONE)):
        p = _lib.PairParams(_lib.PMB200_FP64, 0, ljk, arr(6.5, 8.0, 0, 0), cok,
                            arr(0, 8.0, 0, 0), 8.0, 0.0)
        h = ctypes.c_void_p()
        assert L.pmb200_create_pair(ctypes.byref(p), ctypes.byref(h)) == _lib.PMB200_EUNSUPPORTED


# ---- GPU: both kernels against the reference ------------------------------
def lj_magnitude(d, rc, periodic):
    pos, typ = d["pos"], d["type"]
    lj = np.asarray(d["lj"]).reshape(-1, 4)
    nt = int(round(np.sqrt(lj.shape[0])))
    box = np.asarray(d["box"], float)
    n = len(pos)
    tot = 0.0
    for i in range(n - 1):
        dv = pos[i + 1:] - pos[i]
        if periodic:
            dv -= box * np.rint(dv / box)
        r = np.sqrt((dv ** 2).sum(1))
        m = r <= rc
        p = lj[typ[i] * nt + typ[i + 1:][m]]
        tot += (np.abs(p[:, 0]) * r[m] ** -12 + np.abs(p[:, 1]) * r[m] ** -6).sum()
    return tot


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("fname,case", CASES)
def test_table_force_matches_reference(fx, fname, case, precision):
    d = fx[fname]
    sw = spec(d[f"{case}_lj"])
    vacuum = fname == "vacuum"
    f = NonbondedCutoffB200PairForce(sw, None, 8.0, precision=precision, lj_table=True)
    topo = PeriodicTopology.from_dict(d)
    if vacuum:
        topo.domain = (d["pos"].min(0) - 1.0, d["pos"].max(0) + 1.0)
    F = np.zeros_like(d["pos"])
    E = ScalarStructure(virial=True, molecular_virial=True)
    f.evaluate(topo, d["pos"], F, E)
    f.close()
    fr, er = d[f"{case}_forces"], d[f"{case}_energies"]
    vr, mvr = d[f"{case}_virial"], d[f"{case}_molvirial"]
    assert E[0] == 0.0
    if precision == "fp64":
        c2 = sw[0] == "C2"
        assert rms_rel(F, fr) <= (1e-12 if c2 else 1e-10)
        assert abs(E[1] - er[1]) <= (1e-11 if c2 else 1e-10) * abs(er[1])
        tv = 1e-11 if c2 else 1e-10
        assert np.allclose(E.virial_matrix().ravel(), vr, rtol=tv, atol=tv * np.abs(vr).max())
    else:
        assert rms_rel(F, fr) <= 1e-5
        bound = 1e-6 * lj_magnitude(d, 8.0, not vacuum) + 1e-7 * abs(er[1])
        assert abs(E[1] - er[1]) <= bound
        assert np.abs(E.virial_matrix().ravel() - vr).max() <= 1e-5 * np.abs(vr).max()
    assert np.abs(E.molvirial_matrix().ravel() - mvr).max() <= 1e-5 * max(np.abs(mvr).max(), 1.0)
