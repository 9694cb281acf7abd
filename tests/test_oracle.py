"""The CPU oracle (oracle/pm_oracle.c) against the reference's golden vectors
and, where it was built, against the reference compiled from its sources."""
import numpy as np
import pytest

from oracle import oracle as O
from protomoladdon_b200 import water


def test_golden_water423_energies(water423):
    """t = 0 energies of test/tests/expected/water_CHARMM_PERIODIC_L.energy
    (printed to 8 significant digits)."""
    f, e, v, mv = O.restate_eval(water423, water423["pos"], virial_mode=2)
    assert abs(e[1] - water423["golden_elj"]) <= 5e-5
    assert abs(e[0] - water423["golden_ecoul"]) <= 5e-5


@pytest.mark.parametrize("fx", ["water423", "water648", "modified648"])
def test_restatement_bitexact_vs_reference_fixture(fx, request):
    d = request.getfixturevalue(fx)
    f, e, v, mv = O.restate_eval(d, d["pos"], virial_mode=2)
    assert np.array_equal(f, d["ref_forces"])
    assert np.array_equal(e, d["ref_energies"])
    assert np.array_equal(v, d["ref_virial"])
    assert np.array_equal(mv, d["ref_molvirial"])


def test_restatement_leapfrog_bitexact(water648):
    p, v, e = O.restate_leapfrog(water648, water648["pos"], water648["vel"], 1.0, 20)
    assert np.array_equal(p, water648["lf20_pos"])
    assert np.array_equal(v, water648["lf20_vel"])
    assert np.array_equal(e, water648["lf20_energies"])


def test_cell_walk_equals_all_pairs(water648):
    f, e, v, _ = O.restate_eval(water648, water648["pos"], virial_mode=1)
    fb, eb, vb, _ = O.restate_eval(water648, water648["pos"], virial_mode=1, brute=True)
    assert np.abs(f - fb).max() < 1e-11
    assert np.allclose(e, eb, rtol=1e-12, atol=1e-9)
    assert np.allclose(v, vb, rtol=1e-12, atol=1e-9)


def test_newton_third_law(water648):
    f, _, _, _ = O.restate_eval(water648, water648["pos"], virial_mode=0)
    assert np.abs(f.sum(0)).max() < 1e-9


def test_forces_accumulate(water648):
    pos = water648["pos"]
    f1, _, _, _ = O.restate_eval(water648, pos, 0)
    import ctypes  # noqa: F401
    # accumulate semantics: a second evaluation into the same buffer doubles
    lib = O.restate_lib()
    ar = O._Arrays(water648)
    st = O._pmo_struct(water648, ar)
    p = np.ascontiguousarray(pos).reshape(-1)
    F = f1.reshape(-1).copy()
    E = np.zeros(2)
    assert lib.pmo_eval(ctypes.byref(st), O._ptr(p), O._ptr(F), O._ptr(E), None, None, 0, 0) == 0
    assert np.allclose(F.reshape(-1, 3), 2 * f1, rtol=0, atol=1e-12)


def test_translation_invariance_unwrapped(water648):
    """Positions are not wrapped by the caller; whole-box translations leave
    forces unchanged up to rounding."""
    L = water648["box"]
    shift = np.array([3 * L[0], -2 * L[1], 7 * L[2]])
    f0, e0, _, _ = O.restate_eval(water648, water648["pos"], 0)
    f1, e1, _, _ = O.restate_eval(water648, water648["pos"] + shift, 0)
    assert np.abs(f0 - f1).max() < 1e-8
    assert np.allclose(e0, e1, rtol=1e-10)


def test_empty_and_single_atom():
    s = water.small_648()
    for n in (0, 1):
        d = dict(s)
        for k in ("type", "qscaled", "mol", "mass"):
            d[k] = s[k][:n]
        d["excl"] = np.zeros((0, 3), np.int32)
        f, e, v, _ = O.restate_eval(d, s["pos"][:n], virial_mode=1)
        assert f.shape == (n, 3) and not f.any() and not e.any()


@pytest.mark.skipif(not O.ref_available(), reason="reference oracle library not built")
@pytest.mark.parametrize("seed", [1, 7])
def test_restatement_bitexact_vs_compiled_reference(seed):
    s = water.water_box(5, rc=7.0, ron=6.0, seed=seed)
    s["cellsize"] = 3.1
    R = O.RefForce(s)
    f, e, v, mv = R.evaluate(s["pos"], 2)
    g, ee, vv, mm = O.restate_eval(s, s["pos"], 2)
    R.close()
    assert np.array_equal(f, g) and np.array_equal(e, ee)
    assert np.array_equal(v, vv) and np.array_equal(mv, mm)


def test_pair_count_small(water648):
    n = O.restate_count_pairs(water648, water648["pos"])
    # ~0.5 * rho * 4/3 pi rc^3 per atom for the 648-atom box at rc 8
    assert 60_000 < n < 80_000


def test_settle_constraints_and_shake_agreement():
    from protomoladdon_b200 import rigid
    s = water.small_648()
    w = water.rigid_waters(s)
    assert w.shape == (216, 3)
    rng = np.random.default_rng(0)
    old = s["pos"]
    new = old + rng.normal(0, 0.02, old.shape)
    out = O.restate_settle(w, s["mass"], water.D_OH, water.D_HH, old, new)
    d = out[w]
    assert np.abs(np.linalg.norm(d[:, 1] - d[:, 0], axis=1) - water.D_OH).max() < 1e-12
    assert np.abs(np.linalg.norm(d[:, 2] - d[:, 0], axis=1) - water.D_OH).max() < 1e-12
    assert np.abs(np.linalg.norm(d[:, 2] - d[:, 1], axis=1) - water.D_HH).max() < 1e-12
    m = s["mass"][w][..., None]
    assert np.abs((m * (out[w] - new[w])).sum(1)).max() < 1e-12  # momentum kept
    # an iterative SHAKE on the same three constraints converges to SETTLE's answer
    x = new.copy()
    for _ in range(400):
        for a, b, d0 in ((0, 1, water.D_OH), (0, 2, water.D_OH), (1, 2, water.D_HH)):
            ia, ib = w[:, a], w[:, b]
            r, r0 = x[ib] - x[ia], old[ib] - old[ia]
            ma, mb = s["mass"][ia], s["mass"][ib]
            g = (d0 * d0 - (r * r).sum(1)) / (2 * (r * r0).sum(1) * (1 / ma + 1 / mb))
            x[ia] -= (g / ma)[:, None] * r0
            x[ib] += (g / mb)[:, None] * r0
    assert np.abs(x[w] - out[w]).max() < 1e-10
    # the host copy used by host-side integrators agrees
    host = rigid.settle(w, s["mass"], water.D_OH, water.D_HH, old, new.copy())
    assert np.abs(host - out).max() < 1e-12


def test_rigid_leapfrog_keeps_geometry(water648):
    w = water.rigid_waters(water648)
    p, v, e = O.restate_leapfrog_rigid(water648, water648["pos"], water648["vel"], 1.0, 10, w,
                                       water.D_OH, water.D_HH)
    d = p[w]
    assert np.abs(np.linalg.norm(d[:, 1] - d[:, 0], axis=1) - water.D_OH).max() < 1e-10
    assert np.isfinite(e).all()


# ---- Ewald real-space term --------------------------------------------------
EWALD_FIXTURES = ["ewald_water_ref.npz", "ewald_modified_ref.npz", "ewald_ions_ref.npz"]


@pytest.mark.parametrize("name", EWALD_FIXTURES)
@pytest.mark.parametrize("tag", ["poly5", "exact"])
def test_ewald_restatement_bitexact_vs_reference_fixture(name, tag):
    """Both reference builds (A&S polynomial as shipped; -DUSE_EWALD_EXACT_ERF)
    against the restatement, bit for bit."""
    from tests.conftest import load_fixture
    d = load_fixture(name)
    f, e, v, mv = O.restate_ewald_real(d, d["pos"], float(d["alpha"]), float(d["accuracy"]),
                                       exact_erfc=(tag == "exact"), virial_mode=2)
    assert np.array_equal(f, d[f"{tag}_forces"])
    assert e == float(d[f"{tag}_energy"])
    assert np.array_equal(v, d[f"{tag}_virial"])
    assert np.array_equal(mv, d[f"{tag}_molvirial"])


def test_ewald_cell_walk_equals_all_pairs():
    from tests.conftest import load_fixture
    d = load_fixture("ewald_ions_ref.npz")
    a, acc = float(d["alpha"]), float(d["accuracy"])
    f, e, v, _ = O.restate_ewald_real(d, d["pos"], a, acc, True, 1)
    fb, eb, vb, _ = O.restate_ewald_real(d, d["pos"], a, acc, True, 1, brute=True)
    assert np.abs(f - fb).max() < 1e-11 * np.abs(f).max()
    assert abs(e - eb) <= 1e-12 * abs(e)
    assert np.allclose(v, vb, rtol=1e-12, atol=1e-9)
    assert np.abs(f.sum(axis=0)).max() < 1e-9 * np.abs(f).max()  # Newton's third law


def test_ewald_constants_and_limits(water648):
    """rc = sqrt(-log(accuracy)) / alpha; the default alpha; a box below 2 rc
    is refused (the reference would add lattice images there)."""
    a, rc, a2pi, a2 = O.ewald_constants(water648, 0.30, float(np.exp(-(0.30 * 8.0) ** 2)))
    assert a == 0.30 and abs(rc - 8.0) < 1e-12 and abs(a2pi - 0.6 / np.sqrt(np.pi)) < 1e-15
    n = water648["n"]
    v = float(np.prod(water648["box"]))
    a, rc, _, _ = O.ewald_constants(water648, -1.0, 1e-5)
    assert abs(a - np.sqrt(np.pi) * (5.5 * n / v ** 2) ** (1.0 / 6.0)) < 1e-15
    with pytest.raises(RuntimeError):
        O.restate_ewald_real(water648, water648["pos"], 0.2, 1e-5)  # rc 17 > L / 2


def test_ewald_erfc_forms_agree_to_polynomial_error(water648):
    """The A&S polynomial (|error| <= 1.5e-7 in erfc) and libm erfc agree to
    that order, per pair and in total."""
    acc = float(np.exp(-(0.30 * 8.0) ** 2))
    f1, e1, _, _ = O.restate_ewald_real(water648, water648["pos"], 0.30, acc, False, 0)
    f2, e2, _, _ = O.restate_ewald_real(water648, water648["pos"], 0.30, acc, True, 0)
    assert 0 < abs(e1 - e2) < 1e-3 * abs(e2)
    assert np.sqrt(((f1 - f2) ** 2).sum() / (f2 ** 2).sum()) < 1e-5


@pytest.mark.skipif(not O.ref_available(True), reason="reference oracle library not built")
@pytest.mark.parametrize("seed,exact", [(3, False), (11, True)])
def test_ewald_restatement_bitexact_vs_compiled_reference(seed, exact):
    s = water.water_box(6, rc=8.0, ron=7.0, seed=seed, ion_fraction=0.06)
    s["cellsize"] = 2.9
    R = O.RefForce(s, exact_erfc=exact)
    acc = float(np.exp(-(0.33 * 8.5) ** 2))  # rc 8.5
    f, e, v, mv = R.ewald_real(s["pos"], 0.33, acc, 2)
    R.close()
    g, ee, vv, mm = O.restate_ewald_real(s, s["pos"], 0.33, acc, exact, 2)
    assert np.array_equal(f, g) and e == ee
    assert np.array_equal(v, vv) and np.array_equal(mv, mm)


def test_restatement_bitexact_vs_many_types_fixture():
    """A 30-type table (24 used) with modified H-H pairs: the restatement
    equals the reference's own output bit for bit."""
    from tests.conftest import load_fixture
    d = load_fixture("manytypes_ref.npz")
    f, e, v, mv = O.restate_eval(d, d["pos"], 2)
    assert np.array_equal(f, d["ref_forces"]) and np.array_equal(e, d["ref_energies"])
    assert np.array_equal(v, d["ref_virial"]) and np.array_equal(mv, d["ref_molvirial"])


@pytest.mark.skipif(not O.ref_available(), reason="reference oracle library not built")
def test_triclinic_fixture_is_the_reference_all_pairs_force():
    """The committed general-cell fixture equals a fresh evaluation of the
    reference's all-pairs force, and on an orthogonal box that force equals
    the reference's cell-list force (to summation order)."""
    from tests.conftest import load_fixture
    d = load_fixture("triclinic_ref.npz")
    R = O.RefForce(d)
    f, e, v, mv = R.evaluate_allpairs(d["pos"], 2)
    R.close()
    assert np.array_equal(f, d["ref_forces"]) and np.array_equal(e, d["ref_energies"])
    s = water.water_box(6, rc=8.0, ron=7.0, seed=3)
    R = O.RefForce(s)
    f1, e1, _, _ = R.evaluate(s["pos"], 1)
    f2, e2, _, _ = R.evaluate_allpairs(s["pos"], 1)
    R.close()
    assert np.abs(f1 - f2).max() <= 1e-12 * np.abs(f1).max()
    assert np.allclose(e1, e2, rtol=1e-13)
