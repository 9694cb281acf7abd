"""The ProtoMol plugin (protomoladdon_b200/plugin) inside the reference's own
ForceFactory: the config id `LennardJones Coulomb -algorithm
NonbondedCutoffB200 -switchingFunction C2 -switchingFunction C1` with the
reference's four parameter values resolves to the B200 force, and on a GPU
its results match the reference prototype made by the same factory."""
import numpy as np
import pytest

from oracle import oracle as O

from . import plugin_harness as H

pytestmark = pytest.mark.skipif(not (H.available() and O.ref_available()),
                                reason="plugin harness / reference library not built")


def test_factory_resolves_reference_and_plugin_ids(water648):
    R = O.RefForce(water648)
    rc, msg, f, e, v, mv = H.evaluate(R, 0, water648, water648["pos"])
    assert rc == 0, msg
    assert "NonbondedCutoff" in msg
    np.testing.assert_allclose(f, water648["ref_forces"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(e, water648["ref_energies"], rtol=1e-12)
    R.close()


def test_plugin_id_resolves_to_b200_force(water648):
    """Without a GPU the plugin's constructor reports the missing device;
    with one it evaluates.  Either way the factory picked the B200 force."""
    R = O.RefForce(water648)
    rc, msg, *_ = H.evaluate(R, 1, water648, water648["pos"])
    R.close()
    assert (rc == 0 and "NonbondedCutoffB200" in msg) or "B200 cutoff force" in msg


def test_plugin_rejects_bad_switchon(water648):
    d = dict(water648)
    d["ron"] = d["rc_lj"]  # switchon == cutoff: C2SwitchingFunction::make's rule
    R = O.RefForce(water648)
    rc, msg, *_ = H.evaluate(R, 1, d, d["pos"])
    R.close()
    assert rc == 1 and "B200 cutoff force" in msg


@pytest.mark.gpu
@pytest.mark.parametrize("which", [1, 2])
def test_plugin_matches_reference_through_factory(water648, which):
    R = O.RefForce(water648)
    rc, msg, f, e, v, mv = H.evaluate(R, which, water648, water648["pos"])
    R.close()
    assert rc == 0, msg
    assert "NonbondedCutoffB200" in msg
    fr = water648["ref_forces"]
    assert np.sqrt(((f - fr) ** 2).sum() / (fr ** 2).sum()) <= 1e-5
    assert np.abs(e - water648["ref_energies"]).max() <= 2e-3
    vr = water648["ref_virial"]
    assert np.abs(v - vr).max() <= 1e-5 * np.abs(vr).max()
    assert np.abs(mv - water648["ref_molvirial"]).max() <= 1e-5 * np.abs(vr).max()


def _ewald_fixture():
    from .conftest import load_fixture
    return load_fixture("ewald_water_ref.npz")


def test_factory_resolves_reference_ewald_real_id():
    d = _ewald_fixture()
    R = O.RefForce(d)
    rc, msg, f, e, v, mv = H.evaluate_ewald(R, 0, d, d["pos"], float(d["alpha"]),
                                            float(d["accuracy"]))
    R.close()
    assert rc == 0, msg
    assert "FullEwald -real" in msg
    np.testing.assert_allclose(f, d["poly5_forces"], rtol=0, atol=1e-11)
    assert abs(e[0] - float(d["poly5_energy"])) <= 1e-11 * abs(float(d["poly5_energy"]))


def test_plugin_ewald_id_resolves_to_b200_force():
    d = _ewald_fixture()
    R = O.RefForce(d)
    rc, msg, *_ = H.evaluate_ewald(R, 1, d, d["pos"], float(d["alpha"]), float(d["accuracy"]))
    R.close()
    assert (rc == 0 and "FullEwaldB200 -real" in msg) or "B200 Ewald real-space force" in msg


def test_plugin_ewald_rejects_bad_accuracy():
    d = _ewald_fixture()
    R = O.RefForce(d)
    rc, msg, *_ = H.evaluate_ewald(R, 1, d, d["pos"], 0.3, -1.0)
    R.close()
    assert rc == 1


@pytest.mark.gpu
def test_plugin_ewald_matches_reference_through_factory():
    d = _ewald_fixture()
    R = O.RefForce(d)
    rc, msg, f, e, v, mv = H.evaluate_ewald(R, 1, d, d["pos"], float(d["alpha"]),
                                            float(d["accuracy"]))
    R.close()
    assert rc == 0, msg
    fr = d["poly5_forces"]
    assert np.sqrt(((f - fr) ** 2).sum() / (fr ** 2).sum()) <= 1e-5
    # |dE| <= 1e-6 of the pair magnitudes (64,495 kcal/mol on this box)
    assert abs(e[0] - float(d["poly5_energy"])) <= 0.065 and e[1] == 0.0
    vr = d["poly5_virial"]
    assert np.abs(v - vr).max() <= 1e-5 * np.abs(vr).max()


# ---- the other switch combinations and vacuum boundaries -------------------
def _pair_case(name):
    """(force id, values) of a switch-policy fixture case, as a config gives them."""
    from .conftest import load_fixture
    d = load_fixture("pairs_ref.npz")
    names = {1: "C1", 2: "C2", 3: "Cn", 4: "ComplimentCnCn"}
    pots, sws, vals = [], [], []
    for pot, key in (("LennardJones", f"{name}_lj"), ("Coulomb", f"{name}_coul")):
        a = d[key]
        if a[0] == 0:
            continue
        kind = names[int(a[0])]
        pots.append(pot)
        sws.append(kind)
        ron, rc, order, roff = (float(x) for x in a[1:])
        vals += {"C1": [rc], "C2": [ron, rc], "Cn": [order, ron, roff, rc],
                 "ComplimentCnCn": [ron, roff, rc, order]}[kind]
    vals.append(8.0)  # algorithm cutoff
    fid = " ".join(pots) + "".join(f" -switchingFunction {k}" for k in sws) + \
        " -algorithm NonbondedCutoffB200"
    return d, fid, vals


def test_factory_resolves_switch_policy_ids():
    for case in ("c2_cn", "lj_c1", "coul_cn", "cm_cm", "lj_cm", "coul_cm"):
        d, fid, vals = _pair_case(case)
        R = O.RefForce(d)
        rc, msg, *_ = H.evaluate_pair(R, 0, fid, vals, d["pos"])
        R.close()
        assert (rc == 0 and fid in msg) or "B200 cutoff force" in msg, (case, msg)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["c2_c2", "c2_cn", "cn_cn", "lj_c1", "coul_c2", "cm_cm",
                                  "coul_cm"])
def test_switch_policy_plugin_matches_reference(case):
    d, fid, vals = _pair_case(case)
    R = O.RefForce(d)
    rc, msg, f, e, v, mv = H.evaluate_pair(R, 0, fid, vals, d["pos"])
    R.close()
    assert rc == 0, msg
    fr = d[f"{case}_forces"]
    assert np.sqrt(((f - fr) ** 2).sum() / (fr ** 2).sum()) <= 1e-5


def test_factory_resolves_vacuum_complimentcncn_id():
    """The vacuum registration OneAtomPairTwo<VBC, CmpCnCn, LJ, C1, Coulomb>
    (NonbondedCutoffForceModule.cpp:140-141) resolves through the factory."""
    from .conftest import load_fixture
    d = load_fixture("vacuum_ref.npz")
    R = O.RefForce(d)
    fid = ("LennardJones Coulomb -switchingFunction ComplimentCnCn -switchingFunction C1 "
           "-algorithm NonbondedCutoffB200")
    rc, msg, *_ = H.evaluate_pair(R, 1, fid, [3.0, 6.5, 8.0, 4.0, 8.0, 8.0], d["pos"])
    R.close()
    assert (rc == 0 and fid in msg) or "B200 cutoff force" in msg, msg


@pytest.mark.gpu
def test_vacuum_plugin_matches_reference():
    from .conftest import load_fixture
    d = load_fixture("vacuum_ref.npz")
    R = O.RefForce(d)
    fid = ("LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 "
           "-algorithm NonbondedCutoffB200")
    rc, msg, f, e, v, mv = H.evaluate_pair(R, 1, fid, [7.0, 8.0, 8.0, 8.0], d["pos"])
    R.close()
    assert rc == 0, msg
    fr = d["ref_forces"]
    assert np.sqrt(((f - fr) ** 2).sum() / (fr ** 2).sum()) <= 1e-5
    assert np.abs(e - d["ref_energies"]).max() <= 2e-3


def _table_case(fname, case):
    """(fixture, force id, values) of a tabulated-LJ fixture case."""
    from .conftest import load_fixture
    d = load_fixture(f"ljtable_{fname}_ref.npz")
    a = d[f"{case}_lj"]
    kind = {2: "C2", 3: "Cn", 4: "ComplimentCnCn"}[int(a[0])]
    ron, rc, order, roff = (float(x) for x in a[1:])
    vals = {"C2": [ron, rc], "Cn": [order, ron, roff, rc],
            "ComplimentCnCn": [ron, roff, rc, order]}[kind] + [8.0]
    return d, f"LennardJonesTable -switchingFunction {kind} -algorithm NonbondedCutoffB200", vals


def test_factory_resolves_ljtable_ids():
    """OneAtomPair<BC, Universal, LennardJonesTableForce<S, 7, Real>>
    (NonbondedCutoffForceModule.cpp:67-72, 121-126) for both boundaries."""
    for fname, case, vac in (("water", "t_c2", 0), ("water", "t_cn", 0), ("water", "t_cm", 0),
                             ("vacuum", "t_cm", 1)):
        d, fid, vals = _table_case(fname, case)
        R = O.RefForce(d)
        rc, msg, *_ = H.evaluate_pair(R, vac, fid, vals, d["pos"])
        R.close()
        assert (rc == 0 and fid in msg) or "B200 cutoff force" in msg, (case, msg)


@pytest.mark.gpu
@pytest.mark.parametrize("fname,case,vac", [("water", "t_c2", 0), ("modified", "t_c2", 0),
                                            ("water", "t_cm", 0), ("vacuum", "t_cn", 1)])
def test_ljtable_plugin_matches_reference(fname, case, vac):
    d, fid, vals = _table_case(fname, case)
    R = O.RefForce(d)
    rc, msg, f, e, v, mv = H.evaluate_pair(R, vac, fid, vals, d["pos"])
    R.close()
    assert rc == 0, msg
    fr = d[f"{case}_forces"]
    assert np.sqrt(((f - fr) ** 2).sum() / (fr ** 2).sum()) <= 1e-5
    assert e[0] == 0.0 and abs(e[1] - d[f"{case}_energies"][1]) <= 1e-3


def _parallel_vs_plain(call):
    """(plain result, parallelEvaluate result, blocks) of one harness call."""
    H.set_parallel(False)
    plain = call()
    H.set_parallel(True)
    try:
        par = call()
        blocks = H.last_blocks()
    finally:
        H.set_parallel(False)
    return plain, par, blocks


def test_reference_parallel_evaluate_equals_evaluate(water648):
    """The harness's parallel mode on the reference prototype: without MPI
    Parallel::next() grants every block, so parallelEvaluate == evaluate."""
    R = O.RefForce(water648)
    plain, par, blocks = _parallel_vs_plain(
        lambda: H.evaluate(R, 0, water648, water648["pos"]))
    R.close()
    assert plain[0] == 0 and par[0] == 0, par[1]
    assert blocks >= 1
    np.testing.assert_allclose(par[2], plain[2], rtol=0, atol=1e-12)
    np.testing.assert_allclose(par[3], plain[3], rtol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("which", [1, 2])
def test_plugin_parallel_evaluate_matches_evaluate(water648, which):
    """The B200 forces override parallelEvaluate / numberOfBlocks (the
    default would evaluate everything on every rank); under the reference's
    sequential Parallel every block is granted, so the result is evaluate's,
    and numberOfBlocks is the number of device grid cells."""
    R = O.RefForce(water648)
    plain, par, blocks = _parallel_vs_plain(
        lambda: H.evaluate(R, which, water648, water648["pos"]))
    R.close()
    assert plain[0] == 0 and par[0] == 0, par[1]
    from protomoladdon_b200.force import NonbondedCutoffB200SystemForce, PeriodicTopology
    f = NonbondedCutoffB200SystemForce(water648["ron"], water648["rc_lj"], water648["rc_coul"],
                                       water648["rc_alg"])
    assert blocks == f.number_of_blocks(PeriodicTopology.from_dict(water648))
    f.close()
    # (evaluate's host-buffer call returns the mixed forces rounded to FP32;
    # the block shares come back in FP64)
    np.testing.assert_allclose(par[2], plain[2], rtol=0, atol=1e-7 * np.abs(plain[2]).max())
    np.testing.assert_allclose(par[3], plain[3], rtol=1e-12)
    np.testing.assert_allclose(par[4], plain[4], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(par[5], plain[5], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_plugin_ewald_and_pair_parallel_evaluate(water648):
    """parallelEvaluate == evaluate for the Ewald real-space force, a
    periodic switch-policy force and the vacuum force (sequential Parallel)."""
    from .conftest import load_fixture
    acc = float(np.exp(-(0.35 * 8.0) ** 2))
    dp, fid, vals = _pair_case("c2_cn")
    dv = load_fixture("vacuum_ref.npz")
    vid = ("LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 "
           "-algorithm NonbondedCutoffB200")
    cases = ((water648, lambda R: H.evaluate_ewald(R, 1, water648, water648["pos"], 0.35, acc)),
             (dp, lambda R: H.evaluate_pair(R, 0, fid, vals, dp["pos"])),
             (dv, lambda R: H.evaluate_pair(R, 1, vid, [7.0, 8.0, 8.0, 8.0], dv["pos"])))
    for d, call in cases:
        R = O.RefForce(d)
        plain, par, blocks = _parallel_vs_plain(lambda: call(R))
        R.close()
        assert plain[0] == 0 and par[0] == 0, par[1]
        assert blocks >= 1
        # (mixed forces: FP32 from evaluate's host-buffer call, FP64 shares)
        np.testing.assert_allclose(par[2], plain[2], rtol=0,
                                   atol=1e-7 * np.abs(plain[2]).max())
        np.testing.assert_allclose(par[3], plain[3], rtol=1e-12, atol=1e-12)
