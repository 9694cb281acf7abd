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
