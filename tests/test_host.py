"""Host logic without a GPU: parameter parsing/validation, the water
generator, the C-ABI library's exported symbols and its argument checks."""
import ctypes
import os
import re

import numpy as np
import pytest

from protomoladdon_b200 import _lib, water
from protomoladdon_b200.force import (EwaldRealB200SystemForce, NonbondedCutoffB200SystemForce,
                                      PeriodicTopology)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "pmb200.h")).read()
    return sorted(set(re.findall(r"\b(pmb200_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert set(syms) == set(_lib.EXPORTED)
    for s in syms:
        assert getattr(L, s) is not None


def test_create_validates_before_touching_a_device():
    L = _lib.lib()
    h = ctypes.c_void_p()
    bad = [
        _lib.Params(0, 0, 10.0, 9.0, 9.0, 9.0, 0.0),   # switchon >= cutoff (C2 make)
        _lib.Params(0, 0, -1.0, 9.0, 9.0, 9.0, 0.0),   # negative switchon
        _lib.Params(7, 0, 8.0, 9.0, 9.0, 9.0, 0.0),    # unknown precision
        _lib.Params(0, 0, 8.0, 9.0, 0.0, 9.0, 0.0),    # zero Coulomb cutoff
    ]
    for p in bad:
        assert L.pmb200_create(ctypes.byref(p), ctypes.byref(h)) == _lib.PMB200_EINVAL
    p = _lib.Params(0, 0, 8.0, 9.0, 9.0, 8.5, 0.0)     # algorithm cutoff below switch
    assert L.pmb200_create(ctypes.byref(p), ctypes.byref(h)) == _lib.PMB200_EUNSUPPORTED
    assert L.pmb200_create(None, ctypes.byref(h)) == _lib.PMB200_EINVAL
    assert L.pmb200_destroy(None) == 0


def test_force_id_parse_and_make():
    f = NonbondedCutoffB200SystemForce.from_id(
        "LennardJones Coulomb -algorithm NonbondedCutoffB200 -switchingFunction C2 "
        "-switchingFunction C1 -switchon 9 -cutoff 10 -cutoff 10 -cutoff 10")
    assert (f.switchon, f.cutoff_lj, f.cutoff_coul, f.cutoff_alg) == (9, 10, 10, 10)
    assert NonbondedCutoffB200SystemForce.from_id(f.get_id()).get_id() == f.get_id()
    with pytest.raises(ValueError):
        NonbondedCutoffB200SystemForce.make([10, 10, 10, 10])  # switchon == cutoff
    with pytest.raises(ValueError):
        NonbondedCutoffB200SystemForce.from_id(
            "LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction C2 "
            "-switchingFunction C1 -switchon 9 -cutoff 10 -cutoff 10 -cutoff 10")
    with pytest.raises(ValueError):
        NonbondedCutoffB200SystemForce.make([1, 2, 3])


def test_ewald_create_validates_before_touching_a_device():
    L = _lib.lib()
    h = ctypes.c_void_p()
    bad = [
        _lib.EwaldParams(0, 0, 0, 0.3, 0.0, 0.0),   # accuracy must be > 0
        _lib.EwaldParams(0, 0, 0, 0.3, 1.0, 0.0),   # and < 1 (rc = 0)
        _lib.EwaldParams(0, 0, 5, 0.3, 1e-6, 0.0),  # unknown erfc form
        _lib.EwaldParams(0, 0, 0, float("nan"), 1e-6, 0.0),
        _lib.EwaldParams(0, 0, 0, 0.3, 1e-6, -1.0),  # negative cell size
    ]
    for p in bad:
        assert L.pmb200_create_ewald_real(ctypes.byref(p), ctypes.byref(h)) == _lib.PMB200_EINVAL
    assert L.pmb200_create_ewald_real(None, ctypes.byref(h)) == _lib.PMB200_EINVAL
    a, r = ctypes.c_double(), ctypes.c_double()
    assert L.pmb200_ewald_info(None, ctypes.byref(a), ctypes.byref(r)) == _lib.PMB200_EINVAL


def test_ewald_force_id_parse_and_make():
    f = EwaldRealB200SystemForce.from_id(
        "Coulomb -algorithm FullEwaldB200 -real -alpha 0.3 -accuracy 2.35e-6")
    assert (f.alpha, f.accuracy, f.erfc) == (0.3, 2.35e-6, "poly5")
    assert EwaldRealB200SystemForce.from_id(f.get_id()).get_id() == f.get_id()
    d = EwaldRealB200SystemForce.from_id("Coulomb -algorithm FullEwaldB200 -real")
    assert (d.alpha, d.accuracy) == (-1.0, 1e-5)  # the reference's defaults
    assert EwaldRealB200SystemForce.make([0.25, 1e-6], erfc="exact").erfc == "exact"
    for bad in ("Coulomb -algorithm FullEwaldB200 -real -reciprocal",
                "Coulomb -algorithm FullEwald -real", "LennardJones -algorithm FullEwaldB200"):
        with pytest.raises(ValueError):
            EwaldRealB200SystemForce.from_id(bad)
    with pytest.raises(ValueError):
        EwaldRealB200SystemForce.make([0.3, 0.0])
    with pytest.raises(ValueError):
        EwaldRealB200SystemForce.make([0.3])


@pytest.mark.parametrize("k,n", [(6, 648), (24, 41472)])
def test_water_box_recipe(k, n):
    s = water.water_box(k, rc=10.0, ron=9.0)
    assert s["n"] == n and s["pos"].shape == (n, 3)
    assert np.isclose(s["box"][0], k * water.LATTICE)
    q = s["qscaled"].reshape(-1, 3).sum(1)
    assert np.abs(q).max() < 1e-12  # neutral molecules
    d = s["pos"].reshape(-1, 3, 3)
    oh = np.linalg.norm(d[:, 1] - d[:, 0], axis=1)
    assert np.allclose(oh, water.R_OH)
    ang = np.degrees(np.arccos(np.einsum("ij,ij->i", d[:, 1] - d[:, 0], d[:, 2] - d[:, 0])
                               / water.R_OH ** 2))
    assert np.allclose(ang, 104.52)
    assert s["excl"].shape == (3 * n // 3, 3)
    s2 = water.water_box(k, rc=10.0, ron=9.0)
    assert np.array_equal(s["pos"], s2["pos"])  # seeded


def test_ion_box_and_batch():
    s = water.water_box(10, rc=9.0, ron=8.0, ion_fraction=0.02)
    nion = int(np.isin(s["type"], [water.T_NA, water.T_CL]).sum())
    assert nion == 2 * round(0.02 * 1000 / 2)
    assert abs(s["qscaled"].sum()) < 1e-9
    boxes = water.batch_boxes(count=16)
    for b in boxes:
        assert 300 - 3 <= b["n"] <= 6000 + 3 and b["box"][0] >= 18.0 - 1e-12


def test_topology_wrapper(water648):
    t = PeriodicTopology.from_dict(water648)
    assert t.n == 648 and t.ntypes == 2 and t.e.shape == (3, 3)


def test_host_kick_drift_matches_numpy_settle():
    from protomoladdon_b200 import rigid
    s = water.small_648()
    w = water.rigid_waters(s)
    rng = np.random.default_rng(1)
    F = rng.normal(0, 20, s["pos"].shape)
    p1, v1 = s["pos"].copy(), s["vel"].copy()
    p2, v2 = s["pos"].copy(), s["vel"].copy()
    rigid.kick_drift_settle(p1, v1, F, s["mass"], 1.0, w, water.D_OH, water.D_HH)
    rigid.host_kick_drift(p2, v2, F, s["mass"], 1.0, w, water.D_OH, water.D_HH)
    assert np.abs(p1 - p2).max() < 1e-12 and np.abs(v1 - v2).max() < 1e-9


def test_host_kick_drift_free_atoms_and_bad_water_lists():
    """Atoms outside the listed waters are kicked and drifted only; a water
    list that names an atom twice, or an atom out of range, is refused
    before anything is updated."""
    from protomoladdon_b200 import _lib, rigid
    s = water.small_648()
    w = water.rigid_waters(s)
    rng = np.random.default_rng(2)
    F = rng.normal(0, 20, s["pos"].shape)
    # the last 10 waters are left free: their atoms follow plain leapfrog
    p1, v1 = s["pos"].copy(), s["vel"].copy()
    p2, v2 = s["pos"].copy(), s["vel"].copy()
    rigid.kick_drift_settle(p1, v1, F, s["mass"], 1.0, w[:-10], water.D_OH, water.D_HH)
    rigid.host_kick_drift(p2, v2, F, s["mass"], 1.0, w[:-10], water.D_OH, water.D_HH)
    assert np.abs(p1 - p2).max() < 1e-12 and np.abs(v1 - v2).max() < 1e-9
    free = np.asarray(w[-10:]).reshape(-1)
    h = 1.0 * 0.02045482828087295
    v_ref = s["vel"][free] + F[free] * (h / s["mass"][free])[:, None]
    np.testing.assert_allclose(v2[free], v_ref, rtol=1e-14, atol=0)
    np.testing.assert_allclose(p2[free], s["pos"][free] + v_ref * h, rtol=1e-14, atol=1e-14)
    for bad in (np.concatenate([w[:2], w[:1]]), np.array([[0, 1, s["n"]]], np.int32)):
        p3, v3 = s["pos"].copy(), s["vel"].copy()
        with pytest.raises(_lib.PmbError) as ei:
            rigid.host_kick_drift(p3, v3, F, s["mass"], 1.0, bad, water.D_OH, water.D_HH)
        assert ei.value.code == _lib.PMB200_EINVAL
        assert np.array_equal(p3, s["pos"]) and np.array_equal(v3, s["vel"])


def test_host_kick_drift_any_water_order():
    """Waters listed in any order (not increasing: the one-by-one check) and
    with some waters free give the same result as the increasing listing."""
    from protomoladdon_b200 import rigid
    s = water.small_648()
    w = np.asarray(water.rigid_waters(s)).reshape(-1, 3)
    rng = np.random.default_rng(3)
    F = rng.normal(0, 20, s["pos"].shape)
    for keep in (len(w), len(w) - 7):
        sub = w[:keep]
        p1, v1 = s["pos"].copy(), s["vel"].copy()
        rigid.host_kick_drift(p1, v1, F, s["mass"], 1.0, sub, water.D_OH, water.D_HH)
        p2, v2 = s["pos"].copy(), s["vel"].copy()
        rigid.host_kick_drift(p2, v2, F, s["mass"], 1.0, sub[rng.permutation(keep)],
                              water.D_OH, water.D_HH)
        assert np.array_equal(p1, p2) and np.array_equal(v1, v2)


def test_host_kick_drift_clears_forces_after_use():
    """clear_forces: the same positions and velocities, and every force entry
    (waters and free atoms, including a short last group of waters) zero."""
    from protomoladdon_b200 import rigid
    s = water.small_648()
    w = np.asarray(water.rigid_waters(s)).reshape(-1, 3)[:-5]  # 211 waters, 5 free
    rng = np.random.default_rng(4)
    F = rng.normal(0, 20, s["pos"].shape)
    p1, v1 = s["pos"].copy(), s["vel"].copy()
    rigid.host_kick_drift(p1, v1, F, s["mass"], 1.0, w, water.D_OH, water.D_HH)
    p2, v2, F2 = s["pos"].copy(), s["vel"].copy(), F.copy()
    rigid.host_kick_drift(p2, v2, F2, s["mass"], 1.0, w, water.D_OH, water.D_HH,
                          clear_forces=True)
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)
    assert not F2.any()


def test_lj_table_mixing_matches_the_generator():
    """autograd.lj_table (torch, differentiable) reproduces the water
    generator's table, ions included."""
    import torch
    from protomoladdon_b200.autograd import lj_table
    for ions in (False, True):
        ref = water._lj_table(ions)
        sig = [water.SIG_O, 0.0] + ([water.SIG_NA, water.SIG_CL] if ions else [])
        eps = [water.EPS_O, 0.0] + ([water.EPS_NA, water.EPS_CL] if ions else [])
        t = lj_table(torch.tensor(sig, dtype=torch.float64), torch.tensor(eps, dtype=torch.float64))
        np.testing.assert_allclose(t.numpy(), ref, rtol=1e-13, atol=0)
    s = torch.tensor([3.0, 0.0], dtype=torch.float64, requires_grad=True)
    e = torch.tensor([0.2, 0.0], dtype=torch.float64, requires_grad=True)
    lj_table(s, e).sum().backward()
    assert torch.isfinite(s.grad).all() and torch.isfinite(e.grad).all()


def test_pair_form_create_validates_before_touching_a_device():
    L = _lib.lib()
    h = ctypes.c_void_p()
    D4 = ctypes.c_double * 4

    def P(lk, lp, ck, cp, alg=10.0):
        return _lib.PairParams(0, 0, lk, D4(*lp), ck, D4(*cp), alg, 0.0)
    C2, CN, C1, NO = _lib.PMB200_SW_C2, _lib.PMB200_SW_CN, _lib.PMB200_SW_C1, _lib.PMB200_SW_NONE
    CM = _lib.PMB200_SW_CMPCNCN
    z = (0, 0, 0, 0)
    bad = [P(NO, z, NO, z),                          # no term at all
           P(C2, (9, 9, 0, 0), NO, z),               # C2 switchon == cutoff
           P(CN, (5, 8, 7, 0), NO, z),               # Cn order above 6
           P(CN, (5, 8, 4, 9), NO, z),               # switchoff neither 0 nor the cutoff
           P(C1, (0, -1, 0, 0), NO, z),              # negative cutoff
           P(CM, (6, 8, 4, 5), NO, z),               # ComplimentCnCn switchon above switchoff
           P(CM, (3, 8, 4, 9), NO, z),               # ComplimentCnCn switchoff beyond the cutoff
           P(CM, (3, 8, 7, 6), NO, z),               # ComplimentCnCn order above 6
           P(9, (0, 8, 0, 0), NO, z)]                # unknown switch
    for p in bad:
        assert L.pmb200_create_pair(ctypes.byref(p), ctypes.byref(h)) == _lib.PMB200_EINVAL
    p = P(CN, (5, 8, 5, 0), NO, z)                   # order 5: the reference's zero table
    assert L.pmb200_create_pair(ctypes.byref(p), ctypes.byref(h)) == _lib.PMB200_EUNSUPPORTED
    p = P(CM, (3, 8, 2.5, 6), NO, z)                 # an order the reference would truncate
    assert L.pmb200_create_pair(ctypes.byref(p), ctypes.byref(h)) == _lib.PMB200_EUNSUPPORTED
    p = P(C1, (0, 9, 0, 0), C1, (0, 9, 0, 0), alg=8.0)  # algorithm cutoff below a switch
    assert L.pmb200_create_pair(ctypes.byref(p), ctypes.byref(h)) == _lib.PMB200_EUNSUPPORTED


def test_pair_form_ids_round_trip():
    from protomoladdon_b200.force import NonbondedCutoffB200PairForce as P
    for lj, co in ((("C2", 6.5, 8.0), ("Cn", 5.0, 8.0, 4, 0)), (None, ("C1", 0, 9.0)),
                   (("Cn", 6, 8, 3, 8), None), (("C2", 7, 9), ("C2", 0, 9)),
                   (("ComplimentCnCn", 3, 8, 4, 6), ("ComplimentCnCn", 2, 8, 2, 5))):
        f = P(lj, co)
        g = P.from_id(f.get_id())
        assert g.get_id() == f.get_id() and g.lj == f.lj and g.coulomb == f.coulomb
    with pytest.raises(ValueError):
        P.from_id("LennardJones -algorithm NonbondedCutoffB200 -switchingFunction C2 -cutoff 8 "
                  "-cutoff 8")  # C2 wants -switchon first
    with pytest.raises(ValueError):
        P(("C3", 1, 2), None)


def test_topology_cache_follows_the_object_not_its_id(monkeypatch):
    """A force sends the topology again whenever it is handed another
    topology object -- also one that Python places at the address of a freed
    one, where an id()-keyed cache would keep the old atoms -- and not again
    for the same unchanged object (the C-ABI calls recorded by a fake)."""
    calls = []

    class FakeLib:
        def __getattr__(self, name):
            def call(*args):
                calls.append(name)
                return _lib.PMB200_OK
            return call

    monkeypatch.setattr(_lib, "lib", lambda: FakeLib())
    f = NonbondedCutoffB200SystemForce(7.0, 8.0, 8.0, 8.0, precision="mixed")
    f._ctx = ctypes.c_void_p(1)  # (no context is created: the fake serves every call)
    try:
        boxes = [water.water_box(k, rc=8.0, ron=7.0, seed=k) for k in (3, 4)]
        for s in boxes + boxes:
            topo = PeriodicTopology.from_dict(s)
            f._ensure(topo)
            del topo
        assert calls.count("pmb200_set_topology") == 4
        topo = PeriodicTopology.from_dict(boxes[0])
        f._ensure(topo)
        f._ensure(topo)
        assert calls.count("pmb200_set_topology") == 5
    finally:
        f._ctx = None
