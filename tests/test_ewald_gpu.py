"""GPU parity of the real-space Ewald term (pmb200_create_ewald_real) against
the reference's own outputs (committed fixtures from both of its builds)
and the CPU oracle.

Tolerances (written here, checked below):
* FP64 kernel: forces RMS relative <= 1e-12, energy and virial relative
  <= 1e-11 -- the arithmetic is the reference's, only the summation order and
  the device's exp/erfc (within an ulp of libm) differ.
* mixed kernel: forces RMS relative <= 1e-5; energy
  |dE| <= 1e-6 * sum over pairs |E_pair| (the small boxes' real-space energy
  is a sum of terms of both signs that cancels to a few percent of their
  magnitudes, so the bound is taken on the magnitudes); virial relative
  <= 1e-5 of its largest component.
"""
import ctypes

import numpy as np
import pytest
from scipy.special import erfc

from oracle import oracle as O
from protomoladdon_b200 import _lib, water
from protomoladdon_b200._lib import PmbError
from protomoladdon_b200.force import EwaldRealB200SystemForce, PeriodicTopology, ScalarStructure

from .conftest import load_fixture

pytestmark = pytest.mark.gpu

FIXTURES = ["ewald_water_ref.npz", "ewald_modified_ref.npz", "ewald_ions_ref.npz"]


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def abs_pair_energy(d, alpha, rc):
    """sum over pairs within rc of |q_i q_j erfc(alpha r) / r| (numpy, brute
    force; the scale of the energy's rounding error)."""
    pos, q, box = d["pos"], d["qscaled"], np.asarray(d["box"], float)
    n = len(q)
    full = np.zeros((n, n), bool)
    scale = np.ones((n, n))
    for a, b, k in np.asarray(d["excl"]).reshape(-1, 3):
        if k == 2:
            full[a, b] = full[b, a] = True
        elif k == 1:
            scale[a, b] = scale[b, a] = float(d.get("coulomb_scaling", 1.0))
    tot = 0.0
    for i in range(n - 1):
        dv = pos[i + 1:] - pos[i]
        dv -= box * np.rint(dv / box)
        r = np.sqrt((dv ** 2).sum(1))
        m = (r <= rc) & ~full[i, i + 1:]
        tot += np.abs(q[i] * q[i + 1:][m] * scale[i, i + 1:][m] * erfc(alpha * r[m]) / r[m]).sum()
    return tot


def run(d, precision, erfc_form, alpha, accuracy, virial=True, molvir=True, pos=None):
    topo = PeriodicTopology.from_dict(d)
    f = EwaldRealB200SystemForce(alpha, accuracy, precision=precision, erfc=erfc_form)
    F = np.zeros_like(d["pos"])
    E = ScalarStructure(virial=virial, molecular_virial=molvir)
    f.evaluate(topo, d["pos"] if pos is None else pos, F, E)
    info = f.ewald_info()
    pairs = f.last_pair_count()
    f.close()
    return F, E, info, pairs


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("form", ["poly5", "exact"])
def test_fp64_matches_reference(name, form):
    d = load_fixture(name)
    F, E, _, _ = run(d, "fp64", form, float(d["alpha"]), float(d["accuracy"]))
    assert rms_rel(F, d[f"{form}_forces"]) <= 1e-12
    e = float(d[f"{form}_energy"])
    assert abs(E[0] - e) <= 1e-11 * abs(e)
    assert E[1] == 0.0
    v, mv = d[f"{form}_virial"], d[f"{form}_molvirial"]
    assert np.allclose(E.virial_matrix().ravel(), v, rtol=1e-11, atol=1e-11 * np.abs(v).max())
    assert np.allclose(E.molvirial_matrix().ravel(), mv, rtol=1e-11,
                       atol=1e-11 * np.abs(mv).max())


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("form", ["poly5", "exact"])
def test_mixed_matches_reference(name, form):
    d = load_fixture(name)
    F, E, (alpha, rc), _ = run(d, "mixed", form, float(d["alpha"]), float(d["accuracy"]))
    err = rms_rel(F, d[f"{form}_forces"])
    assert err <= 1e-5, err
    e = float(d[f"{form}_energy"])
    scale = abs_pair_energy(d, alpha, rc)
    assert abs(E[0] - e) <= 1e-6 * scale, (E[0], e, scale)
    v, mv = d[f"{form}_virial"], d[f"{form}_molvirial"]
    assert np.abs(E.virial_matrix().ravel() - v).max() <= 1e-5 * np.abs(v).max()
    assert np.abs(E.molvirial_matrix().ravel() - mv).max() <= 1e-5 * np.abs(mv).max()


def test_default_alpha_and_cutoff_match_the_reference():
    d = load_fixture("ewald_modified_ref.npz")  # made with alpha <= 0 (the default)
    _, _, (alpha, rc), pairs = run(d, "mixed", "poly5", -1.0, float(d["accuracy"]),
                                   virial=False, molvir=False)
    a0, rc0, _, _ = O.ewald_constants(d, -1.0, float(d["accuracy"]))
    assert abs(alpha - a0) <= 1e-15 * a0 and abs(rc - rc0) <= 1e-14 * rc0
    assert pairs == O.restate_count_pairs_ewald(d, d["pos"], -1.0, float(d["accuracy"]))


def test_box_before_topology_with_default_alpha():
    """Through the C ABI in the other call order: the cutoff, which needs N,
    is settled when the topology arrives."""
    d = load_fixture("ewald_water_ref.npz")
    L = _lib.lib()
    h = ctypes.c_void_p()
    p = _lib.EwaldParams(_lib.PMB200_FP64, 0, _lib.PMB200_ERFC_EXACT, -1.0, 1e-5, 0.0)
    assert L.pmb200_create_ewald_real(ctypes.byref(p), ctypes.byref(h)) == 0
    e = np.diag(np.asarray(d["box"], float))
    org = np.zeros(3)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rows = [np.ascontiguousarray(e[k]) for k in range(3)]
    assert L.pmb200_set_box(h, *[ptr(r) for r in rows], ptr(org)) == 0
    a, r = ctypes.c_double(), ctypes.c_double()
    assert L.pmb200_ewald_info(h, ctypes.byref(a), ctypes.byref(r)) == _lib.PMB200_ESTATE
    t = np.ascontiguousarray(d["type"], np.int32)
    q = np.ascontiguousarray(d["qscaled"], float)
    mol = np.ascontiguousarray(d["mol"], np.int32)
    mass = np.ascontiguousarray(d["mass"], float)
    lj = np.ascontiguousarray(d["lj"], float).reshape(-1)
    ex = np.ascontiguousarray(d["excl"], np.int32).reshape(-1)
    nt = int(round((lj.size // 4) ** 0.5))
    assert L.pmb200_set_topology(h, t.size, ptr(t), ptr(q), ptr(mol), ptr(mass), nt, ptr(lj),
                                 ex.size // 3, ptr(ex), 1.0) == 0
    assert L.pmb200_ewald_info(h, ctypes.byref(a), ctypes.byref(r)) == 0
    a0, rc0, _, _ = O.ewald_constants(d, -1.0, 1e-5)
    assert abs(a.value - a0) <= 1e-15 * a0 and abs(r.value - rc0) <= 1e-14 * rc0
    pos = np.ascontiguousarray(d["pos"], float).reshape(-1)
    F = np.zeros_like(pos)
    en, vir, mvir = np.zeros(2), np.zeros(9), np.zeros(9)
    assert L.pmb200_eval(h, ptr(pos), ptr(F), ptr(en), ptr(vir), ptr(mvir),
                         _lib.PMB200_ENERGY) == 0
    L.pmb200_destroy(h)
    fo, eo, _, _ = O.restate_ewald_real(d, d["pos"], -1.0, 1e-5, True, 0)
    assert rms_rel(F.reshape(-1, 3), fo) <= 1e-12
    assert abs(en[0] - eo) <= 1e-11 * abs(eo)


def test_box_below_twice_the_cutoff_is_refused():
    d = load_fixture("ewald_water_ref.npz")  # 18.6 A box
    with pytest.raises(PmbError) as ei:
        run(d, "mixed", "poly5", 0.2, 1e-5)  # rc = 17 A
    assert ei.value.code == _lib.PMB200_EUNSUPPORTED


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_seeded_boxes_vs_oracle(precision):
    """Unwrapped, shifted positions in a non-cubic box with ions, against the
    oracle on the same inputs."""
    s = water.water_box(7, rc=9.0, ron=8.0, seed=5, ion_fraction=0.08)
    s["box"] = np.asarray(s["box"], float) * np.array([1.0, 1.07, 0.97])
    pos = s["pos"] + np.array([31.0, -47.5, 12.25])
    acc = float(np.exp(-(0.31 * 9.0) ** 2))
    fo, eo, vo, _ = O.restate_ewald_real(s, pos, 0.31, acc, False, 1)
    F, E, _, _ = run(s, precision, "poly5", 0.31, acc, molvir=False, pos=pos)
    tol = 1e-5 if precision == "mixed" else 1e-12
    assert rms_rel(F, fo) <= tol
    assert np.abs(E.virial_matrix().ravel() - vo).max() <= tol * np.abs(vo).max()


def test_large_box_mixed_against_fp64():
    """The 331,776-atom ion box at alpha 0.30, rc 12 (the large benchmark
    system): mixed against the FP64 kernel, and Newton's third law."""
    s = water.large_331k()
    acc = float(np.exp(-(0.30 * 12.0) ** 2))
    Fm, Em, (alpha, rc), pm = run(s, "mixed", "poly5", 0.30, acc, molvir=False)
    Fd, Ed, _, pd = run(s, "fp64", "poly5", 0.30, acc, molvir=False)
    # pairs within an FP32 rounding of rc^2 may be classified differently
    # (their erfc(3.6)/12 terms are ~1e-5 kcal/mol)
    assert abs(rc - 12.0) < 1e-9 and abs(pm - pd) <= 1e-6 * pd
    assert rms_rel(Fm, Fd) <= 1e-5
    # energy bound on the pair magnitudes, as for the small boxes: their sum
    # per atom, measured on the 648-atom box of the same recipe (~100
    # kcal/mol at alpha 0.30; the pairs beyond 8 A add < 0.1%), times n
    small = water.small_648()
    per_atom = abs_pair_energy(small, 0.30, 8.0) / small["n"]
    assert abs(Em[0] - Ed[0]) <= 1e-6 * per_atom * s["n"]
    # Newton's third law up to the fixed-point rounding of the j forces
    # (2^-18 cell units per pair contribution, random in sign): the net force
    # is a sum of n independent errors each far below 1e-5 of the RMS force
    rms = np.sqrt((Fm ** 2).sum(1).mean())
    assert np.abs(Fm.sum(0)).max() <= 1e-5 * rms * np.sqrt(len(Fm))
    assert np.abs(Fd.sum(0)).max() <= 1e-9 * rms * np.sqrt(len(Fd))


def test_step_device_runs_the_ewald_force():
    """The device leapfrog step is potential-agnostic: one step with the
    Ewald force equals kick + drift around an evaluation of it."""
    import torch
    d = load_fixture("ewald_water_ref.npz")
    s = water.small_648()
    topo = PeriodicTopology.from_dict(d)
    f = EwaldRealB200SystemForce(float(d["alpha"]), float(d["accuracy"]), precision="fp64")
    dev = torch.device("cuda", 0)
    pos = torch.tensor(d["pos"], dtype=torch.float64, device=dev)
    vel = torch.tensor(s["vel"], dtype=torch.float64, device=dev)
    frc = torch.zeros_like(pos)
    st = torch.cuda.Stream()
    f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), None, 0, st.cuda_stream)
    st.synchronize()
    f.sync()
    F0 = frc.cpu().numpy()
    f.step_device(topo, pos.data_ptr(), vel.data_ptr(), frc.data_ptr(), 1.0, st.cuda_stream)
    st.synchronize()
    f.sync()
    f.close()
    h = 1.0 * 0.02045482828087295
    m = d["mass"][:, None]
    v1 = s["vel"] + F0 * h / m
    x1 = d["pos"] + v1 * h
    assert np.abs(pos.cpu().numpy() - x1).max() <= 1e-12 * np.abs(x1).max()
    fo, _, _, _ = O.restate_ewald_real(d, x1, float(d["alpha"]), float(d["accuracy"]), False, 0)
    assert rms_rel(frc.cpu().numpy(), fo) <= 1e-11
